// Matrix-free field solve: the implicit Maxwell operator
//   A(v) = v + delta^2 curl_C2N(curl_N2C v) + k (M v)/V
// fused into one kernel per interior node, and restarted GMRES with FP64
// reductions and device-side Givens rotations, restating
// Gmres::host_blocking_solve (ecsim/gmres/gmres_device.hpp:353-454) and its
// kernels (:137-292). TPIC reads two scalars back after every Arnoldi step
// to decide whether to stop; here the decision is taken on the device (an
// ArnoldiControl record the step kernels read and a one-thread kernel
// updates), and the steps of a restart cycle run as one CUDA graph whose
// WHILE node repeats the step until that kernel clears its condition, so the
// host waits once per restart cycle. The stopping rule, and so the
// iteration count, is TPIC's.
//
// The reference applies A in four launches with three intermediate fields
// (N2C curl, C2N curl, M v, combination; ecsim/maxwell/maxwell_device.hpp:433-484).
// Here one thread evaluates the eight cell curls around its node in
// registers, the C2N curl of those, the 27-block mass product and the
// combination ((1*v + delta^2*curl) + k*Mv) in the same arithmetic type and
// order, and stores the image straight into the compact Krylov vector: the
// M records (504 B/node FP32, 1008 B/node FP64) are the only HBM stream.
#include "kernels.cuh"
#include "tcgen05.cuh"

#include <cuda.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <limits>
#include <vector>

namespace tpicb200 {
namespace {

constexpr int kThreads = 256;
constexpr int kDotTile = 8;
// Krylov basis columns start kColumnAlign elements apart (vector loads).
constexpr long long kColumnAlign = 64;
// Largest GMRES restart the context accepts.
constexpr int kMaxRestart = 1024;

// Device-side state of one restart cycle's Arnoldi steps.
struct ArnoldiControl {
  int col;        // the step the step kernels take (0-based)
  int completed;  // steps completed in this cycle
  int columns;    // step limit of this cycle
  int stop;       // 0 running; 1 stopped (tolerance, breakdown or limit); 2 nonfinite estimate
  int breakdown;  // the last step's subdiagonal was zero
  int pad;
  double tolerance;
};

// Interior coordinates of compact index t (32-bit arithmetic: solver_create
// requires 3 (n+1)^3 < 2^31).
__device__ __forceinline__ void compact_coordinates(const Geom& g, long long t, int& i, int& j, int& k) {
  const uint32_t u = uint32_t(t), inx = uint32_t(g.inx), row = u / inx;
  i = int(u - row * inx);
  j = int(row % uint32_t(g.iny));
  k = int(row / uint32_t(g.iny));
}

// curl_N2C at cell (i,j,k) of the double node field `v` in arithmetic C.
template <class C>
__device__ __forceinline__ void cell_curl(const Geom& g, const double* __restrict__ v, int i, int j, int k,
                                          const C inv[3], C out[3]) {
  const long long nn = g.nodes;
  const long long b = g.node(i, j, k), sy = g.NX, sz = (long long)g.NX * g.NY;
  C s[3][8];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const double* p = v + c * nn + b;
    s[c][0] = C(p[0]); s[c][1] = C(p[1]); s[c][2] = C(p[sy]); s[c][3] = C(p[sz]);
    s[c][4] = C(p[1 + sy]); s[c][5] = C(p[1 + sz]); s[c][6] = C(p[sy + sz]); s[c][7] = C(p[1 + sy + sz]);
  }
  auto dx = [&](const C* q) { return C(0.25) * inv[0] * (q[1] - q[0] + (q[5] - q[3]) + (q[4] - q[2]) + (q[7] - q[6])); };
  auto dy = [&](const C* q) { return C(0.25) * inv[1] * (q[2] - q[0] + (q[6] - q[3]) + (q[4] - q[1]) + (q[7] - q[5])); };
  auto dz = [&](const C* q) { return C(0.25) * inv[2] * (q[3] - q[0] + (q[5] - q[1]) + (q[6] - q[2]) + (q[7] - q[4])); };
  out[0] = dy(s[2]) - dz(s[1]);
  out[1] = dz(s[0]) - dx(s[2]);
  out[2] = dx(s[1]) - dy(s[0]);
}

// One 3x3 block times (vx, vy, vz); kTranspose multiplies by the block's
// transpose (the adjoint operator A^T keeps the stencil walk of A and
// transposes every block).
template <class C, class M, bool kTranspose = false>
__device__ __forceinline__ void block_product(const M* __restrict__ b, long long es, C vx, C vy, C vz, C& x, C& y,
                                              C& z) {
  if constexpr (kTranspose) {
    x = vx * C(b[0]) + vy * C(b[3 * es]) + vz * C(b[6 * es]);
    y = vx * C(b[es]) + vy * C(b[4 * es]) + vz * C(b[7 * es]);
    z = vx * C(b[2 * es]) + vy * C(b[5 * es]) + vz * C(b[8 * es]);
  } else {
    x = vx * C(b[0]) + vy * C(b[es]) + vz * C(b[2 * es]);
    y = vx * C(b[3 * es]) + vy * C(b[4 * es]) + vz * C(b[5 * es]);
    z = vx * C(b[6 * es]) + vy * C(b[7 * es]) + vz * C(b[8 * es]);
  }
}

// (M v)_g before the row volume scale: centre, then per stencil the forward
// neighbour with this vertex's block and the backward neighbour with the
// neighbour vertex's block, untransposed (apply_mass_matrix_node,
// ecsim/mass_matrix/mass_matrix_stencil.hpp:119-149).
template <class C, class M>
__device__ __forceinline__ void mass_product(const Geom& g, const M* __restrict__ mass,
                                             const double* __restrict__ v, int i, int j, int k, C out[3]) {
  const long long nn = g.nodes;
  const long long at = g.node(i, j, k), mat = g.mass_vertex(i, j, k);
  C x, y, z;
  const long long es = g.mes;
  block_product<C>(mass + g.mass_index(mat, 0), es, C(v[at]), C(v[nn + at]), C(v[2 * nn + at]), x, y, z);
#pragma unroll
  for (int s = 1; s < 14; ++s) {
    const long long d = stencil_offset(s, 0) + (long long)g.NX * (stencil_offset(s, 1) + (long long)g.NY * stencil_offset(s, 2));
    const long long md = g.mass_offset(stencil_offset(s, 0), stencil_offset(s, 1), stencil_offset(s, 2));
    C bx, by, bz;
    const long long f = at + d, b = at - d;
    block_product<C>(mass + g.mass_index(mat, s * 9), es, C(v[f]), C(v[nn + f]), C(v[2 * nn + f]), bx, by, bz);
    x += bx; y += by; z += bz;
    block_product<C>(mass + g.mass_index(mat - md, s * 9), es, C(v[b]), C(v[nn + b]), C(v[2 * nn + b]), bx, by, bz);
    x += bx; y += by; z += bz;
  }
  out[0] = x; out[1] = y; out[2] = z;
}

// Tile of unique nodes per CTA, 256 threads: 32 (x) x 4 (y) x 2 (z), or
// 32 x 8 x 1 on grids of one cell along z, where a second z layer would hold
// no node (when that leaves enough CTAs to fill the GPU).
constexpr int kTX = 32, kTY = 4, kTZ = 2;
constexpr int kThinTY = 8;

// A(v) over the unique nodes [0,n)^3 of a tile. The input (ghosts filled) is
// staged in shared memory with its one-node halo, each cell curl the tile
// needs is computed once into shared memory, then every thread forms its
// node's C2N curl, 27-block mass product and combination. Rows of the
// duplicate endpoint planes equal their unique node's row (same inputs, same
// operations) and are copied by duplicate_rows_kernel. Registers are bounded
// for four CTAs per SM in float (64) and three in double (85).
template <class C, class M, class Out, int TX, int TY, int TZ, bool kResponse = false, bool kTranspose = false>
__global__ void __launch_bounds__(TX * TY * TZ, sizeof(C) == 4 ? 4 : 3) maxwell_apply_kernel(Geom g, C d2, C kfac, C inv_volume,
                                                                        const M* __restrict__ mass,
                                                                        const double* __restrict__ v,
                                                                        Out* __restrict__ out,
                                                                        const double* __restrict__ response) {
  wait_for_predecessor();
  constexpr int VX = TX + 2, VY = TY + 2, VZ = TZ + 2;   // nodes i0-1 .. i0+TX
  constexpr int CX = TX + 1, CY = TY + 1, CZ = TZ + 1;   // cells i0-1 .. i0+TX-1
  __shared__ C vs[3][VZ][VY][VX];
  __shared__ C cs[3][CZ][CY][CX];
  const C inv[3] = {C(g.inv[0]), C(g.inv[1]), C(g.inv[2])};
  const int tiles_x = (g.nx + TX - 1) / TX, tiles_y = (g.ny + TY - 1) / TY;
  const int tx = blockIdx.x % tiles_x, ty = (blockIdx.x / tiles_x) % tiles_y, tz = blockIdx.x / (tiles_x * tiles_y);
  const int i0 = tx * TX, j0 = ty * TY, k0 = tz * TZ;
  const long long nn = g.nodes;
  // The centre block and the first stencil's forward and backward rows of
  // this thread's node are requested into L2 before the staging below, so
  // the mass stream is in flight while v and the curls are staged.
  if constexpr (!kResponse) {
    const int pi = i0 + int(threadIdx.x % TX), pj = j0 + int((threadIdx.x / TX) % TY),
              pk = k0 + int(threadIdx.x / (TX * TY));
    if (pi < g.nx && pj < g.ny && pk < g.nz) {
      const long long pat = g.mass_vertex(pi, pj, pk);
      const long long d1 = g.mass_offset(stencil_offset(1, 0), stencil_offset(1, 1), stencil_offset(1, 2));
#pragma unroll
      for (int e = 0; e < 9; ++e) {
        prefetch_l2(mass + g.mass_index(pat, e));
        prefetch_l2(mass + g.mass_index(pat, 9 + e));
        prefetch_l2(mass + g.mass_index(pat - d1, 9 + e));
      }
    }
  }
  // Stage v over nodes [i0-1, i0+TX] x [j0-1, j0+TY] x [k0-1, k0+TZ]; nodes
  // beyond n+1 (partial tiles) are never read by a live node and load 0.
  for (int t = threadIdx.x; t < 3 * VZ * VY * VX; t += blockDim.x) {
    const int c = t / (VZ * VY * VX), r = t % (VZ * VY * VX);
    const int lx = r % VX, ly = (r / VX) % VY, lz = r / (VX * VY);
    const int i = i0 - 1 + lx, j = j0 - 1 + ly, k = k0 - 1 + lz;
    C val = C(0);
    if (i <= g.nx + 1 && j <= g.ny + 1 && k <= g.nz + 1) val = C(v[c * nn + g.node(i, j, k)]);
    vs[c][lz][ly][lx] = val;
  }
  __syncthreads();
  // Cell curls (curl_N2C, ecsim/fields/node_cell_curl.hpp:116-126) of cells
  // [i0-1, i0+TX-1] x ... from the staged nodes.
  for (int t = threadIdx.x; t < CZ * CY * CX; t += blockDim.x) {
    const int lx = t % CX, ly = (t / CX) % CY, lz = t / (CX * CY);
    C q[3][8];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      q[c][0] = vs[c][lz][ly][lx];         q[c][1] = vs[c][lz][ly][lx + 1];
      q[c][2] = vs[c][lz][ly + 1][lx];     q[c][3] = vs[c][lz + 1][ly][lx];
      q[c][4] = vs[c][lz][ly + 1][lx + 1]; q[c][5] = vs[c][lz + 1][ly][lx + 1];
      q[c][6] = vs[c][lz + 1][ly + 1][lx]; q[c][7] = vs[c][lz + 1][ly + 1][lx + 1];
    }
    auto dx = [&](const C* p) { return C(0.25) * inv[0] * (p[1] - p[0] + (p[5] - p[3]) + (p[4] - p[2]) + (p[7] - p[6])); };
    auto dy = [&](const C* p) { return C(0.25) * inv[1] * (p[2] - p[0] + (p[6] - p[3]) + (p[4] - p[1]) + (p[7] - p[5])); };
    auto dz = [&](const C* p) { return C(0.25) * inv[2] * (p[3] - p[0] + (p[5] - p[1]) + (p[6] - p[2]) + (p[7] - p[4])); };
    // The cell curl is stored in the solver storage (double) between the two
    // curls of the reference; a float curl survives that round trip exactly.
    cs[0][lz][ly][lx] = C(double(dy(q[2]) - dz(q[1])));
    cs[1][lz][ly][lx] = C(double(dz(q[0]) - dx(q[2])));
    cs[2][lz][ly][lx] = C(double(dx(q[1]) - dy(q[0])));
  }
  __syncthreads();
  const int lx = threadIdx.x % TX, ly = (threadIdx.x / TX) % TY, lz = threadIdx.x / (TX * TY);
  const int i = i0 + lx, j = j0 + ly, k = k0 + lz;
  if (i >= g.nx || j >= g.ny || k >= g.nz) return;
  // C2N curl of the cell curls (cell sources: anchor - neighbour); the cell
  // (i-a, j-b, k-c) of the reference's samples is cs[..][lz+1-c][ly+1-b][lx+1-a].
  C curl2[3];
  {
    C p[3][8];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      p[c][0] = cs[c][lz + 1][ly + 1][lx + 1]; p[c][1] = cs[c][lz + 1][ly + 1][lx];
      p[c][2] = cs[c][lz + 1][ly][lx + 1];     p[c][3] = cs[c][lz][ly + 1][lx + 1];
      p[c][4] = cs[c][lz + 1][ly][lx];         p[c][5] = cs[c][lz][ly + 1][lx];
      p[c][6] = cs[c][lz][ly][lx + 1];         p[c][7] = cs[c][lz][ly][lx];
    }
    auto dx = [&](const C* q) { return C(0.25) * inv[0] * (q[0] - q[1] + (q[3] - q[5]) + (q[2] - q[4]) + (q[6] - q[7])); };
    auto dy = [&](const C* q) { return C(0.25) * inv[1] * (q[0] - q[2] + (q[3] - q[6]) + (q[1] - q[4]) + (q[5] - q[7])); };
    auto dz = [&](const C* q) { return C(0.25) * inv[2] * (q[0] - q[3] + (q[1] - q[5]) + (q[2] - q[6]) + (q[4] - q[7])); };
    curl2[0] = dy(p[2]) - dz(p[1]);
    curl2[1] = dz(p[0]) - dx(p[2]);
    curl2[2] = dx(p[1]) - dy(p[0]);
  }
  // With smoothing (kResponse) the mass term is the smoothed response node
  // field S^n(M S^n v) / V, read in the apply arithmetic (combine_image,
  // maxwell_device.hpp:420-432).
  if constexpr (kResponse) {
    const long long at = g.node(i, j, k);
    const long long row = i + (long long)g.inx * (j + (long long)g.iny * k);
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const C m = C(response[c * nn + at]);
      const C value = (C(1) * vs[c][lz + 1][ly + 1][lx + 1] + d2 * C(double(curl2[c]))) + kfac * m;
      out[c * g.interior + row] = Out(value);
    }
    return;
  }
  // Mass product: centre, then forward and backward blocks per stencil,
  // untransposed (apply_mass_matrix_node, mass_matrix_stencil.hpp:119-149).
  const long long at = g.mass_vertex(i, j, k), es = g.mes;
  auto vv = [&](int c, int a, int b, int d) { return vs[c][lz + 1 + d][ly + 1 + b][lx + 1 + a]; };
  C x, y, z;
  block_product<C, M, kTranspose>(mass + g.mass_index(at, 0), es, vv(0, 0, 0, 0), vv(1, 0, 0, 0), vv(2, 0, 0, 0), x,
                                  y, z);
#pragma unroll
  for (int s = 1; s < 14; ++s) {
    const int ox = stencil_offset(s, 0), oy = stencil_offset(s, 1), oz = stencil_offset(s, 2);
    const long long d = g.mass_offset(ox, oy, oz);
    // The next stencil's forward and backward rows are requested into L2
    // while this one is applied: the loads of a block then wait for L2, not
    // for HBM (the kernel is bound by memory latency; prefetches hold no
    // registers).
    if (s + 1 < 14) {
      const int sn = s + 1;
      const long long dn = g.mass_offset(stencil_offset(sn, 0), stencil_offset(sn, 1), stencil_offset(sn, 2));
#pragma unroll
      for (int e = 0; e < 9; ++e) {
        prefetch_l2(mass + g.mass_index(at, sn * 9 + e));
        prefetch_l2(mass + g.mass_index(at - dn, sn * 9 + e));
      }
    }
    C bx, by, bz;
    block_product<C, M, kTranspose>(mass + g.mass_index(at, s * 9), es, vv(0, ox, oy, oz), vv(1, ox, oy, oz),
                                    vv(2, ox, oy, oz), bx, by, bz);
    x += bx; y += by; z += bz;
    block_product<C, M, kTranspose>(mass + g.mass_index(at - d, s * 9), es, vv(0, -ox, -oy, -oz),
                                    vv(1, -ox, -oy, -oz), vv(2, -ox, -oy, -oz), bx, by, bz);
    x += bx; y += by; z += bz;
  }
  const C mv[3] = {x, y, z};
  const long long row = i + (long long)g.inx * (j + (long long)g.iny * k);
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    // The mass image is narrowed to the solver storage (double) before the
    // combination reads it back (maxwell_device.hpp:424-429,471-484).
    const C m = C(double(mv[c] * inv_volume));
    const C value = (C(1) * vv(c, 0, 0, 0) + d2 * C(double(curl2[c]))) + kfac * m;
    out[c * g.interior + row] = Out(value);
  }
}

// A(v) with the mass rows staged by tensor-memory-access (TMA) copies, for
// mass buffers whose rows start on 16-byte boundaries (the tiled layout).
// Per stencil s = (ox, oy, oz) one 4-D box of the mass tensor (x, y, z,
// entry) holds the stencil's 9 entries over the tile plus a one-node halo
// on the side of -s: x elements i0 .. i0+35 (nodes i0-1 .. i0+34; element
// i0 is 16-byte aligned), y nodes j0 - max(oy,0) .. + TY, z likewise. The
// forward block of a node (at the node) and its backward block (at the
// node - s) are both in that box. The boxes stream through S stages with one
// mbarrier each; one thread issues the copies (after the kernel's
// predecessor has completed), every thread waits (bounded) for a stage's
// copy, and the stage is refilled with stencil s + S after a CTA barrier. The
// input v and the cell curls are staged as in maxwell_apply_kernel, and every
// sum runs in the same order, so the result equals it bit for bit. A copy
// that does not arrive within `polls` polls adds 1 << 21 to *invalid; the
// CTA then waits (with the default bound) for its copies in flight and
// returns without writing its rows.
constexpr int kBoxX = 36;

// Flat: a grid one cell thick along z (thin tiles). Every block a node of
// plane 0 needs is then in plane 0: the planes -1 and 1 are the fold's copies
// of it, so the box holds that plane alone and the products are unchanged bit
// for bit, with half the mass bytes read.
template <int TY, int TZ, class M, bool Flat = false> struct TmaBox {
  static constexpr int X = kBoxX, Y = TY + 1, Z = Flat ? 1 : TZ + 1;
  static constexpr int entry = X * Y * Z;              // elements of one entry's box
  static constexpr int elems = 9 * entry;              // one stencil's box
  static constexpr int bytes = elems * int(sizeof(M));
  static constexpr int stage = (bytes + 1023) / 1024 * 1024;  // 1024-byte aligned stages
};

template <class C, class M, int TX, int TY, int TZ, int S, bool Flat = false>
struct TmaApplyShared {
  static constexpr int VX = TX + 2, VY = TY + 2, VZ = TZ + 2;
  static constexpr int CX = TX + 1, CY = TY + 1, CZ = TZ + 1;
  static constexpr int stages = S * TmaBox<TY, TZ, M, Flat>::stage;
  static constexpr int bars = stages;                              // S + 1 mbarriers
  static constexpr int vs = (bars + (S + 1) * 8 + 15) / 16 * 16;   // C [3][VZ][VY][VX]
  static constexpr int cs = vs + 3 * VZ * VY * VX * int(sizeof(C));  // C [3][CZ][CY][CX]
  static constexpr int total = cs + 3 * CZ * CY * CX * int(sizeof(C));
};

template <class C, class M, class Out, int TX, int TY, int TZ, int S, bool kTranspose, bool kFlat>
__global__ void __launch_bounds__(TX * TY * TZ, sizeof(C) == 4 ? 4 : 2)
    maxwell_apply_tma_kernel(const __grid_constant__ CUtensorMap map, Geom g, C d2, C kfac, C inv_volume,
                             const double* __restrict__ v, Out* __restrict__ out, uint32_t* invalid,
                             uint32_t polls, int stall) {
  static_assert(!kFlat || TZ == 1, "flat boxes hold one z plane");
  using Box = TmaBox<TY, TZ, M, kFlat>;
  using L = TmaApplyShared<C, M, TX, TY, TZ, S, kFlat>;
  constexpr int VX = L::VX, VY = L::VY, VZ = L::VZ, CX = L::CX, CY = L::CY, CZ = L::CZ;
  extern __shared__ __align__(1024) uint8_t tma_smem[];
  uint64_t* bars = reinterpret_cast<uint64_t*>(tma_smem + L::bars);  // S stage barriers, then `never`
  auto vs = reinterpret_cast<C (*)[VZ][VY][VX]>(tma_smem + L::vs);
  auto cs = reinterpret_cast<C (*)[CZ][CY][CX]>(tma_smem + L::cs);
  const C inv[3] = {C(g.inv[0]), C(g.inv[1]), C(g.inv[2])};
  const int tiles_x = (g.nx + TX - 1) / TX, tiles_y = (g.ny + TY - 1) / TY;
  const int tx = blockIdx.x % tiles_x, ty = (blockIdx.x / tiles_x) % tiles_y, tz = blockIdx.x / (tiles_x * tiles_y);
  const int i0 = tx * TX, j0 = ty * TY, k0 = tz * TZ;
  const long long nn = g.nodes;
  auto issue = [&](int s) {
    const int oy = stencil_offset(s, 1), oz = stencil_offset(s, 2);
    uint64_t* bar = &bars[s % S];
    tc::mbar_arrive_expect_tx(bar, uint32_t(Box::bytes));
    tc::tma_load_4d(tma_smem + (s % S) * Box::stage, &map, i0, j0 + 1 - (oy > 0 ? oy : 0),
                    kFlat ? k0 + 1 : k0 + 1 - (oz > 0 ? oz : 0), 9 * s, bar);
  };
  if (threadIdx.x == 0) {
#pragma unroll
    for (int b = 0; b <= S; ++b) tc::mbar_init(&bars[b], 1);
    tc::fence_mbar_init();
  }
  __syncthreads();
  wait_for_predecessor();
  if (threadIdx.x == 0) {
#pragma unroll
    for (int s = 0; s < S; ++s) issue(s);
  }
  // Stage v over nodes [i0-1, i0+TX] x [j0-1, j0+TY] x [k0-1, k0+TZ]; nodes
  // beyond n+1 (partial tiles) are never read by a live node and load 0.
  for (int t = threadIdx.x; t < 3 * VZ * VY * VX; t += blockDim.x) {
    const int c = t / (VZ * VY * VX), r = t % (VZ * VY * VX);
    const int lx = r % VX, ly = (r / VX) % VY, lz = r / (VX * VY);
    const int i = i0 - 1 + lx, j = j0 - 1 + ly, k = k0 - 1 + lz;
    C val = C(0);
    if (i <= g.nx + 1 && j <= g.ny + 1 && k <= g.nz + 1) val = C(v[c * nn + g.node(i, j, k)]);
    vs[c][lz][ly][lx] = val;
  }
  __syncthreads();
  for (int t = threadIdx.x; t < CZ * CY * CX; t += blockDim.x) {
    const int lx = t % CX, ly = (t / CX) % CY, lz = t / (CX * CY);
    C q[3][8];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      q[c][0] = vs[c][lz][ly][lx];         q[c][1] = vs[c][lz][ly][lx + 1];
      q[c][2] = vs[c][lz][ly + 1][lx];     q[c][3] = vs[c][lz + 1][ly][lx];
      q[c][4] = vs[c][lz][ly + 1][lx + 1]; q[c][5] = vs[c][lz + 1][ly][lx + 1];
      q[c][6] = vs[c][lz + 1][ly + 1][lx]; q[c][7] = vs[c][lz + 1][ly + 1][lx + 1];
    }
    auto dx = [&](const C* p) { return C(0.25) * inv[0] * (p[1] - p[0] + (p[5] - p[3]) + (p[4] - p[2]) + (p[7] - p[6])); };
    auto dy = [&](const C* p) { return C(0.25) * inv[1] * (p[2] - p[0] + (p[6] - p[3]) + (p[4] - p[1]) + (p[7] - p[5])); };
    auto dz = [&](const C* p) { return C(0.25) * inv[2] * (p[3] - p[0] + (p[5] - p[1]) + (p[6] - p[2]) + (p[7] - p[4])); };
    cs[0][lz][ly][lx] = C(double(dy(q[2]) - dz(q[1])));
    cs[1][lz][ly][lx] = C(double(dz(q[0]) - dx(q[2])));
    cs[2][lz][ly][lx] = C(double(dx(q[1]) - dy(q[0])));
  }
  __syncthreads();
  const int lx = threadIdx.x % TX, ly = (threadIdx.x / TX) % TY, lz = threadIdx.x / (TX * TY);
  const int i = i0 + lx, j = j0 + ly, k = k0 + lz;
  const bool live = i < g.nx && j < g.ny && k < g.nz;
  C curl2[3] = {C(0), C(0), C(0)};
  if (live) {
    C p[3][8];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      p[c][0] = cs[c][lz + 1][ly + 1][lx + 1]; p[c][1] = cs[c][lz + 1][ly + 1][lx];
      p[c][2] = cs[c][lz + 1][ly][lx + 1];     p[c][3] = cs[c][lz][ly + 1][lx + 1];
      p[c][4] = cs[c][lz + 1][ly][lx];         p[c][5] = cs[c][lz][ly + 1][lx];
      p[c][6] = cs[c][lz][ly][lx + 1];         p[c][7] = cs[c][lz][ly][lx];
    }
    auto dx = [&](const C* q) { return C(0.25) * inv[0] * (q[0] - q[1] + (q[3] - q[5]) + (q[2] - q[4]) + (q[6] - q[7])); };
    auto dy = [&](const C* q) { return C(0.25) * inv[1] * (q[0] - q[2] + (q[3] - q[6]) + (q[1] - q[4]) + (q[5] - q[7])); };
    auto dz = [&](const C* q) { return C(0.25) * inv[2] * (q[0] - q[3] + (q[1] - q[5]) + (q[2] - q[6]) + (q[4] - q[7])); };
    curl2[0] = dy(p[2]) - dz(p[1]);
    curl2[1] = dz(p[0]) - dx(p[2]);
    curl2[2] = dx(p[1]) - dy(p[0]);
  }
  auto vv = [&](int c, int a, int b, int d) { return vs[c][lz + 1 + d][ly + 1 + b][lx + 1 + a]; };
  C x = C(0), y = C(0), z = C(0);
  bool failed = false;
  int consumed = 0;
  // Unrolled (the stencil offsets fold into constants); `failed` is uniform
  // over the CTA, so the barriers below are reached by every thread.
#pragma unroll
  for (int s = 0; s < 14; ++s) {
    if (failed) continue;
    // stall == s (a test of the bound) waits on bars[S], which nothing
    // arrives on.
    const bool ok = s == stall ? tc::mbar_wait(&bars[S], 0u, polls)
                               : tc::mbar_wait(&bars[s % S], uint32_t((s / S) & 1), polls);
    if (__syncthreads_or(!ok)) {
      failed = true;
      continue;
    }
    consumed = s + 1;
    if (live) {
      const M* box = reinterpret_cast<const M*>(tma_smem + (s % S) * Box::stage);
      const int ox = stencil_offset(s, 0), oy = stencil_offset(s, 1), oz = stencil_offset(s, 2);
      const int my = oy > 0 ? oy : 0, mz = oz > 0 ? oz : 0;
      const int fwd = (lx + 1) + Box::X * ((ly + my) + Box::Y * (kFlat ? 0 : lz + mz));
      if (s == 0) {
        block_product<C, M, kTranspose>(box + fwd, Box::entry, vv(0, 0, 0, 0), vv(1, 0, 0, 0), vv(2, 0, 0, 0), x, y, z);
      } else {
        const int bwd = (lx + 1 - ox) + Box::X * ((ly - oy + my) + Box::Y * (kFlat ? 0 : lz - oz + mz));
        C bx, by, bz;
        block_product<C, M, kTranspose>(box + fwd, Box::entry, vv(0, ox, oy, oz), vv(1, ox, oy, oz),
                                        vv(2, ox, oy, oz), bx, by, bz);
        x += bx; y += by; z += bz;
        block_product<C, M, kTranspose>(box + bwd, Box::entry, vv(0, -ox, -oy, -oz), vv(1, -ox, -oy, -oz),
                                        vv(2, -ox, -oy, -oz), bx, by, bz);
        x += bx; y += by; z += bz;
      }
    }
    __syncthreads();
    if (threadIdx.x == 0 && s + S < 14) {
      tc::fence_proxy_async_smem();
      issue(s + S);
    }
  }
  if (failed) {
    // Copies issued but not consumed may still land: wait for them (with the
    // default bound) before the CTA's shared memory is released.
    if (threadIdx.x == 0) {
      if (invalid) atomicAdd(invalid, 1u << 21);
      for (int s = consumed; s < 14 && s < consumed + S; ++s)
        tc::mbar_wait(&bars[s % S], uint32_t((s / S) & 1), kDefaultWaitPolls);
    }
    __syncthreads();
    return;
  }
  if (!live) return;
  const C mv[3] = {x, y, z};
  const long long row = i + (long long)g.inx * (j + (long long)g.iny * k);
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const C m = C(double(mv[c] * inv_volume));
    const C value = (C(1) * vv(c, 0, 0, 0) + d2 * C(double(curl2[c]))) + kfac * m;
    out[c * g.interior + row] = Out(value);
  }
}

// Rows of the duplicate endpoint planes (index n on some axis) copy the row
// of their periodic unique node.
template <class Out>
__global__ void __launch_bounds__(kThreads) duplicate_rows_kernel(Geom g, Out* __restrict__ out) {
  wait_for_predecessor();
  // Compact rows with i == n, or j == n, or k == n: three slabs as in shell_coordinates.
  const uint32_t zs = uint32_t(g.inx) * g.iny, ys = uint32_t(g.inx) * g.nz, xs = uint32_t(g.ny) * g.nz;
  const uint32_t total = zs + ys + xs;
  for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < 3 * total; t += gridDim.x * blockDim.x) {
    const int c = int(t / total);
    uint32_t r = t - c * total;
    int i, j, k;
    if (r < zs) { k = g.nz; i = int(r % g.inx); j = int(r / g.inx); }
    else if ((r -= zs) < ys) { j = g.ny; i = int(r % g.inx); k = int(r / g.inx); }
    else { r -= ys; i = g.nx; j = int(r % g.ny); k = int(r / g.ny); }
    const int ui = i == g.nx ? 0 : i, uj = j == g.ny ? 0 : j, uk = k == g.nz ? 0 : k;
    out[c * g.interior + i + (long long)g.inx * (j + (long long)g.iny * k)] =
        out[c * g.interior + ui + (long long)g.inx * (uj + (long long)g.iny * uk)];
  }
}

// The mass response of a node field with filled ghosts over the interior
// nodes 0..n, in arithmetic C, stored (M v)/V in double
// (enqueue_mass_response of the smoothed schedule, maxwell_device.hpp:413-414).
template <class C, class M>
__global__ void __launch_bounds__(kThreads) mass_image_kernel(Geom g, C inv_volume, const M* __restrict__ mass,
                                                             const double* __restrict__ v, double* __restrict__ out) {
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < g.interior;
       t += (long long)gridDim.x * blockDim.x) {
    int i, j, k;
    compact_coordinates(g, t, i, j, k);
    C mv[3];
    mass_product<C>(g, mass, v, i, j, k, mv);
    const long long at = g.node(i, j, k);
#pragma unroll
    for (int c = 0; c < 3; ++c) out[c * g.nodes + at] = double(mv[c] * inv_volume);
  }
}

template <class M>
__global__ void __launch_bounds__(kThreads) mass_apply_kernel(Geom g, double inv_volume, const M* __restrict__ mass,
                                                              const double* __restrict__ v, double* __restrict__ out) {
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < g.interior;
       t += (long long)gridDim.x * blockDim.x) {
    int i, j, k;
    compact_coordinates(g, t, i, j, k);
    double mv[3];
    mass_product<double>(g, mass, v, i, j, k, mv);
    const long long at = g.node(i, j, k);
#pragma unroll
    for (int c = 0; c < 3; ++c) out[c * g.nodes + at] = mv[c] * inv_volume;
  }
}

// Compact vector <-> node field interiors (gmres_field_vector_transfer_kernel,
// gmres_device.hpp:137-157).
template <class V>
__global__ void __launch_bounds__(kThreads) pack_kernel(Geom g, const double* __restrict__ f, V* __restrict__ vec) {
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < g.interior;
       t += (long long)gridDim.x * blockDim.x) {
    int i, j, k;
    compact_coordinates(g, t, i, j, k);
    const long long at = g.node(i, j, k);
#pragma unroll
    for (int c = 0; c < 3; ++c) vec[c * g.interior + t] = V(f[c * g.nodes + at]);
  }
}
template <class V>
__global__ void __launch_bounds__(kThreads) unpack_kernel(Geom g, const V* __restrict__ vec, double* __restrict__ f) {
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < g.interior;
       t += (long long)gridDim.x * blockDim.x) {
    int i, j, k;
    compact_coordinates(g, t, i, j, k);
    const long long at = g.node(i, j, k);
#pragma unroll
    for (int c = 0; c < 3; ++c) f[c * g.nodes + at] = double(vec[c * g.interior + t]);
  }
}
template <class T>
__global__ void __launch_bounds__(kThreads) pack_storage_kernel(Geom g, const T* __restrict__ f, double* __restrict__ vec) {
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < g.interior;
       t += (long long)gridDim.x * blockDim.x) {
    int i, j, k;
    compact_coordinates(g, t, i, j, k);
    const long long at = g.node(i, j, k);
#pragma unroll
    for (int c = 0; c < 3; ++c) vec[c * g.interior + t] = double(f[c * g.nodes + at]);
  }
}

// Four consecutive elements of a basis column or of the image (16-byte
// aligned: columns are kColumnAlign elements apart), widened to double.
struct Quad {
  double v[4];
};
__device__ __forceinline__ Quad load_quad(const float* p) {
  const float4 q = *reinterpret_cast<const float4*>(p);
  return Quad{{q.x, q.y, q.z, q.w}};
}
__device__ __forceinline__ Quad load_quad(const double* p) {
  const double2 a = reinterpret_cast<const double2*>(p)[0], b = reinterpret_cast<const double2*>(p)[1];
  return Quad{{a.x, a.y, b.x, b.y}};
}
__device__ __forceinline__ void store_quad(float* p, const float (&v)[4]) {
  *reinterpret_cast<float4*>(p) = make_float4(v[0], v[1], v[2], v[3]);
}
__device__ __forceinline__ void store_quad(double* p, const double (&v)[4]) {
  reinterpret_cast<double2*>(p)[0] = make_double2(v[0], v[1]);
  reinterpret_cast<double2*>(p)[1] = make_double2(v[2], v[3]);
}

// Dots of `image` with basis columns [first, first + kDotTile) per block row,
// block partials per column (gmres_dot_batch_kernel, gmres_device.hpp:163-192).
// Each thread takes four consecutive elements at a time (one 16-byte load per
// column); the `count % 4` tail elements go to the first threads. Columns
// are `ld` elements apart.
template <class S>
__global__ void __launch_bounds__(kThreads) dot_batch_kernel(const S* __restrict__ basis, const S* __restrict__ image,
                                                             double* __restrict__ partials, long long count,
                                                             long long ld, const ArnoldiControl* __restrict__ ctl) {
  wait_for_predecessor();
  __shared__ double scratch[kDotTile][kThreads / 32];
  const int columns = ctl->col + 1;
  const long long quads = count >> 2, stride = (long long)gridDim.x * blockDim.x;
  const long long start = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  for (int first = blockIdx.y * kDotTile; first < columns; first += gridDim.y * kDotTile) {
    const int tile = min(kDotTile, columns - first);
    const S* col = basis + (long long)first * ld;
    double sum[kDotTile];
#pragma unroll
    for (int r = 0; r < kDotTile; ++r) sum[r] = 0.0;
    for (long long q = start; q < quads; q += stride) {
      const Quad x = load_quad(image + 4 * q);
#pragma unroll
      for (int r = 0; r < kDotTile; ++r)
        if (r < tile) {
          const Quad b = load_quad(col + r * ld + 4 * q);
#pragma unroll
          for (int e = 0; e < 4; ++e) sum[r] += b.v[e] * x.v[e];
        }
    }
    const long long tail = 4 * quads + start;
    if (tail < count) {
      const double value = double(image[tail]);
#pragma unroll
      for (int r = 0; r < kDotTile; ++r)
        if (r < tile) sum[r] += double(col[r * ld + tail]) * value;
    }
#pragma unroll
    for (int r = 0; r < kDotTile; ++r)
      if (r < tile) {
        const double total = block_sum<kThreads>(sum[r], scratch[r]);
        if (threadIdx.x == 0) partials[(long long)(first + r) * gridDim.x + blockIdx.x] = total;
      }
    __syncthreads();
  }
}

// r = b - image with block partials of |r|^2 (and |b|^2)
// (gmres_residual_squared_norm_kernel, gmres_device.hpp:197-216).
template <bool RhsNorm>
__global__ void __launch_bounds__(kThreads) residual_kernel(const double* __restrict__ b, const double* __restrict__ image,
                                                            double* __restrict__ r, double* __restrict__ partials,
                                                            long long count) {
  __shared__ double scratch[2][kThreads / 32];
  double s0 = 0, s1 = 0;
  for (long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x; n < count;
       n += (long long)gridDim.x * blockDim.x) {
    const double bv = b[n];
    const double value = bv - image[n];
    r[n] = value;
    s0 += value * value;
    if (RhsNorm) s1 += bv * bv;
  }
  s0 = block_sum<kThreads>(s0, scratch[0]);
  if (RhsNorm) s1 = block_sum<kThreads>(s1, scratch[1]);
  if (threadIdx.x == 0) {
    partials[blockIdx.x] = s0;
    if (RhsNorm) partials[gridDim.x + blockIdx.x] = s1;
  }
}

// Classical Gram-Schmidt with the reduced dots, squared-norm partials of the
// stored result; block 0 copies the dots into the Hessenberg column
// (gmres_orthogonalize_squared_norm_kernel, gmres_device.hpp:243-263).
// Every element subtracts the columns in order 0, 1, ...; a thread takes four
// consecutive elements at a time (16-byte loads, the columns' loads issued
// four at once), the `count % 4` tail elements go to the first threads.
template <class S>
__global__ void __launch_bounds__(kThreads) orthogonalize_kernel(const S* __restrict__ basis, const double* __restrict__ dots,
                                                                 S* __restrict__ image, double* __restrict__ hessenberg,
                                                                 int leading, double* __restrict__ partials,
                                                                 long long count, long long ld,
                                                                 const ArnoldiControl* __restrict__ ctl) {
  wait_for_predecessor();
  __shared__ double scratch[kThreads / 32];
  __shared__ double h[kMaxRestart + 1];
  const int columns = ctl->col + 1;
  for (int c = threadIdx.x; c < columns; c += blockDim.x) h[c] = dots[c];
  __syncthreads();
  double* column = hessenberg + (long long)ctl->col * leading;
  double norm2 = 0;
  const long long quads = count >> 2, stride = (long long)gridDim.x * blockDim.x;
  const long long start = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  for (long long q = start; q < quads; q += stride) {
    const Quad x = load_quad(image + 4 * q);
    double value[4] = {x.v[0], x.v[1], x.v[2], x.v[3]};
    int c = 0;
    for (; c + 4 <= columns; c += 4) {
      Quad b[4];
#pragma unroll
      for (int r = 0; r < 4; ++r) b[r] = load_quad(basis + (long long)(c + r) * ld + 4 * q);
#pragma unroll
      for (int r = 0; r < 4; ++r)
#pragma unroll
        for (int e = 0; e < 4; ++e) value[e] -= h[c + r] * b[r].v[e];
    }
    for (; c < columns; ++c) {
      const Quad b = load_quad(basis + (long long)c * ld + 4 * q);
#pragma unroll
      for (int e = 0; e < 4; ++e) value[e] -= h[c] * b.v[e];
    }
    S stored[4];
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      stored[e] = S(value[e]);
      norm2 += double(stored[e]) * double(stored[e]);
    }
    store_quad(image + 4 * q, stored);
  }
  const long long tail = 4 * quads + start;
  if (tail < count) {
    double value = double(image[tail]);
    for (int c = 0; c < columns; ++c) value -= h[c] * double(basis[(long long)c * ld + tail]);
    const S stored = S(value);
    image[tail] = stored;
    norm2 += double(stored) * double(stored);
  }
  if (blockIdx.x == 0 && threadIdx.x == 0)
    for (int row = 0; row < columns; ++row) column[row] = h[row];
  const double total = block_sum<kThreads>(norm2, scratch);
  if (threadIdx.x == 0) partials[blockIdx.x] = total;
}

struct ArnoldiTail {
  double* column;  // the Hessenberg matrix (column `step` at step * leading)
  double* cosine;
  double* sine;
  double* rhs;
  double* status;
  int step;        // -1: restart tail (rhs[0] = norm)
  int leading;
};

// Restart tail and Arnoldi least-squares update
// (RestartRhsTail / ArnoldiLeastSquaresUpdate, gmres_device.hpp:52-98).
__device__ void run_tail(const ArnoldiTail& t, double norm2) {
  if (t.step < 0) {
    t.rhs[0] = sqrt(norm2);
    return;
  }
  const int step = t.step;
  const double sub = sqrt(norm2);
  double* column = t.column + (long long)step * t.leading;
  column[step + 1] = sub;
  for (int row = 0; row < step; ++row) {
    const double upper = column[row], lower = column[row + 1];
    column[row] = t.cosine[row] * upper + t.sine[row] * lower;
    column[row + 1] = -t.sine[row] * upper + t.cosine[row] * lower;
  }
  const double diagonal = column[step];
  const double den = hypot(diagonal, sub);
  const double c = den != 0.0 ? diagonal / den : 1.0;
  const double s = den != 0.0 ? sub / den : 0.0;
  t.cosine[step] = c;
  t.sine[step] = s;
  column[step] = c * diagonal + s * sub;
  column[step + 1] = 0.0;
  const double upper = t.rhs[step], lower = t.rhs[step + 1];
  t.rhs[step] = c * upper + s * lower;
  t.rhs[step + 1] = -s * upper + c * lower;
  t.status[0] = fabs(t.rhs[step + 1]);
  t.status[1] = sub == 0.0 ? 1.0 : 0.0;
}

// target = source / sqrt(norm2[0]) (zero for a zero norm), also stored into
// the operator input field (gmres_normalize_kernel, gmres_device.hpp:224-237).
// With `ctl`, the step's column: target is basis column ctl->col + 1 of
// `target` (columns `stride` apart) and the tail runs step ctl->col.
template <class Src, class S>
__global__ void __launch_bounds__(kThreads) normalize_kernel(Geom g, const Src* __restrict__ source,
                                                             const double* __restrict__ norm2, S* __restrict__ target,
                                                             long long stride, double* __restrict__ input,
                                                             ArnoldiTail tail, const ArnoldiControl* __restrict__ ctl) {
  wait_for_predecessor();
  if (ctl) {
    tail.step = ctl->col;
    target += (long long)(tail.step + 1) * stride;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) run_tail(tail, norm2[0]);
  const double n2 = norm2[0];
  const double scale = n2 > 0.0 ? 1.0 / sqrt(n2) : 0.0;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < g.interior;
       t += (long long)gridDim.x * blockDim.x) {
    int i, j, k;
    compact_coordinates(g, t, i, j, k);
    const long long at = g.node(i, j, k);
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const S value = S(double(source[c * g.interior + t]) * scale);
      target[c * g.interior + t] = value;
      input[c * g.nodes + at] = double(value);
    }
  }
}

// gmres_back_substitute_kernel, gmres_device.hpp:267-277 (one thread).
__global__ void back_substitute_kernel(const double* hessenberg, const double* rhs, double* coefficients,
                                       int leading, const ArnoldiControl* ctl) {
  const int columns = ctl->completed;
  for (int row = columns - 1; row >= 0; --row) {
    double sum = 0;
    for (int column = row + 1; column < columns; ++column)
      sum += hessenberg[(long long)column * leading + row] * coefficients[column];
    const double diagonal = hessenberg[(long long)row * leading + row];
    coefficients[row] = diagonal != 0.0 ? (rhs[row] - sum) / diagonal : 0.0;
  }
}

// x += sum of coefficient * basis column (gmres_update_solution_kernel, :281-292).
template <class S>
__global__ void __launch_bounds__(kThreads) update_solution_kernel(const S* __restrict__ basis,
                                                                   const double* __restrict__ coefficients,
                                                                   double* __restrict__ x, long long count,
                                                                   long long ld,
                                                                   const ArnoldiControl* __restrict__ ctl) {
  const int columns = ctl->completed;
  for (long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x; n < count;
       n += (long long)gridDim.x * blockDim.x) {
    double value = x[n];
    for (int c = 0; c < columns; ++c) value += coefficients[c] * double(basis[(long long)c * ld + n]);
    x[n] = value;
  }
}

// Sums of the dot partials of the step's columns (rows [0, ctl->col]).
__global__ void __launch_bounds__(256) reduce_columns_kernel(const double* __restrict__ partials, double* out,
                                                             int row_stride, const ArnoldiControl* __restrict__ ctl) {
  wait_for_predecessor();
  __shared__ double scratch[8];
  const int row = blockIdx.x;
  if (row > ctl->col) return;
  double sum = 0;
  for (int i = threadIdx.x; i < row_stride; i += blockDim.x) sum += partials[(long long)row * row_stride + i];
  sum = block_sum<256>(sum, scratch);
  if (threadIdx.x == 0) out[row] = sum;
}

// role 0: zero the counter and clear the condition; role 1 (the IF body):
// count a run.
__global__ void condition_probe_kernel(cudaGraphConditionalHandle handle, unsigned* counter, int role) {
  if (role == 0) {
    *counter = 0;
    cudaGraphSetConditional(handle, 0u);
  } else {
    *counter += 1;
  }
}

__global__ void arnoldi_begin_kernel(ArnoldiControl* ctl, int columns, double tolerance) {
  ctl->col = 0;
  ctl->completed = 0;
  ctl->columns = columns;
  ctl->stop = 0;
  ctl->breakdown = 0;
  ctl->tolerance = tolerance;
}

// After step ctl->col: TPIC's stopping rule on the least-squares residual
// estimate status[0] and the breakdown flag status[1]
// (gmres_device.hpp:420-436); in the graph, the WHILE condition stays set
// while the cycle runs and is cleared at the latest after ctl->columns steps.
__global__ void arnoldi_end_kernel(ArnoldiControl* ctl, const double* status, cudaGraphConditionalHandle handle,
                                   int conditional) {
  wait_for_predecessor();
  const int col = ctl->col;
  const double estimate = status[0], breakdown = status[1];
  const bool finite = isfinite(estimate) && isfinite(breakdown);
  ctl->completed = col + 1;
  ctl->breakdown = breakdown != 0.0;
  const bool stop = !finite || estimate <= ctl->tolerance || breakdown != 0.0 || col + 1 >= ctl->columns;
  ctl->stop = !finite ? 2 : (stop ? 1 : 0);
  ctl->col = col + 1;
  if (conditional) cudaGraphSetConditional(handle, stop ? 0u : 1u);
}

}  // namespace

struct SolverWorkspace {
  int precision;
  bool transpose = false;       // applies use A^T (every mass block transposed): the adjoint solve
  uint32_t* invalid = nullptr;  // the context's invalid counter (smoothing passes, TMA apply waits)
  uint32_t wait_polls = 0;      // TMA apply wait bound (0: kDefaultWaitPolls)
  int stall_stencil = -1;       // a test of that bound: the stencil whose wait targets no copy
  Geom g;
  int restart;
  double dt, theta, c, delta, kfac;
  long long count;  // 3 * interior
  long long ld;     // basis column stride: count rounded up to kColumnAlign
  unsigned rblocks;
  void* basis = nullptr;   // (restart+1) columns of count Scalar, ld apart
  void* image = nullptr;   // count Scalar
  double* x = nullptr;
  double* b = nullptr;
  double* r = nullptr;
  double* ximage = nullptr;
  double* input = nullptr;  // node field (3 * nodes)
  double* rhs = nullptr;    // node field
  double* values = nullptr;
  double* partials = nullptr;
  double* state = nullptr;
  double* pinned = nullptr;
  ArnoldiControl* ctl = nullptr;
  // Energy-conserving smoothing: its plan and three node fields of scratch
  // (allocated only when it is on).
  SmoothingPlan smoothing;
  double* smooth_a = nullptr;
  double* smooth_b = nullptr;
  double* smooth_image = nullptr;
  int batch;
  size_t scalar_bytes;
  // The Arnoldi-step loop as a graph (built for one mass pointer).
  cudaStream_t capture = nullptr;
  // Index 0: the operator A; index 1: A^T (the adjoint solve).
  cudaGraph_t loop_graph[2] = {nullptr, nullptr};
  cudaGraphExec_t loop_exec[2] = {nullptr, nullptr};
  const void* loop_mass[2] = {nullptr, nullptr};
  unsigned loop_launches[2] = {0, 0};  // kernels of one step
  bool loop_unavailable = false;
  bool conditional_checked = false;
  // Tensor maps of mass buffers for the TMA-staged apply, per mass pointer
  // and tile shape (0: 32x4x2, 1: thin 32x8x1); built on first use.
  struct MassMap {
    CUtensorMap map;
    const void* mass = nullptr;
    int tile = -1;
    bool usable = false;
  };
  MassMap maps[4];
  int next_map = 0;

  double* hessenberg() { return state; }
  double* cosine() { return state + (size_t)restart * (restart + 1); }
  double* sine() { return cosine() + restart; }
  double* ls_rhs() { return sine() + restart; }
  double* coefficients() { return ls_rhs() + restart + 1; }
  double* status() { return coefficients() + restart; }
  template <class S> S* basis_col(int c) { return (S*)basis + (size_t)c * ld; }
};

SolverWorkspace* solver_create(int precision, const Geom& g, int restart, double dt, double theta,
                               double c, const SmoothingPlan& smoothing, cudaError_t* err) {
  if (3 * g.interior >= (1LL << 31)) {  // the compact-index kernels use 32-bit arithmetic
    *err = cudaErrorInvalidValue;
    return nullptr;
  }
  auto* w = new SolverWorkspace();
  w->precision = precision;
  w->g = g;
  w->restart = restart;
  w->dt = dt;
  w->theta = theta;
  w->c = c;
  w->delta = c * theta * dt;
  w->kfac = 4 * 3.14159265358979323846 * (theta * dt);
  w->count = 3 * g.interior;
  w->ld = (w->count + kColumnAlign - 1) / kColumnAlign * kColumnAlign;
  int device = 0, sms = 148;
  cudaGetDevice(&device);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  w->rblocks = unsigned(std::min<long long>((w->count + kThreads - 1) / kThreads, 4LL * sms));
  w->batch = std::max(restart, 2);
  // TPICB200_STEP_GRAPH=0 keeps the host-stepped Arnoldi loop (one launch per
  // kernel, which a kernel profiler lists one by one).
  if (const char* v = std::getenv("TPICB200_STEP_GRAPH")) w->loop_unavailable = std::strcmp(v, "0") == 0;
  w->scalar_bytes = precision == TPICB200_PRECISION_DOUBLE ? 8 : 4;
  cudaError_t e = cudaSuccess;
  auto alloc = [&](void** p, size_t bytes) {
    if (e == cudaSuccess) e = cudaMalloc(p, bytes);
  };
  w->smoothing = smoothing;
  if (smoothing.iterations > 0) {
    alloc((void**)&w->smooth_a, 3 * g.nodes * sizeof(double));
    alloc((void**)&w->smooth_b, 3 * g.nodes * sizeof(double));
    alloc((void**)&w->smooth_image, 3 * g.nodes * sizeof(double));
  }
  alloc(&w->basis, (size_t)(restart + 1) * w->ld * w->scalar_bytes);
  alloc(&w->image, (size_t)w->count * w->scalar_bytes);
  alloc((void**)&w->x, w->count * sizeof(double));
  alloc((void**)&w->b, w->count * sizeof(double));
  alloc((void**)&w->r, w->count * sizeof(double));
  alloc((void**)&w->ximage, w->count * sizeof(double));
  alloc((void**)&w->input, 3 * g.nodes * sizeof(double));
  alloc((void**)&w->rhs, 3 * g.nodes * sizeof(double));
  alloc((void**)&w->values, w->batch * sizeof(double));
  alloc((void**)&w->partials, (size_t)w->batch * w->rblocks * sizeof(double));
  alloc((void**)&w->state, ((size_t)restart * (restart + 1) + 4 * restart + 3) * sizeof(double));
  alloc((void**)&w->ctl, sizeof(ArnoldiControl));
  if (e == cudaSuccess) e = cudaMallocHost((void**)&w->pinned, 2 * sizeof(double) + sizeof(ArnoldiControl));
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&w->capture, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaMemset(w->input, 0, 3 * g.nodes * sizeof(double));
  if (e == cudaSuccess) e = cudaMemset(w->rhs, 0, 3 * g.nodes * sizeof(double));
  *err = e;
  if (e != cudaSuccess) {
    solver_destroy(w);
    return nullptr;
  }
  return w;
}

void solver_destroy(SolverWorkspace* w) {
  if (!w) return;
  cudaFree(w->basis); cudaFree(w->image); cudaFree(w->x); cudaFree(w->b); cudaFree(w->r);
  cudaFree(w->ximage); cudaFree(w->input); cudaFree(w->rhs); cudaFree(w->values);
  cudaFree(w->partials); cudaFree(w->state); cudaFree(w->ctl);
  cudaFree(w->smooth_a); cudaFree(w->smooth_b); cudaFree(w->smooth_image);
  for (int t = 0; t < 2; ++t) {
    if (w->loop_exec[t]) cudaGraphExecDestroy(w->loop_exec[t]);
    if (w->loop_graph[t]) cudaGraphDestroy(w->loop_graph[t]);
  }
  if (w->capture) cudaStreamDestroy(w->capture);
  if (w->pinned) cudaFreeHost(w->pinned);
  delete w;
}

namespace {

using TensorMapEncodeTiled = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                          const cuuint64_t*, const cuuint32_t*, const cuuint32_t*,
                                          CUtensorMapInterleave, CUtensorMapSwizzle, CUtensorMapL2promotion,
                                          CUtensorMapFloatOOBfill);

TensorMapEncodeTiled tensor_map_encoder() {
  static std::atomic<TensorMapEncodeTiled> fn{nullptr};
  TensorMapEncodeTiled f = fn.load();
  if (f) return f;
  void* p = nullptr;
  cudaDriverEntryPointQueryResult found;
  if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &found) != cudaSuccess ||
      found != cudaDriverEntryPointSuccess || !p) {
    cudaGetLastError();
    return nullptr;
  }
  f = reinterpret_cast<TensorMapEncodeTiled>(p);
  fn.store(f);
  return f;
}

// The tensor map of a mass buffer as a 4-D tensor (x pitch MX, y NY, z NZ,
// 126 entries) with the apply's box {36, TY+1, TZ+1, 9}, or nullptr when the
// buffer does not meet the copies' alignment rules (vertex stride 1, the
// base, the row pitch and the entry-plane stride multiples of 16 bytes):
// those buffers take maxwell_apply_kernel.
template <class M>
const CUtensorMap* mass_tensor_map(SolverWorkspace* w, const M* mass, bool thin) {
  const Geom& g = w->g;
  const bool flat = thin;  // thin tiles are on grids one cell thick along z
  const int tile = thin ? 1 : 0;
  for (auto& m : w->maps)
    if (m.mass == mass && m.tile == tile) return m.usable ? &m.map : nullptr;
  auto& m = w->maps[w->next_map];
  w->next_map = (w->next_map + 1) % 4;
  m.mass = mass;
  m.tile = tile;
  m.usable = false;
  const size_t es = sizeof(M);
  if (g.mvs != 1 || (reinterpret_cast<uintptr_t>(mass) % 16) != 0 || ((size_t)g.MX * es) % 16 != 0 ||
      ((size_t)g.mes * es) % 16 != 0 || (size_t)g.mes < (size_t)g.mnodes)
    return nullptr;
  TensorMapEncodeTiled encode = tensor_map_encoder();
  if (!encode) return nullptr;
  const cuuint64_t dims[4] = {cuuint64_t(g.MX), cuuint64_t(g.NY), cuuint64_t(g.NZ), 126};
  const cuuint64_t strides[3] = {cuuint64_t(g.MX) * es, cuuint64_t(g.MX) * g.NY * es, cuuint64_t(g.mes) * es};
  const cuuint32_t box[4] = {cuuint32_t(kBoxX), cuuint32_t((thin ? kThinTY : kTY) + 1),
                             cuuint32_t(flat ? 1 : kTZ + 1), 9};
  const cuuint32_t unit[4] = {1, 1, 1, 1};
  const CUresult r = encode(&m.map, es == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4,
                            const_cast<M*>(mass), dims, strides, box, unit, CU_TENSOR_MAP_INTERLEAVE_NONE,
                            CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  m.usable = r == CUDA_SUCCESS;
  return m.usable ? &m.map : nullptr;
}

// Launches the TMA-staged apply; the kernel's dynamic shared memory limit is
// raised once per device.
template <class C, class M, class Out, int TY, int TZ, bool kTranspose, bool kFlat = false>
cudaError_t launch_apply_tma(const CUtensorMap& map, unsigned tiles, cudaStream_t st, const Geom& g, C d2, C kf,
                             C civ, const double* in, Out* out, uint32_t* invalid, uint32_t polls, int stall) {
  // Two stages: four CTAs per SM in the float apply (three in the mixed
  // residual apply); three stages gave three (two) and a slower solve.
  constexpr int S = 2;
  constexpr int bytes = TmaApplyShared<C, M, kTX, TY, TZ, S, kFlat>::total;
  static_assert(bytes <= 227 * 1024, "apply tile exceeds shared memory");
  auto kernel = maxwell_apply_tma_kernel<C, M, Out, kTX, TY, TZ, S, kTranspose, kFlat>;
  static std::atomic<uint64_t> ready{0};
  int device = 0;
  cudaError_t e = cudaGetDevice(&device);
  if (e != cudaSuccess) return e;
  const uint64_t bit = device < 64 ? 1ull << device : 0;
  if (!bit || !(ready.load() & bit)) {
    e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (e != cudaSuccess) return e;
    ready.fetch_or(bit);
  }
  return launch_programmatic(kernel, tiles, kTX * TY * TZ, bytes, st, map, g, d2, kf, civ, in, out, invalid,
                             polls ? polls : kDefaultWaitPolls, stall);
}

template <class P>
struct Solve {
  using S = typename P::EC;     // Krylov basis and Arnoldi arithmetic
  using Mass = typename P::Mass;
  using Fld = typename P::Fld;
  static constexpr bool refined = sizeof(S) < sizeof(double);

  SolverWorkspace* w;
  cudaStream_t s;
  cudaError_t err = cudaSuccess;
  int waits = 0;

  unsigned blocks() const { return grid_for(w->g.interior, kThreads); }
  void check() { if (err == cudaSuccess) err = cudaGetLastError(); }

  // The step's kernels are launched with programmatic stream serialization:
  // each may be scheduled while its predecessor drains and waits for it
  // (wait_for_predecessor) before reading its results.
  template <class C, class Out> void apply(const Mass* mass, Out* out, cudaStream_t st) {
    const Geom& g = w->g;
    launch_node_ghosts(g, w->input, 3, st, true);
    const double iv = g.inv_volume;
    // Smoothed schedule (complete_apply_smoothed, maxwell_device.hpp:389-418):
    // S^n(v), its mass response, S^n of that, then the fused kernel combines
    // with the curl-curl term.
    const double* response = nullptr;
    if (w->smoothing.iterations > 0) {
      const SmoothingPlan& sp = w->smoothing;
      const bool dbl = sizeof(C) == 8;
      if (err == cudaSuccess)
        err = launch_smooth(dbl, g, sp.iterations, sp.op, sp.alpha, w->input, w->smooth_a, w->smooth_b, w->invalid, st);
      mass_image_kernel<C, Mass><<<grid_for(g.interior, kThreads), kThreads, 0, st>>>(g, C(iv), mass, w->smooth_a,
                                                                                     w->smooth_image);
      count_launches(1);
      launch_node_ghosts(g, w->smooth_image, 3, st);
      if (err == cudaSuccess)
        err = launch_smooth(dbl, g, sp.iterations, sp.op, sp.alpha, w->smooth_image, w->smooth_a, w->smooth_b, w->invalid, st);
      response = w->smooth_a;
    }
    // The thin tile (flat boxes in the TMA apply) on every grid one cell thick
    // along z. Limited to grids of at least two thin tiles per SM, the smaller
    // ones took the 32 x 4 x 2 tile with three z planes per box: 2.337 against
    // 2.334 ms per cycle on a 256 x 128 x 1 deck, 5.37 against 5.32 ms on a
    // 1024 x 1 x 1 deck.
    const long long thin_tiles = (long long)((g.nx + kTX - 1) / kTX) * ((g.ny + kThinTY - 1) / kThinTY);
    const bool thin = g.nz == 1;
    const unsigned tiles = thin ? unsigned(thin_tiles)
                                : unsigned(((g.nx + kTX - 1) / kTX) * ((g.ny + kTY - 1) / kTY) *
                                           ((g.nz + kTZ - 1) / kTZ));
    const C d2 = C(w->delta * w->delta), kf = C(w->kfac), civ = C(iv);
    const double* in = w->input;
    const CUtensorMap* map = response ? nullptr : mass_tensor_map(w, mass, thin);
    if (map) {
      const uint32_t polls = w->wait_polls;
      const int stall = w->stall_stencil;
      cudaError_t e;
      // Thin tiles are on grids one cell thick along z: flat boxes.
      if (w->transpose && thin)
        e = launch_apply_tma<C, Mass, Out, kThinTY, 1, true, true>(*map, tiles, st, g, d2, kf, civ, in, out,
                                                                   w->invalid, polls, stall);
      else if (w->transpose)
        e = launch_apply_tma<C, Mass, Out, kTY, kTZ, true>(*map, tiles, st, g, d2, kf, civ, in, out, w->invalid,
                                                           polls, stall);
      else if (thin)
        e = launch_apply_tma<C, Mass, Out, kThinTY, 1, false, true>(*map, tiles, st, g, d2, kf, civ, in, out,
                                                                    w->invalid, polls, stall);
      else
        e = launch_apply_tma<C, Mass, Out, kTY, kTZ, false>(*map, tiles, st, g, d2, kf, civ, in, out, w->invalid,
                                                            polls, stall);
      if (err == cudaSuccess) err = e;
    } else if (w->transpose) {
      // The adjoint solve (no smoothing): every mass block transposed.
      if (thin)
        launch_programmatic(maxwell_apply_kernel<C, Mass, Out, kTX, kThinTY, 1, false, true>, tiles, kTX * kThinTY, 0,
                            st, g, d2, kf, civ, mass, in, out, response);
      else
        launch_programmatic(maxwell_apply_kernel<C, Mass, Out, kTX, kTY, kTZ, false, true>, tiles, kTX * kTY * kTZ, 0,
                            st, g, d2, kf, civ, mass, in, out, response);
    } else if (thin && response)
      launch_programmatic(maxwell_apply_kernel<C, Mass, Out, kTX, kThinTY, 1, true>, tiles, kTX * kThinTY, 0, st, g,
                          d2, kf, civ, mass, in, out, response);
    else if (thin)
      launch_programmatic(maxwell_apply_kernel<C, Mass, Out, kTX, kThinTY, 1>, tiles, kTX * kThinTY, 0, st, g, d2,
                          kf, civ, mass, in, out, response);
    else if (response)
      launch_programmatic(maxwell_apply_kernel<C, Mass, Out, kTX, kTY, kTZ, true>, tiles, kTX * kTY * kTZ, 0, st, g,
                          d2, kf, civ, mass, in, out, response);
    else
      launch_programmatic(maxwell_apply_kernel<C, Mass, Out, kTX, kTY, kTZ>, tiles, kTX * kTY * kTZ, 0, st, g, d2,
                          kf, civ, mass, in, out, response);
    const long long dup = (long long)g.inx * g.iny + (long long)g.inx * g.nz + (long long)g.ny * g.nz;
    launch_programmatic(duplicate_rows_kernel<Out>, grid_for(3 * dup, kThreads), kThreads, 0, st, g, out);
    count_launches(2);
    check();
  }
  void reduce(int filled) {
    launch_reduce_rows(w->partials, w->values, w->batch, w->rblocks, w->rblocks, filled, s);
  }
  // Waits for the stream and copies two doubles at `src` (and, with
  // `control`, the Arnoldi control record) to the host.
  bool read_back(const double* src, double out[2], ArnoldiControl* control = nullptr) {
    if (err != cudaSuccess) return false;
    if (src) err = cudaMemcpyAsync(w->pinned, src, 2 * sizeof(double), cudaMemcpyDeviceToHost, s);
    if (control && err == cudaSuccess)
      err = cudaMemcpyAsync(w->pinned + 2, w->ctl, sizeof(ArnoldiControl), cudaMemcpyDeviceToHost, s);
    if (err == cudaSuccess) err = cudaStreamSynchronize(s);
    ++waits;
    if (src) {
      out[0] = w->pinned[0];
      out[1] = w->pinned[1];
    }
    if (control) std::memcpy(control, w->pinned + 2, sizeof(ArnoldiControl));
    return err == cudaSuccess;
  }
  void apply_solution(const Mass* mass) {
    unpack_kernel<double><<<blocks(), kThreads, 0, s>>>(w->g, w->x, w->input);
    count_launches(1);
    apply<double, double>(mass, w->ximage, s);
  }

  // One Arnoldi step (the step index and the stopping decision live in
  // w->ctl): A v_col, classical Gram-Schmidt against columns 0..col, the
  // normalized v_{col+1} with the Givens update of the least-squares
  // problem, and the stopping rule.
  void step(const Mass* mass, cudaStream_t st, cudaGraphConditionalHandle handle, int conditional) {
    const Geom& g = w->g;
    const long long N = w->count;
    const int m = w->restart;
    S* image = (S*)w->image;
    S* basis = w->template basis_col<S>(0);
    apply<S, S>(mass, image, st);
    const dim3 grid(w->rblocks, (m + kDotTile - 1) / kDotTile);
    launch_programmatic(dot_batch_kernel<S>, grid, kThreads, 0, st, (const S*)basis, (const S*)image, w->partials, N,
                        w->ld, (const ArnoldiControl*)w->ctl);
    launch_programmatic(reduce_columns_kernel, unsigned(m), 256, 0, st, (const double*)w->partials, w->values,
                        int(w->rblocks), (const ArnoldiControl*)w->ctl);
    launch_programmatic(orthogonalize_kernel<S>, w->rblocks, kThreads, 0, st, (const S*)basis,
                        (const double*)w->values, image, w->hessenberg(), m + 1, w->partials, N, w->ld,
                        (const ArnoldiControl*)w->ctl);
    launch_reduce_rows(w->partials, w->values, w->batch, w->rblocks, w->rblocks, 1, st, true);
    launch_programmatic(normalize_kernel<S, S>, w->rblocks, kThreads, 0, st, g, (const S*)image,
                        (const double*)w->values, basis, w->ld, w->input,
                        ArnoldiTail{w->hessenberg(), w->cosine(), w->sine(), w->ls_rhs(), w->status(), 0, m + 1},
                        (const ArnoldiControl*)w->ctl);
    launch_programmatic(arnoldi_end_kernel, 1u, 1u, 0, st, w->ctl, (const double*)w->status(), handle, conditional);
    count_launches(5);
    check();
  }

  // The restart cycle's steps as one graph: a WHILE node whose body is one
  // step(); arnoldi_end_kernel clears the condition when the cycle stops,
  // at the latest after ctl->columns <= restart steps. Before the first such
  // graph, conditional_self_test() checks on this device that a kernel's
  // cudaGraphSetConditional takes effect. Built once per mass pointer; false
  // when conditional graphs are not available, and the host loop steps.
  bool loop_ready(const Mass* mass) {
    if (w->loop_unavailable || err != cudaSuccess) return false;
    const int t = w->transpose ? 1 : 0;
    if (w->loop_exec[t] && w->loop_mass[t] == (const void*)mass) return true;
    if (w->loop_exec[t]) cudaGraphExecDestroy(w->loop_exec[t]);
    if (w->loop_graph[t]) cudaGraphDestroy(w->loop_graph[t]);
    w->loop_exec[t] = nullptr;
    w->loop_graph[t] = nullptr;
    const char* stage = "self-test";
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    bool ok = conditional_self_test();
    if (ok) {
      stage = "graph";
      ok = cudaGraphCreate(&graph, 0) == cudaSuccess;
    }
    cudaGraphConditionalHandle handle{};
    if (ok) {
      stage = "handle";
      ok = cudaGraphConditionalHandleCreate(&handle, graph, 1u, cudaGraphCondAssignDefault) == cudaSuccess;
    }
    cudaGraphNodeParams params{};
    params.type = cudaGraphNodeTypeConditional;
    params.conditional.handle = handle;
    params.conditional.type = cudaGraphCondTypeWhile;
    params.conditional.size = 1;
    cudaGraphNode_t node;
    if (ok) {
      stage = "conditional node";
      ok = cudaGraphAddNode(&node, graph, nullptr, 0, &params) == cudaSuccess;
    }
    if (ok) {
      stage = "capture";
      const unsigned long long before = launches_so_far();
      cudaGraph_t body = params.conditional.phGraph_out[0];
      ok = cudaStreamBeginCaptureToGraph(w->capture, body, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed) ==
           cudaSuccess;
      if (ok) {
        const cudaError_t saved = err;
        step(mass, w->capture, handle, 1);
        cudaGraph_t captured = nullptr;
        ok = cudaStreamEndCapture(w->capture, &captured) == cudaSuccess && err == cudaSuccess;
        err = saved;
      }
      const unsigned long long captured_launches = launches_so_far() - before;
      uncount_launches(captured_launches);
      w->loop_launches[t] = unsigned(captured_launches);
    }
    if (ok) {
      stage = "instantiate";
      ok = cudaGraphInstantiate(&exec, graph, 0) == cudaSuccess;
    }
    if (!ok) {
      const cudaError_t why = cudaGetLastError();
      if (exec) cudaGraphExecDestroy(exec);
      if (graph) cudaGraphDestroy(graph);
      std::fprintf(stderr,
                   "tpicb200: the GMRES step graph is unavailable (%s: %s); the host steps the Arnoldi loop\n", stage,
                   cudaGetErrorString(why));
      w->loop_unavailable = true;
      return false;
    }
    w->loop_graph[t] = graph;
    w->loop_exec[t] = exec;
    w->loop_mass[t] = mass;
    return true;
  }

  // A graph of one kernel that clears a conditional handle (default 1)
  // followed by an IF node on it whose body counts its runs: true when the
  // body did not run, i.e. the device-side condition took effect.
  bool conditional_self_test() {
    if (w->conditional_checked) return true;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    cudaGraphConditionalHandle handle{};
    bool ok = cudaGraphCreate(&graph, 0) == cudaSuccess &&
              cudaGraphConditionalHandleCreate(&handle, graph, 1u, cudaGraphCondAssignDefault) == cudaSuccess;
    unsigned* counter = reinterpret_cast<unsigned*>(w->ctl);  // free between solves
    cudaGraphNode_t clear_node = nullptr, if_node = nullptr;
    if (ok) {
      ok = cudaStreamBeginCaptureToGraph(w->capture, graph, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed) ==
           cudaSuccess;
      if (ok) {
        condition_probe_kernel<<<1, 1, 0, w->capture>>>(handle, counter, 0);
        cudaGraph_t captured = nullptr;
        ok = cudaStreamEndCapture(w->capture, &captured) == cudaSuccess;
      }
    }
    size_t count = 1;
    ok = ok && cudaGraphGetNodes(graph, &clear_node, &count) == cudaSuccess && count == 1;
    cudaGraphNodeParams params{};
    params.type = cudaGraphNodeTypeConditional;
    params.conditional.handle = handle;
    params.conditional.type = cudaGraphCondTypeIf;
    params.conditional.size = 1;
    ok = ok && cudaGraphAddNode(&if_node, graph, &clear_node, 1, &params) == cudaSuccess;
    if (ok) {
      ok = cudaStreamBeginCaptureToGraph(w->capture, params.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                         cudaStreamCaptureModeRelaxed) == cudaSuccess;
      if (ok) {
        condition_probe_kernel<<<1, 1, 0, w->capture>>>(handle, counter, 1);
        cudaGraph_t captured = nullptr;
        ok = cudaStreamEndCapture(w->capture, &captured) == cudaSuccess;
      }
    }
    ok = ok && cudaGraphInstantiate(&exec, graph, 0) == cudaSuccess;
    ok = ok && cudaGraphLaunch(exec, s) == cudaSuccess;
    unsigned ran = 1;
    ok = ok && cudaMemcpyAsync(&ran, counter, sizeof(unsigned), cudaMemcpyDeviceToHost, s) == cudaSuccess &&
         cudaStreamSynchronize(s) == cudaSuccess;
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    w->conditional_checked = ok && ran == 0;
    return w->conditional_checked;
  }

  // With rhs_in (a double node field, the adjoint solve): that right-hand
  // side and a zero initial guess; otherwise the Maxwell RHS from e, bcell
  // and j with the guess E^n.
  int run(const void* e, const void* bcell, const void* j, const void* mass_v, double* etheta,
          tpicb200_gmres_result* result, int max_iterations, double tolerance, const double* rhs_in = nullptr) {
    const Geom& g = w->g;
    const Mass* mass = (const Mass*)mass_v;
    const long long N = w->count;
    const int m = w->restart;
    tpicb200_gmres_result res{};
    const bool graph = loop_ready(mass);
    if (rhs_in) {
      if (err == cudaSuccess) err = cudaMemsetAsync(w->x, 0, size_t(N) * sizeof(double), s);
      pack_kernel<double><<<blocks(), kThreads, 0, s>>>(g, rhs_in, w->b);
      count_launches(1);
      check();
    } else {
    // Initial guess E^n (the copy of E into theta, maxwell_device.hpp:134-147) and the RHS.
    pack_storage_kernel<Fld><<<blocks(), kThreads, 0, s>>>(g, (const Fld*)e, w->x);
    if (w->smoothing.iterations > 0) {
      // RHS with S^n(J-hat) (complete_rhs, maxwell_device.hpp:152-172): the
      // current widened to double with its ghosts refilled, then smoothed in
      // the field arithmetic.
      const SmoothingPlan& sp = w->smoothing;
      if (err == cudaSuccess) err = launch_widen(P::id, g, j, w->smooth_image, s);
      launch_node_ghosts(g, w->smooth_image, 3, s);
      if (err == cudaSuccess)
        err = launch_smooth(P::id == TPICB200_PRECISION_DOUBLE, g, sp.iterations, sp.op, sp.alpha, w->smooth_image,
                            w->smooth_a, w->smooth_b, w->invalid, s);
      launch_rhs(P::id, g, w->delta, w->kfac, e, bcell, w->smooth_a, w->rhs, s, true);
    } else {
      launch_rhs(P::id, g, w->delta, w->kfac, e, bcell, j, w->rhs, s);
    }
    pack_kernel<double><<<blocks(), kThreads, 0, s>>>(g, w->rhs, w->b);
    count_launches(2);
    check();
    }
    apply_solution(mass);
    residual_kernel<true><<<w->rblocks, kThreads, 0, s>>>(w->b, w->ximage, w->r, w->partials, N);
    count_launches(1);
    reduce(2);
    double controls[2];
    if (!read_back(w->values, controls)) return TPICB200_BACKEND_FAILURE;
    if (!std::isfinite(controls[0]) || !std::isfinite(controls[1])) return TPICB200_OVERFLOW;
    res.residual = res.initial_residual = std::sqrt(controls[0]);
    res.rhs_norm = std::sqrt(controls[1]);
    const double scale = res.rhs_norm == 0.0 ? 1.0 : res.rhs_norm;
    const double atol = scale * tolerance;
    auto converged = [&] {
      res.relative_residual = res.residual / scale;
      res.converged = res.residual <= atol;
    };
    converged();
    while (!res.converged && res.iterations < max_iterations) {
      cudaMemsetAsync(w->state, 0, ((size_t)m * (m + 1) + 4 * m + 3) * sizeof(double), s);
      // values[0] holds |r|^2 of the residual just formed.
      normalize_kernel<double, S><<<w->rblocks, kThreads, 0, s>>>(
          g, w->r, w->values, w->template basis_col<S>(0), w->ld, w->input,
          ArnoldiTail{nullptr, nullptr, nullptr, w->ls_rhs(), nullptr, -1, 0}, nullptr);
      const int columns = std::min(m, max_iterations - res.iterations);
      const double cycle_tolerance =
          refined ? std::max(atol, res.residual * 16.0 * double(std::numeric_limits<S>::epsilon())) : atol;
      arnoldi_begin_kernel<<<1, 1, 0, s>>>(w->ctl, columns, cycle_tolerance);
      count_launches(2);
      check();
      ArnoldiControl control{};
      if (graph) {
        if (err == cudaSuccess) err = cudaGraphLaunch(w->loop_exec[w->transpose ? 1 : 0], s);
      } else {
        for (int col = 0; col < columns; ++col) {
          step(mass, s, cudaGraphConditionalHandle{}, 0);
          if (!read_back(nullptr, nullptr, &control)) return TPICB200_BACKEND_FAILURE;
          if (control.stop) break;
        }
      }
      back_substitute_kernel<<<1, 1, 0, s>>>(w->hessenberg(), w->ls_rhs(), w->coefficients(), m + 1, w->ctl);
      update_solution_kernel<S><<<grid_for(N, kThreads), kThreads, 0, s>>>(w->template basis_col<S>(0),
                                                                          w->coefficients(), w->x, N, w->ld,
                                                                          w->ctl);
      count_launches(2);
      check();
      apply_solution(mass);
      residual_kernel<false><<<w->rblocks, kThreads, 0, s>>>(w->b, w->ximage, w->r, w->partials, N);
      count_launches(1);
      reduce(1);
      if (!read_back(w->values, controls, &control)) return TPICB200_BACKEND_FAILURE;
      if (graph) count_launches(w->loop_launches[w->transpose ? 1 : 0] * unsigned(control.completed));
      if (control.stop == 2) return TPICB200_OVERFLOW;
      if (!std::isfinite(controls[0]) || controls[0] < 0) return TPICB200_OVERFLOW;
      res.iterations += control.completed;
      res.residual = std::sqrt(controls[0]);
      converged();
      if (control.breakdown && !res.converged) break;
    }
    res.host_waits = waits;
    if (result) *result = res;
    if (!res.converged) return TPICB200_NOT_CONVERGED;
    unpack_kernel<double><<<blocks(), kThreads, 0, s>>>(g, w->x, etheta);
    count_launches(1);
    launch_node_ghosts(g, etheta, 3, s);
    check();
    return err == cudaSuccess ? TPICB200_SUCCESS : TPICB200_BACKEND_FAILURE;
  }
};

}  // namespace

int solver_solve(SolverWorkspace* w, const void* e, const void* bcell, const void* j, const void* mass,
                 double* etheta, tpicb200_gmres_result* result, int max_iterations, double tol,
                 cudaStream_t s, cudaError_t* err) {
  int status;
  if (w->precision == TPICB200_PRECISION_DOUBLE) {
    Solve<PDouble> solve{w, s};
    status = solve.run(e, bcell, j, mass, etheta, result, max_iterations, tol);
    *err = solve.err;
  } else {
    Solve<PMixed> solve{w, s};
    status = solve.run(e, bcell, j, mass, etheta, result, max_iterations, tol);
    *err = solve.err;
  }
  return status;
}

void solver_set_invalid(SolverWorkspace* w, uint32_t* invalid) { w->invalid = invalid; }

void solver_set_waits(SolverWorkspace* w, uint32_t polls, int stall_stencil) {
  if (polls == w->wait_polls && stall_stencil == w->stall_stencil) return;
  w->wait_polls = polls;
  w->stall_stencil = stall_stencil;
  // The step graphs hold the apply's arguments: capture them again.
  for (int t = 0; t < 2; ++t) w->loop_mass[t] = nullptr;
}

int solver_solve_adjoint(SolverWorkspace* w, const double* rhs, const void* mass, double* lambda,
                         tpicb200_gmres_result* result, int max_iterations, double tol, cudaStream_t s,
                         cudaError_t* err) {
  if (w->smoothing.iterations > 0) {
    *err = cudaSuccess;
    return TPICB200_INVALID_STATE;
  }
  w->transpose = true;
  int status;
  if (w->precision == TPICB200_PRECISION_DOUBLE) {
    Solve<PDouble> solve{w, s};
    status = solve.run(nullptr, nullptr, nullptr, mass, lambda, result, max_iterations, tol, rhs);
    *err = solve.err;
  } else {
    Solve<PMixed> solve{w, s};
    status = solve.run(nullptr, nullptr, nullptr, mass, lambda, result, max_iterations, tol, rhs);
    *err = solve.err;
  }
  w->transpose = false;
  return status;
}

cudaError_t solver_smooth(SolverWorkspace* w, const double* in, double* out, cudaStream_t s) {
  const SmoothingPlan& sp = w->smoothing;
  if (sp.iterations <= 0) return cudaErrorInvalidValue;
  return launch_smooth(w->precision == TPICB200_PRECISION_DOUBLE, w->g, sp.iterations, sp.op, sp.alpha, in, out,
                       w->smooth_b, w->invalid, s);
}

cudaError_t solver_mass_apply(SolverWorkspace* w, const void* mass, const double* in, double* out,
                              cudaStream_t s) {
  const unsigned blocks = grid_for(w->g.interior, kThreads);
  if (w->precision == TPICB200_PRECISION_DOUBLE)
    mass_apply_kernel<double><<<blocks, kThreads, 0, s>>>(w->g, w->g.inv_volume, (const double*)mass, in, out);
  else
    mass_apply_kernel<float><<<blocks, kThreads, 0, s>>>(w->g, w->g.inv_volume, (const float*)mass, in, out);
  count_launches(1);
  return cudaGetLastError();
}

}  // namespace tpicb200
