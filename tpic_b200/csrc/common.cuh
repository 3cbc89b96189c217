// Shared device definitions of the ECSIM cycle kernels: grid geometry,
// precision modes, CIC weights, the particle response, warp/block reductions.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>
#include <cstddef>

#include "../../include/tpicb200.h"

namespace tpicb200 {

// Geometry of a fully periodic grid in the layouts of tpicb200.h.
struct Geom {
  int nx, ny, nz;
  int NX, NY, NZ;      // node extents (n + 3)
  int CX, CY, CZ;      // cell extents (n + 2)
  int ex, ey, ez;      // particle key extents (n + 4)
  long long nodes;     // NX*NY*NZ
  long long cells;     // CX*CY*CZ
  long long bins;      // ex*ey*ez
  int inx, iny, inz;   // interior nodes per axis (n + 1)
  long long interior;  // inx*iny*inz
  double dx, dy, dz;
  double inv[3];       // 1/spacing
  double volume;       // (dx*dy)*dz
  double inv_volume;   // 1/volume
  // Mass storage: entry k = 9*stencil + component of vertex v lives at
  // v*mvs + k*mes: (126, 1) for TPIC's records, (1, mnodes) stencil-major.
  // A mass vertex is mass_vertex(i, j, k): the node index, except in the
  // tiled layout, whose x pitch MX pads the n + 3 nodes of a row to a
  // multiple of 4 (16-byte rows for the tensor-memory-access copies).
  long long mvs, mes;
  int MX;             // mass x pitch: NX, or NX rounded up to a multiple of 4 (tiled)
  long long mnodes;   // vertices of one mass entry plane: MX*NY*NZ
  // Cells per run of the run mover and the binned sort (a power of two,
  // 1..kRunCells): a warp walks one run's records, so small grids use
  // shorter runs to keep enough warps in flight.
  int run_len;

  __host__ __device__ __forceinline__ long long mass_index(long long vertex, int k) const {
    return vertex * mvs + (long long)k * mes;
  }
  __host__ __device__ __forceinline__ long long mass_vertex(int i, int j, int k) const {
    return (long long)(i + 1) + (long long)MX * ((j + 1) + (long long)NY * (k + 1));
  }
  // Mass-vertex offset of a stencil (dx, dy, dz).
  __host__ __device__ __forceinline__ long long mass_offset(int dx, int dy, int dz) const {
    return (long long)dx + (long long)MX * (dy + (long long)NY * dz);
  }

  __host__ __device__ __forceinline__ long long node(int i, int j, int k) const {
    return (long long)(i + 1) + (long long)NX * ((j + 1) + (long long)NY * (k + 1));
  }
  __host__ __device__ __forceinline__ long long cell(int i, int j, int k) const {
    return (long long)(i + 1) + (long long)CX * ((j + 1) + (long long)CY * (k + 1));
  }
  __host__ __device__ __forceinline__ int32_t encode(int i, int j, int k) const {
    return (i + 2) + ex * ((j + 2) + ey * (k + 2));
  }
  __host__ __device__ __forceinline__ void decode(int32_t key, int& i, int& j, int& k) const {
    const int yz = key / ex;
    i = key - yz * ex - 2;
    j = yz % ey - 2;
    k = yz / ey - 2;
  }
  __host__ __device__ __forceinline__ bool interior_cell(int i, int j, int k) const {
    return i >= 0 && i < nx && j >= 0 && j < ny && k >= 0 && k < nz;
  }
};

Geom make_geom(const tpicb200_grid& g);

// Precision modes: storage types (Pos, Vel, Fld, Mass) and the arithmetic of
// the mover/current (VC) and of the Arnoldi operator applies (EC).
struct PDouble {
  using Pos = double; using Vel = double; using VC = double; using Fld = double;
  using Mass = double; using EC = double;
  static constexpr int id = TPICB200_PRECISION_DOUBLE;
};
struct PMixed {
  using Pos = double; using Vel = float; using VC = float; using Fld = float;
  using Mass = float; using EC = float;
  static constexpr int id = TPICB200_PRECISION_MIXED;
};

// CIC weights with the reference's (wx*wy)*wz grouping and corner order
// (ecsim/particles/cic.hpp:24-36): corner a has offset (a&1, a>>1&1, a>>2&1).
template <class C>
__device__ __forceinline__ void cic_weights(C x, C y, C z, C w[8]) {
  const C cx = C(1) - x, cy = C(1) - y, cz = C(1) - z;
  w[0] = cx * cy * cz; w[1] = x * cy * cz; w[2] = cx * y * cz; w[3] = x * y * cz;
  w[4] = cx * cy * z;  w[5] = x * cy * z;  w[6] = cx * y * z;  w[7] = x * y * z;
}

// The particle response alpha = (I + w w^T + [w]x) / (1 + w.w), w = beta/c B
// (ecsim/particles/particle_response.hpp:16-42). All nine entries, row-major.
template <class C>
struct Response {
  C a[9];
  C norm_square;
  __device__ __forceinline__ Response(C bx, C by, C bz, C beta_over_c) {
    const C x = beta_over_c * bx, y = beta_over_c * by, z = beta_over_c * bz;
    norm_square = x * x + y * y + z * z;
    const C inverse = C(1) / (C(1) + norm_square);
    a[0] = (C(1) + x * x) * inverse;
    a[4] = (C(1) + y * y) * inverse;
    a[8] = (C(1) + z * z) * inverse;
    const C xy = x * y * inverse, xz = x * z * inverse, yz = y * z * inverse;
    const C sx = x * inverse, sy = y * inverse, sz = z * inverse;
    a[1] = xy + sz; a[2] = xz - sy; a[3] = xy - sz;
    a[5] = yz + sx; a[6] = xz + sy; a[7] = yz - sx;
  }
  __device__ __forceinline__ void apply(C x, C y, C z, C& ox, C& oy, C& oz) const {
    ox = a[0] * x + a[1] * y + a[2] * z;
    oy = a[3] * x + a[4] * y + a[5] * z;
    oz = a[6] * x + a[7] * y + a[8] * z;
  }
};

template <class T> __device__ __forceinline__ bool finite_value(T v) {
  return isfinite(v);
}

// Canonical stencil offsets of the compact mass record
// (data/mass_matrix/mass_matrix_layout.hpp:17-24).
__host__ __device__ constexpr int stencil_offset(int s, int axis) {
  constexpr int offsets[14][3] = {{0, 0, 0}, {1, 0, 0}, {0, 1, 0}, {0, 0, 1}, {1, 1, 0},
                                  {1, -1, 0}, {1, 0, 1}, {1, 0, -1}, {0, 1, 1}, {0, 1, -1},
                                  {1, -1, 1}, {1, 1, -1}, {-1, 1, 1}, {1, 1, 1}};
  return offsets[s][axis];
}

// Stencil of the ordered corner pair (a, b), or -1 when the reverse pair owns
// the block (the table of ecsim/mass_matrix/mass_matrix_stencil.hpp:13-40).
__host__ __device__ constexpr int pair_stencil(int a, int b) {
  const int d0 = (b & 1) - (a & 1), d1 = ((b >> 1) & 1) - ((a >> 1) & 1),
            d2 = ((b >> 2) & 1) - ((a >> 2) & 1);
  for (int s = 0; s < 14; ++s)
    if (stencil_offset(s, 0) == d0 && stencil_offset(s, 1) == d1 && stencil_offset(s, 2) == d2)
      return s;
  return -1;
}

__device__ __forceinline__ int wrap_index(int i, int n) {
  // Periodic unique index in [0, n) (n = 1 maps the ghost n+1 = 2 to 0 too).
  const int r = i % n;
  return r < 0 ? r + n : r;
}

// Step d = to - from along a periodic axis of n cells, folded to -1 / +1
// across the periodic face (other values are returned unchanged). With n = 2
// the move 0 -> 1 is -1 and 1 -> 0 is +1; with n = 1 every step is 0.
__host__ __device__ __forceinline__ int periodic_step(int d, int n) {
  if (d == n - 1) return -1;
  if (d == 1 - n) return 1;
  return d;
}

// Direction code (dx+1) + 3(dy+1) + 9(dz+1) < 27 of a move from cell
// (i, j, k) to cell (a, b, c) of a periodic grid, or
// -1 when the destination is not one of the 27 cells around the source.
__device__ __forceinline__ int move_code(const Geom& g, int i, int j, int k, int a, int b, int c) {
  const int dx = periodic_step(a - i, g.nx), dy = periodic_step(b - j, g.ny), dz = periodic_step(c - k, g.nz);
  if (dx < -1 || dx > 1 || dy < -1 || dy > 1 || dz < -1 || dz > 1) return -1;
  return (dx + 1) + 3 * (dy + 1) + 9 * (dz + 1);
}

// Runs of the binned sort and the run mover: up to g.run_len (at most
// kRunCells = 32) consecutive interior cells of one x-row (segment, j, k). A record's run code packs its move
// direction d < 27 (bits 0-4) and its cell's offset in the run (bits 5-9);
// kNoMove marks a record that did not move to a neighbour.
constexpr int kRunCells = 32;
constexpr uint16_t kNoMove = 0xffff;
// Runs wanted before the run length shrinks below kRunCells.
constexpr long long kRunTarget = 16384;
__host__ __device__ __forceinline__ long long run_count(const Geom& g) {
  return (long long)((g.nx + g.run_len - 1) / g.run_len) * g.ny * g.nz;
}
__host__ __device__ __forceinline__ void run_cells(const Geom& g, long long run, int& i0, int& len, int& j, int& k) {
  const int segments = (g.nx + g.run_len - 1) / g.run_len;
  const int seg = int(run % segments);
  const long long row = run / segments;
  j = int(row % g.ny);
  k = int(row / g.ny);
  i0 = seg * g.run_len;
  len = g.nx - i0 < g.run_len ? g.nx - i0 : g.run_len;
}

// The non-unique vertices of a node field: every vertex of the (n+3)^3 box
// outside the unique periodic nodes [0, n)^3, enumerated as three z slabs
// (k = -1, n, n+1), then three y slabs and three x slabs of the remainder.
__host__ __device__ __forceinline__ long long shell_count(const Geom& g) {
  return 3LL * g.NX * g.NY + 3LL * g.NX * g.nz + 3LL * g.ny * g.nz;
}
__device__ __forceinline__ void shell_coordinates(const Geom& g, long long t, int& i, int& j, int& k) {
  const long long zs = (long long)g.NX * g.NY, ys = (long long)g.NX * g.nz, xs = (long long)g.ny * g.nz;
  if (t < 3 * zs) {
    const int p = int(t / zs);
    const long long r = t - p * zs;
    k = p == 0 ? -1 : g.nz + p - 1;
    i = int(r % g.NX) - 1;
    j = int(r / g.NX) - 1;
    return;
  }
  t -= 3 * zs;
  if (t < 3 * ys) {
    const int p = int(t / ys);
    const long long r = t - p * ys;
    j = p == 0 ? -1 : g.ny + p - 1;
    i = int(r % g.NX) - 1;
    k = int(r / g.NX);
    return;
  }
  t -= 3 * ys;
  const int p = int(t / xs);
  const long long r = t - p * xs;
  i = p == 0 ? -1 : g.nx + p - 1;
  j = int(r % g.ny);
  k = int(r / g.ny);
}

// Requests the 128-byte line holding p into L2 (no register, no wait).
__device__ __forceinline__ void prefetch_l2(const void* p) {
  asm volatile("prefetch.global.L2 [%0];" :: "l"(p));
}

// Programmatic dependent launch: a kernel launched with programmatic stream
// serialization may be scheduled while its predecessor drains; it waits here
// for the predecessor's completion and memory before touching its results.
// Without that launch attribute the wait returns at once.
__device__ __forceinline__ void wait_for_predecessor() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

// Launches `kernel` so that it may overlap the tail of the previous kernel
// on the stream (it must call wait_for_predecessor() first).
template <class... Params, class... Args>
inline cudaError_t launch_programmatic(void (*kernel)(Params...), dim3 grid, dim3 block, size_t smem,
                                       cudaStream_t s, Args... args) {
  cudaLaunchConfig_t config{};
  config.gridDim = grid;
  config.blockDim = block;
  config.dynamicSmemBytes = smem;
  config.stream = s;
  cudaLaunchAttribute attribute[1];
  attribute[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attribute[0].val.programmaticStreamSerializationAllowed = 1;
  config.attrs = attribute;
  config.numAttrs = 1;
  return cudaLaunchKernelEx(&config, kernel, args...);
}

// shell_coordinates in 32-bit arithmetic (t < shell_count < 2^31).
__device__ __forceinline__ void shell_coordinates32(const Geom& g, uint32_t t, int& i, int& j, int& k) {
  const uint32_t NX = uint32_t(g.NX), zs = NX * uint32_t(g.NY), ys = NX * uint32_t(g.nz),
                 xs = uint32_t(g.ny) * uint32_t(g.nz);
  if (t < 3 * zs) {
    const uint32_t p = t / zs, r = t - p * zs;
    k = p == 0 ? -1 : g.nz + int(p) - 1;
    i = int(r % NX) - 1;
    j = int(r / NX) - 1;
    return;
  }
  t -= 3 * zs;
  if (t < 3 * ys) {
    const uint32_t p = t / ys, r = t - p * ys;
    j = p == 0 ? -1 : g.ny + int(p) - 1;
    i = int(r % NX) - 1;
    k = int(r / NX);
    return;
  }
  t -= 3 * ys;
  const uint32_t p = t / xs, r = t - p * xs;
  i = p == 0 ? -1 : g.nx + int(p) - 1;
  j = int(r % uint32_t(g.ny));
  k = int(r / uint32_t(g.ny));
}

template <class T> __device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Block-wide sum for blockDim.x == Threads; every thread receives the total.
template <int Threads, class T>
__device__ __forceinline__ T block_sum(T v, T* scratch /* Threads/32 */) {
  v = warp_sum(v);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  __syncthreads();
  if (lane == 0) scratch[warp] = v;
  __syncthreads();
  T total = 0;
#pragma unroll
  for (int w = 0; w < Threads / 32; ++w) total += scratch[w];
  return total;
}

inline unsigned grid_for(long long n, int threads, unsigned cap = 148u * 16u) {
  long long b = (n + threads - 1) / threads;
  if (b < 1) b = 1;
  if (b > cap) b = cap;
  return unsigned(b);
}

}  // namespace tpicb200
