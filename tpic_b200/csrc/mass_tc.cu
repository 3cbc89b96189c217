// Tensor-core (tcgen05) mass-matrix and implicit-current assembly over the
// sorted records of up to two species per launch.
//
// The mass block of a corner pair is K_ab = sum_p s_p alpha_p W_pa W_pb with
// s = (beta/c) q (ecsim/mass_matrix/mass_matrix_scalar_device.hpp:25-97). With
// CIC weights W_pa = X_p(a_x) Y_p(a_y) Z_p(a_z), the pair weight factors per
// axis into one of three products, (1-x)^2, x(1-x) or x^2, so W_pa W_pb is the
// monomial m_pt of the per-axis class t = (a_x+b_x) + 3(a_y+b_y) + 9(a_z+b_z).
// A cell's 36 canonical pair blocks are therefore 27 monomial moments
//   G[t][c] = sum_p m_pt (s_p alpha_p[c]),  t < 27, c < 9,
// a dense contraction over the cell's particles: D = A^T B with K = particles.
// The implicit current of corner a, J_a = sum_p W_pa j_p with
// j_p = q_p/V alpha_p v_p (ecsim/current/implicit_current_device.hpp), rides
// along in three more B columns: since sum_b W_pb = 1, W_pa = sum_b W_pa W_pb
// and J_a[c] = sum_b H[t(a, b)][c] with H[t][c] = sum_p m_pt j_p[c].
//
// Tensor-core mapping (one CTA of four warps works on four cells at once):
//   A (tensor memory, M = 128 lanes x K columns): lane 32w + t holds m_pt of
//     cell w's particles (rows 27..31 of each quadrant are zero);
//   B (shared memory, K x N, no swizzle): columns 12w..12w+11 (TF32, N = 48,
//     K-major core matrices of 8 N-rows x 4 K-values) or 16w..16w+11 (BF16,
//     N = 64, MN-major core matrices of 8 K-rows x 8 N-values) hold
//     (s_p alpha_p, j_p) of cell w's particle p (the rest zero);
//   D (tensor memory, 128 x 48 / 64 FP32): D[32w + t][12w + c] = G_w[t][c]
//     (c < 9) and H_w[t][c - 9]; the off-diagonal blocks are never read.
// Column k of a chunk holds the k-th particle of each of the four cells, so
// the four cells share every MMA. Each 32-particle chunk is four
// tcgen05.mma.kind::tf32 (K = 8) issued by one thread; A and B are
// double-buffered so the next chunk is produced while the tensor core
// consumes the previous one (tcgen05.commit -> mbarrier, bounded waits).
// Operands are rounded to nearest (TF32 ties away, bf16 RN split) so the
// rounding is unbiased; accumulation is FP32. The epilogue reads G and H with
// tcgen05.ld, forms the 8x3 corner currents and stores the cell's moments
// (27x9 + 8x3 values; each group of four consecutive cells has one
// contiguous record of 16-byte words, word q = entry q of the four cells; a
// later launch adds to them in place). No atomics: the reference's flush issues up to 324
// atomics per cell (mass_matrix_mma_device.hpp:141-150).
// assemble_moments_kernel then forms every record entry of a unique node as
// the sum of the 1, 2, 4 or 8 cell moments that share it, in a fixed order.
//
// A cell's records of both species form one stream (species 0 first), so
// the chunk padding is paid once per cell rather than once per species.
//
// BF16x3 form: every operand v is split into hi = bf16(v) and lo = bf16(v - hi)
// (round-to-nearest) and D accumulates A_hi B_hi + A_hi B_lo + A_lo B_hi with
// tcgen05.mma.kind::f16 (BF16 inputs, FP32 accumulation, K = 16); B then has
// 16 columns per cell (N = 64) so each cell's block is whole 16-byte core rows.
#include "kernels.cuh"
#include "tcgen05.cuh"

#include <algorithm>

#include <cuda_bf16.h>

namespace tpicb200 {
namespace {

constexpr int kCells = 4;          // cells per CTA group (one per warp)
constexpr int kChunk = 32;         // particles per chunk (one per lane)
constexpr int kFuse = 2;           // species per launch
constexpr int kFacStride = 36;     // floats per factor row (16-byte aligned rows)
constexpr uint32_t kTmemCols = 128;
constexpr int kMassMoments = 27 * 9;                  // G[t][c] per cell
constexpr int kMoments = kMassMoments + 24;           // + J corner sums [a][c]
// Moment layout: each group of four consecutive cells has one contiguous
// record of kMoments 16-byte words, word q holding entry q of the four cells.
__host__ __device__ constexpr long long moment_index(long long cell, int q) {
  return ((cell >> 2) * kMoments + q) * 4 + (cell & 3);
}
constexpr uint32_t kDcol = 64;
constexpr int kCtasPerSm = 4;      // 4 x 128 tensor-memory columns = all 512
constexpr int kPermBuf = 256;      // ranks of a cell staged ahead (per warp and group)
// Per form: B columns per cell, N, bytes of one B tile, B tiles per buffer.
// TF32 (K-major): 8 K-chunks of 4 particles, each 6 N-groups x 128 bytes,
// padded by 16 bytes (K-chunk stride 784 B) so the 32 lanes' 4-byte stores
// of one column fall in 32 different banks.
// BF16 (MN-major): 8 N-chunks of 8 values, each 4 K-groups x 128 bytes.
constexpr uint32_t kTf32KChunk = 6 * 128 + 16;
template <bool Bf16> struct Form {
  static constexpr int cols = Bf16 ? 16 : 12;
  static constexpr int n = kCells * cols;
  static constexpr uint32_t tile_bytes = Bf16 ? uint32_t(n / 8) * 512u : 8u * kTf32KChunk;
  static constexpr int tiles = Bf16 ? 2 : 1;         // hi (+ lo)
};

// Monomial class of the corner pair (a, b).
__host__ __device__ constexpr int monomial_class(int a, int b) {
  return ((a & 1) + (b & 1)) + 3 * (((a >> 1) & 1) + ((b >> 1) & 1)) + 9 * (((a >> 2) & 1) + ((b >> 2) & 1));
}

struct TcSpecies {
  const double* rx;
  const double* ry;
  const double* rz;
  const float* u;
  const float* v;
  const float* w;
  const double* q;
  const int32_t* key;
  const uint32_t* counts;
  const uint32_t* offsets;
  float beta_over_c;
  // Sorted copy (perm null: records read in place).
  const uint32_t* perm;
  double* orx;
  double* ory;
  double* orz;
  float* ou;
  float* ov;
  float* ow;
  double* oq;
  int32_t* okey;
};

struct TcParams {
  TcSpecies sp[kFuse];
  int ns;
  float inv_volume;
  uint32_t wait_polls;  // polls of the stream kernel's chunk-loop waits before they give up
  uint32_t stall_chunk; // nonzero: the wait for chunk stall_chunk - 1 targets `never` (a test of the waits)
};

template <bool Bf16> struct __align__(128) TcShared {
  uint8_t btile[2][Form<Bf16>::tiles][Form<Bf16>::tile_bytes];
  float fac[kCells][13][kFacStride];  // row 12 stays zero (rows 27..31 of A)
  float bpoly[kCells][24];            // B(x, y, z) polynomial coefficients [c][k]
  float stage[kCells][kMoments + 1];
  float hsum[kCells][27 * 3];
  uint32_t sperm[2][kCells][kPermBuf];  // ranks of the cell of the current / next group
  uint64_t mbar[2];  // MMAs that read buffer b have completed
  uint64_t full[2];  // the four warps have written buffer b
  uint32_t tmem_base;
  uint32_t count[kCells];
};

__device__ __forceinline__ uint32_t pack_bf16(float lo_elem, float hi_elem) {
  const __nv_bfloat162 v = __floats2bfloat162_rn(lo_elem, hi_elem);  // .x (low half) = first element
  return *reinterpret_cast<const uint32_t*>(&v);
}
// s_p alpha_p (all nine entries, row-major) and the unscaled alpha for the
// current, as Response<float> but with the fast reciprocal: its ~1e-7
// relative error is far below the operand rounding of the tensor-core forms.
struct ScaledResponse {
  float a[9];
  float norm_square;
  __device__ __forceinline__ ScaledResponse(float bx, float by, float bz, float beta_over_c) {
    const float x = beta_over_c * bx, y = beta_over_c * by, z = beta_over_c * bz;
    norm_square = x * x + y * y + z * z;
    const float inverse = __fdividef(1.0f, 1.0f + norm_square);
    a[0] = (1.0f + x * x) * inverse;
    a[4] = (1.0f + y * y) * inverse;
    a[8] = (1.0f + z * z) * inverse;
    const float xy = x * y * inverse, xz = x * z * inverse, yz = y * z * inverse;
    const float sx = x * inverse, sy = y * inverse, sz = z * inverse;
    a[1] = xy + sz; a[2] = xz - sy; a[3] = xy - sz;
    a[5] = yz + sx; a[6] = xz + sy; a[7] = yz - sx;
  }
};

// Two values split into packed hi and lo bf16 pairs: hi = RN(v), lo = RN(v - hi)
// (v - hi is exact; the packed FMA v + (-1) hi evaluates both lanes at once).
__device__ __forceinline__ void split_pair(float2 v, uint32_t& hi, uint32_t& lo) {
  const __nv_bfloat162 h = __float22bfloat162_rn(v);
  const float2 r = __ffma2_rn(__bfloat1622float2(h), make_float2(-1.0f, -1.0f), v);
  hi = *reinterpret_cast<const uint32_t*>(&h);
  lo = pack_bf16(r.x, r.y);
}

template <bool Bf16>
__global__ void __launch_bounds__(128, kCtasPerSm) tc_deposit_kernel(Geom g, TcParams tp,
    const float* __restrict__ bnode, float* __restrict__ mom, int accumulate,
    uint32_t* invalid) {
  using F = Form<Bf16>;
  constexpr int kCols = F::cols;
  constexpr int kN = F::n;
  __shared__ TcShared<Bf16> sh;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const long long nn = g.nodes;
  if (warp == 0) {
    tc::tmem_alloc(&sh.tmem_base, kTmemCols);
    tc::tmem_relinquish();
  }
  if (threadIdx.x == 0) {
    tc::mbar_init(&sh.mbar[0], 1);
    tc::mbar_init(&sh.mbar[1], 1);
    tc::mbar_init(&sh.full[0], kCells);
    tc::mbar_init(&sh.full[1], kCells);
    tc::fence_mbar_init();
  }
  sh.fac[warp][12][lane] = 0.0f;
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tmem = sh.tmem_base;
  const uint32_t lane_base = uint32_t(32 * warp) << 16;
  constexpr uint32_t idesc = tc::instr_desc(Bf16 ? 1u : 2u, 128, kN, Bf16 ? 1u : 0u);
  // Bit b of `phase` / `pending`: the parity to wait for on mbar[b] and
  // whether MMAs reading buffer b are in flight.
  uint32_t phase = 0, pending = 0;
  uint32_t full_phase = 0;  // bit b: the parity of full[b] the MMA thread waits for
  int buf = 0;
  bool failed = false;
  // A bounded wait that timed out: the warps finish the group, which then
  // ends the kernel with the error bit (every warp reaches the same barriers).
  bool bad = false;

  const long long cells = (long long)g.nx * g.ny * g.nz;
  const long long groups = (cells + kCells - 1) / kCells;
  // Monomial row of this thread in its warp's quadrant.
  const int t_row = lane;
  const int tx = t_row % 3, tyz = t_row / 3;
  const bool two = tp.ns > 1;

  // Software pipeline: the metadata and B corners of the next group and the
  // records of the next chunk (possibly the next group's first) are loaded
  // while the current chunk is produced and consumed.
  struct Meta {
    int ci, cj, ck;
    uint32_t c0, c1, f0, f1;
    int32_t bin;
    bool live;
    float bval;  // lane < 24: B corner (lane / 3) component (lane % 3)
  };
  struct Rec {
    double fx, fy, fz, q;
    float u, v, w;
    int32_t key;
    uint32_t pos;  // sorted position
    bool present, second;
  };
  auto load_meta = [&](long long grp_) {
    Meta m{0, 0, 0, 0u, 0u, 0u, 0u, -1, false, 0.0f};
    const long long cell = grp_ * kCells + warp;
    if (grp_ < groups && cell < cells) {
      m.live = true;
      m.ci = int(cell % g.nx); m.cj = int((cell / g.nx) % g.ny); m.ck = int(cell / ((long long)g.nx * g.ny));
      m.bin = g.encode(m.ci, m.cj, m.ck);
      m.c0 = tp.sp[0].counts[m.bin];
      m.f0 = tp.sp[0].offsets[m.bin];
      if (two) {
        m.c1 = tp.sp[1].counts[m.bin];
        m.f1 = tp.sp[1].offsets[m.bin];
      }
      if (lane < 24) {
        const int a = lane / 3, c = lane % 3;
        m.bval = bnode[c * nn + g.node(m.ci + (a & 1), m.cj + ((a >> 1) & 1), m.ck + ((a >> 2) & 1))];
      }
    }
    return m;
  };
  // Records read through ranks: each warp copies its next cell's ranks to
  // shared memory a group ahead (cp.async), so that a record load waits for
  // a shared-memory read rather than a second global load.
  const bool gathered = tp.sp[0].perm || (two && tp.sp[1].perm);
  auto prefetch_ranks = [&](const Meta& m, int b) {
    if (!m.live) return;
    const uint32_t total = min(m.c0 + m.c1, uint32_t(kPermBuf));
    for (uint32_t k = lane; k < total; k += 32) {
      const bool s1 = k >= m.c0;
      const uint32_t* perm = s1 ? tp.sp[1].perm : tp.sp[0].perm;
      if (perm) tc::cp_async4(&sh.sperm[b][warp][k], perm + (s1 ? m.f1 + (k - m.c0) : m.f0 + k));
    }
    tc::cp_async_commit();
  };
  auto load_rec = [&](const Meta& m, uint32_t k, int b) {
    Rec r{0.0, 0.0, 0.0, 0.0, 0.0f, 0.0f, 0.0f, -1, 0u, false, false};
    if (k < m.c0 + m.c1) {
      const bool s1 = k >= m.c0;
      r.pos = s1 ? m.f1 + (k - m.c0) : m.f0 + k;
      const uint32_t* perm = s1 ? tp.sp[1].perm : tp.sp[0].perm;
      const uint32_t n = perm ? (k < uint32_t(kPermBuf) ? sh.sperm[b][warp][k] : perm[r.pos]) : r.pos;
      r.present = true;
      r.second = s1;
      r.fx = (s1 ? tp.sp[1].rx : tp.sp[0].rx)[n];
      r.fy = (s1 ? tp.sp[1].ry : tp.sp[0].ry)[n];
      r.fz = (s1 ? tp.sp[1].rz : tp.sp[0].rz)[n];
      r.q = (s1 ? tp.sp[1].q : tp.sp[0].q)[n];
      r.u = (s1 ? tp.sp[1].u : tp.sp[0].u)[n];
      r.v = (s1 ? tp.sp[1].v : tp.sp[0].v)[n];
      r.w = (s1 ? tp.sp[1].w : tp.sp[0].w)[n];
      r.key = (s1 ? tp.sp[1].key : tp.sp[0].key)[n];
    }
    return r;
  };
  Meta cur = load_meta(blockIdx.x);
  int rb = 0;  // rank buffer of the current group
  if (gathered) {
    prefetch_ranks(cur, rb);
    tc::cp_async_wait_all();
    __syncwarp();
  }
  Rec pre = load_rec(cur, lane, rb);

  for (long long grp = blockIdx.x; grp < groups && !failed; grp += gridDim.x) {
    const Meta nxt = load_meta(grp + gridDim.x);
    const bool live = cur.live;
    const uint32_t count = cur.c0 + cur.c1;
    const int32_t bin = cur.bin;
    // Trilinear B as a polynomial in the cell fractions,
    // B = c0 + c1 x + c2 y + c3 z + c4 xy + c5 xz + c6 yz + c7 xyz, from the
    // corner values b_a (corner a = x + 2y + 4z).
    {
      float bc[8];
#pragma unroll
      for (int a = 0; a < 8; ++a) bc[a] = __shfl_sync(0xffffffffu, cur.bval, 3 * a + (lane < 3 ? lane : 0));
      if (lane < 3) {
        float* cp = sh.bpoly[warp] + 8 * lane;
        const float z0 = live ? 1.0f : 0.0f;
        cp[0] = z0 * bc[0];
        cp[1] = z0 * (bc[1] - bc[0]);
        cp[2] = z0 * (bc[2] - bc[0]);
        cp[3] = z0 * (bc[4] - bc[0]);
        cp[4] = z0 * ((bc[3] - bc[2]) - (bc[1] - bc[0]));
        cp[5] = z0 * ((bc[5] - bc[4]) - (bc[1] - bc[0]));
        cp[6] = z0 * ((bc[6] - bc[4]) - (bc[2] - bc[0]));
        cp[7] = z0 * (((bc[7] - bc[6]) - (bc[5] - bc[4])) - ((bc[3] - bc[2]) - (bc[1] - bc[0])));
      }
    }
    if (lane == 0) sh.count[warp] = count;
    __syncthreads();
    uint32_t maxc = sh.count[0];
#pragma unroll
    for (int c = 1; c < kCells; ++c) maxc = max(maxc, sh.count[c]);
    // The next group's ranks travel while this group is processed.
    if (gathered) prefetch_ranks(nxt, rb ^ 1);
    auto load_next_group = [&]() {
      if (gathered) {
        tc::cp_async_wait_all();
        __syncwarp();
      }
      return load_rec(nxt, lane, rb ^ 1);
    };
    if (maxc == 0) pre = load_next_group();

    for (uint32_t chunk = 0; chunk < maxc; chunk += kChunk) {
      // The buffer is free once the MMAs that read it have completed.
      if (pending & (1u << buf)) {
        if (!tc::mbar_wait(&sh.mbar[buf], (phase >> buf) & 1u)) bad = true;
        phase ^= 1u << buf;
        pending &= ~(1u << buf);
      }
      const Rec rec = pre;
      pre = chunk + kChunk < maxc ? load_rec(cur, chunk + kChunk + lane, rb) : load_next_group();
      // Particle phase: one record per lane.
      float bv[kCols];
      float fac[12];
#pragma unroll
      for (int c = 0; c < kCols; ++c) bv[c] = 0.0f;
#pragma unroll
      for (int f = 0; f < 12; ++f) fac[f] = 0.0f;
      if (rec.present) {
        // The sorted copy of the record, when the sort left it to this pass.
        const TcSpecies& sp = rec.second ? tp.sp[1] : tp.sp[0];
        if (sp.orx) {
          const uint32_t o = rec.pos;
          sp.orx[o] = rec.fx; sp.ory[o] = rec.fy; sp.orz[o] = rec.fz;
          sp.ou[o] = rec.u; sp.ov[o] = rec.v; sp.ow[o] = rec.w;
          sp.oq[o] = rec.q; sp.okey[o] = rec.key;
        }
        const double fx = rec.fx, fy = rec.fy, fz = rec.fz;
        bool ok = rec.key == bin && fx >= 0 && fx < 1 && fy >= 0 && fy < 1 && fz >= 0 && fz < 1;
        if (ok) {
          const float x = float(fx), y = float(fy), z = float(fz);
          float b[3];
#pragma unroll
          for (int c = 0; c < 3; ++c) {
            const float4 lo4 = *reinterpret_cast<const float4*>(&sh.bpoly[warp][8 * c]);
            const float4 hi4 = *reinterpret_cast<const float4*>(&sh.bpoly[warp][8 * c + 4]);
            const float t1 = fmaf(z, hi4.w, hi4.x);              // c4 + z c7
            const float t2 = fmaf(z, hi4.y, fmaf(y, t1, lo4.y));  // c1 + y (c4 + z c7) + z c5
            const float t3 = fmaf(z, hi4.z, lo4.z);              // c2 + z c6
            b[c] = fmaf(z, lo4.w, fmaf(y, t3, fmaf(x, t2, lo4.x)));
          }
          const float bo = rec.second ? tp.sp[1].beta_over_c : tp.sp[0].beta_over_c;
          const ScaledResponse r(b[0], b[1], b[2], bo);
          const float charge = float(rec.q);
          const float hx = r.a[0] * rec.u + r.a[1] * rec.v + r.a[2] * rec.w;
          const float hy = r.a[3] * rec.u + r.a[4] * rec.v + r.a[5] * rec.w;
          const float hz = r.a[6] * rec.u + r.a[7] * rec.v + r.a[8] * rec.w;
          const float qv = charge * tp.inv_volume;
          const float scale = bo * charge;
          bv[9] = qv * hx; bv[10] = qv * hy; bv[11] = qv * hz;
#pragma unroll
          for (int e = 0; e < 9; ++e) bv[e] = r.a[e] * scale;
          // One test covers every product: a non-finite input makes the sum non-finite.
          ok = isfinite(bv[9] + bv[10] + bv[11] + r.norm_square + scale);
          if (ok) {
            const float cx = 1.0f - x, cy = 1.0f - y, cz = 1.0f - z;
            const float X[3] = {cx * cx, x * cx, x * x};
            const float Y[3] = {cy * cy, y * cy, y * y};
            const float Z[3] = {cz * cz, z * cz, z * z};
            fac[0] = X[0]; fac[1] = X[1]; fac[2] = X[2];
#pragma unroll
            for (int tz = 0; tz < 3; ++tz)
#pragma unroll
              for (int ty = 0; ty < 3; ++ty) fac[3 + ty + 3 * tz] = Y[ty] * Z[tz];
          } else {
#pragma unroll
            for (int c = 0; c < 12; ++c) bv[c] = 0.0f;
          }
        }
        if (!ok) atomicAdd(invalid, 1u);
      }
      // B tile.
      if constexpr (!Bf16) {
        // K-major: value (n, k) at (n%8)*16 + (n/8)*128 + (k/4)*784 + (k%4)*4.
        uint8_t* bt = sh.btile[buf][0] + (lane >> 2) * kTf32KChunk + (lane & 3) * 4;
#pragma unroll
        for (int c = 0; c < kCols; ++c) {
          const int n = kCols * warp + c;
          *reinterpret_cast<uint32_t*>(bt + (n & 7) * 16 + (n >> 3) * 128) = tc::to_tf32(bv[c]);
        }
      } else {
        // MN-major: 8 K-rows x 16 bytes of N-values per core matrix, K-groups
        // 128 B apart, 16-byte N-chunks 512 B apart.
#pragma unroll
        for (int j = 0; j < 2; ++j) {
          uint32_t ph[4], pl[4];
#pragma unroll
          for (int e = 0; e < 4; ++e) split_pair(make_float2(bv[8 * j + 2 * e], bv[8 * j + 2 * e + 1]), ph[e], pl[e]);
          const int off = (2 * warp + j) * 512 + (lane >> 3) * 128 + (lane & 7) * 16;
          *reinterpret_cast<uint4*>(sh.btile[buf][0] + off) = make_uint4(ph[0], ph[1], ph[2], ph[3]);
          *reinterpret_cast<uint4*>(sh.btile[buf][1] + off) = make_uint4(pl[0], pl[1], pl[2], pl[3]);
        }
      }
#pragma unroll
      for (int f = 0; f < 12; ++f) sh.fac[warp][f][lane] = fac[f];
      __syncwarp();
      // A: lane t of warp w writes m_pt of the chunk's 32 particles into
      // tensor-memory lane 32w + t (TF32: columns 32*buf .. +31; BF16: the
      // hi pairs in columns 32*buf .. +15 and the lo pairs in +16 .. +31).
      const bool row = t_row < 27;
      const float* xrow = sh.fac[warp][row ? tx : 12];
      const float* yzrow = sh.fac[warp][row ? 3 + tyz : 12];
      if constexpr (!Bf16) {
#pragma unroll
        for (int q8 = 0; q8 < 4; ++q8) {
          uint32_t m[8];
#pragma unroll
          for (int h = 0; h < 2; ++h) {
            const float4 xf = *reinterpret_cast<const float4*>(xrow + 8 * q8 + 4 * h);
            const float4 yzf = *reinterpret_cast<const float4*>(yzrow + 8 * q8 + 4 * h);
            const float2 lo2 = __fmul2_rn(make_float2(xf.x, xf.y), make_float2(yzf.x, yzf.y));
            const float2 hi2 = __fmul2_rn(make_float2(xf.z, xf.w), make_float2(yzf.z, yzf.w));
            m[4 * h + 0] = tc::to_tf32(lo2.x);
            m[4 * h + 1] = tc::to_tf32(lo2.y);
            m[4 * h + 2] = tc::to_tf32(hi2.x);
            m[4 * h + 3] = tc::to_tf32(hi2.y);
          }
          tc::tmem_st8(tmem + lane_base + (buf ? 32u : 0u) + 8 * q8, m);
        }
      } else {
#pragma unroll
        for (int q16 = 0; q16 < 2; ++q16) {
          uint32_t mh[8], ml[8];
#pragma unroll
          for (int h = 0; h < 4; ++h) {
            const float4 xf = *reinterpret_cast<const float4*>(xrow + 16 * q16 + 4 * h);
            const float4 yzf = *reinterpret_cast<const float4*>(yzrow + 16 * q16 + 4 * h);
            split_pair(__fmul2_rn(make_float2(xf.x, xf.y), make_float2(yzf.x, yzf.y)), mh[2 * h + 0], ml[2 * h + 0]);
            split_pair(__fmul2_rn(make_float2(xf.z, xf.w), make_float2(yzf.z, yzf.w)), mh[2 * h + 1], ml[2 * h + 1]);
          }
          tc::tmem_st8(tmem + lane_base + (buf ? 32u : 0u) + 8 * q16, mh);
          tc::tmem_st8(tmem + lane_base + (buf ? 32u : 0u) + 16 + 8 * q16, ml);
        }
      }
      tc::tmem_wait_st();
      tc::fence_proxy_async_smem();
      tc::fence_before_sync();
      // This warp's share of the chunk is written: one arrival per warp; the
      // MMA thread waits for all four, the other warps go on.
      __syncwarp();
      if (lane == 0) tc::mbar_arrive(&sh.full[buf]);
      if (threadIdx.x == 0) {
        if (!tc::mbar_wait(&sh.full[buf], (full_phase >> buf) & 1u)) bad = true;
        full_phase ^= 1u << buf;
        tc::fence_after_sync();
        const uint32_t abase = tmem + (buf ? 32u : 0u);
        if constexpr (!Bf16) {
          const uint32_t bbase = tc::smem_u32(sh.btile[buf][0]);
#pragma unroll
          for (int s = 0; s < 4; ++s)
            tc::mma_tf32_ts(tmem + kDcol, abase + 8 * s,
                            tc::smem_desc(bbase + 2 * s * kTf32KChunk, kTf32KChunk, 128), idesc,
                            (chunk > 0 || s > 0) ? 1u : 0u);
        } else {
          const uint32_t bhi = tc::smem_u32(sh.btile[buf][0]), blo = tc::smem_u32(sh.btile[buf][1]);
#pragma unroll
          for (int s = 0; s < 2; ++s) {
            const uint32_t a_hi = abase + 8 * s, a_lo = abase + 16 + 8 * s;
            tc::mma_f16_ts(tmem + kDcol, a_hi, tc::smem_desc(bhi + s * 256, 128, 512), idesc,
                           (chunk > 0 || s > 0) ? 1u : 0u);
            tc::mma_f16_ts(tmem + kDcol, a_hi, tc::smem_desc(blo + s * 256, 128, 512), idesc, 1u);
            tc::mma_f16_ts(tmem + kDcol, a_lo, tc::smem_desc(bhi + s * 256, 128, 512), idesc, 1u);
          }
        }
        tc::commit(&sh.mbar[buf]);
      }
      pending |= 1u << buf;
      buf ^= 1;
    }

    // Moments: wait for the group's last MMA, read G and H of this warp's
    // cell and form the corner currents J[a][c] = sum_b H[t(a, b)][c].
    float* stage = sh.stage[warp];
    float* hs = sh.hsum[warp];
    if (maxc > 0) {
      const int last = buf ^ 1;
      const bool ok = tc::mbar_wait(&sh.mbar[last], (phase >> last) & 1u);
      phase ^= 1u << last;
      pending &= ~(1u << last);
      tc::fence_after_sync();
      if (__syncthreads_or(!ok || bad)) {
        failed = true;
        break;
      }
      uint32_t g8[8], g4[4];
      tc::tmem_ld8(tmem + lane_base + kDcol + kCols * warp, g8);
      tc::tmem_ld4(tmem + lane_base + kDcol + kCols * warp + 8, g4);
      tc::tmem_wait_ld();
      if (t_row < 27) {
        const bool use = live && count > 0;
#pragma unroll
        for (int e = 0; e < 8; ++e) stage[t_row * 9 + e] = use ? __uint_as_float(g8[e]) : 0.0f;
        stage[t_row * 9 + 8] = use ? __uint_as_float(g4[0]) : 0.0f;
#pragma unroll
        for (int c = 0; c < 3; ++c) hs[t_row * 3 + c] = use ? __uint_as_float(g4[1 + c]) : 0.0f;
      }
      __syncwarp();
      if (lane < 24) {
        const int a = lane / 3, c = lane - 3 * (lane / 3);
        float sum = 0.0f;
#pragma unroll
        for (int b = 0; b < 8; ++b) sum += hs[monomial_class(a, b) * 3 + c];
        stage[kMassMoments + lane] = sum;
      }
    } else {
      for (int i = lane; i < kMoments; i += 32) stage[i] = 0.0f;
    }
    __syncthreads();
    // Moment store: entry q of the group's four cells is one 16-byte word of
    // the group's contiguous record (coalesced across q).
    bool bad_value = false;
    for (int qi = threadIdx.x; qi < kMoments; qi += blockDim.x) {
      float4 val = make_float4(sh.stage[0][qi], sh.stage[1][qi], sh.stage[2][qi], sh.stage[3][qi]);
      if (!isfinite(val.x + val.y + val.z + val.w)) {
        bad_value = true;
        val.x = isfinite(val.x) ? val.x : 0.0f;
        val.y = isfinite(val.y) ? val.y : 0.0f;
        val.z = isfinite(val.z) ? val.z : 0.0f;
        val.w = isfinite(val.w) ? val.w : 0.0f;
      }
      float4* dst = reinterpret_cast<float4*>(mom + (grp * kMoments + qi) * kCells);
      if (accumulate) {
        const float4 old = *dst;
        val.x += old.x; val.y += old.y; val.z += old.z; val.w += old.w;
      }
      *dst = val;
    }
    if (bad_value) atomicAdd(invalid, 1u);
    // D is overwritten by the next group's first MMA only after every warp
    // has read it.
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    cur = nxt;
    rb ^= 1;
  }

  if (failed && threadIdx.x == 0) atomicAdd(invalid, 1u << 20);
  // Retire in-flight MMAs (bounded) before freeing tensor memory.
#pragma unroll
  for (int b = 0; b < 2; ++b)
    if (pending & (1u << b)) tc::mbar_wait(&sh.mbar[b], (phase >> b) & 1u);
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  if (warp == 0) tc::tmem_dealloc(tmem, kTmemCols);
}


// ---------------------------------------------------------------------------
// Stream form of the BF16x3 deposition.
//
// Each warp owns a sequence of batches of four consecutive cells (batches
// gw, gw + W, gw + 2W, ... for global warp gw of W) and walks a batch's
// records as one stream - cell by cell, species 0 before species 1 in a
// cell - in chunks of up to 32 records (one per lane). A chunk never crosses
// the end of a cell, so its cell is the same for every lane and the warp's
// quadrant of D holds one accumulator block, which is flushed - read from
// tensor memory, then zeroed - once the MMAs of the cell's last chunk have
// completed and before the warp's next chunk is written. A chunk may cross
// from the cell's species-0 records to its species-1 records (each lane
// reads its own species' arrays): a cell of c0 + c1 records takes
// ceil((c0 + c1) / 32) chunks, not ceil(c0 / 32) + ceil(c1 / 32). Every batch
// starts a new chunk, so a cell's summation order depends only on its
// batch's counts: the moments are reproducible.
//
// The four warps of a CTA share every MMA (M = 128 = four quadrants of 32
// monomial rows; rows 27..31 of a quadrant stay zero):
//   A (shared memory, MN-major, 128 x 32, BF16 hi and lo): row 32w + t,
//     column k holds m_t of warp w's lane-k record;
//   B (shared memory, MN-major, 32 x 64, BF16 hi and lo): columns
//     16w..16w+11 hold the 12 values (s alpha, j) of warp w's lane-k record
//     in row k, columns 16w+12..16w+15 stay zero;
//   D (tensor memory, 128 x 64 FP32): D[32w + t][16w + c] = G[t][c] (c < 9)
//     and H[t][c - 9] (9 <= c < 12); the off-diagonal blocks are never read.
// Both operands are single-buffered: a warp writes chunk j's A and B after the
// MMAs of chunk j - 1 have completed, which it waits for anyway to flush the
// cell that ended in chunk j - 1. The warps build the A rows of their own
// records directly (27 products per lane), with no transposition. The last
// warp to finish writing a chunk's operands (an acquire-release counter per
// chunk parity) issues its MMAs, so no warp waits for the others.
//
// Records are fetched in a software pipeline per warp: the walk of chunk
// j + 3 copies the ranks (cp.async), chunk j + 2's records are requested
// into L2 (when read through ranks), chunk j + 1's record loads are in
// flight while chunk j is computed. A warp that has run out of batches keeps
// arriving with no data while any warp of its CTA still has chunks (each
// warp publishes, per chunk, whether it has another; the issuer publishes
// the CTA's answer), and the CTA's warps leave the loop together.
constexpr int kBatch = 4;                  // cells per batch
constexpr int kStreamN = 64;               // B columns: 4 quadrants x 16 (12 used)
constexpr uint32_t kStreamTmemCols = 64;
constexpr int kMetaSlots = 4;              // batches of chunks j .. j + 3 (the walk of j + 3 precedes chunk j)

struct StreamMeta {
  int32_t bin[kBatch];
  float bpoly[kBatch][24];
};

struct __align__(16) StreamShared {
  uint8_t a[2][128 * 32 * 2];        // A hi, lo: 16 M-chunks x 512 B (4 K-groups x 128 B)
  uint8_t b[2][kStreamN / 8 * 512];  // B hi, lo: 12 N-chunks x 512 B
  float stage[kCells][kBatch][kMoments + 1];
  float scratch[kCells][96];  // a batch's B corners / the H rows of a flushed cell
  StreamMeta meta[kCells][kMetaSlots];
  uint32_t rank[kCells][4][32];  // per warp, chunk j & 3: each lane's record index (cp.async)
  uint32_t more[2];     // byte w of word j & 1: warp w has a chunk after chunk j
  uint32_t arrived[2];  // arrivals of the chunks of each parity (monotonic)
  uint32_t decision;    // (chunk << 1) | (some warp has a chunk after it)
  uint64_t mma_bar;     // the MMAs of a chunk have completed
  uint64_t never;       // an mbarrier that nothing arrives on (TcParams::stall_chunk)
  uint32_t tmem_base;
};

// Per-lane record of a chunk: rank (record index in the read slot), sorted
// position, flags (bit 0 present, bit 1 species 1).
struct StreamLane {
  uint32_t idx, pos, flags;
};
// Warp-uniform chunk description: batch and bits (ended cells 0-3,
// nonempty cells 4-7, valid 13, metadata slot 14-15, cell slot 16-17).
struct StreamInfo {
  int bid;
  uint32_t bits;
};
struct StreamRec {
  double fx, fy, fz, q;
  float u, v, w;
  int32_t key;
  uint32_t pos, flags;
};
struct MetaRegs {
  uint32_t c0, c1, f0, f1;
  int32_t bin;
  float corner[3];
};

__global__ void __launch_bounds__(128, kCtasPerSm) tc_stream_kernel(Geom g, TcParams tp,
    const float* __restrict__ bnode, float* __restrict__ mom, int accumulate,
    uint32_t* invalid, int batches) {
  extern __shared__ __align__(16) uint8_t stream_smem[];
  StreamShared& sh = *reinterpret_cast<StreamShared*>(stream_smem);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int W = int(gridDim.x) * kCells;
  const long long nn = g.nodes;
  const long long cells = (long long)g.nx * g.ny * g.nz;
  const bool two = tp.ns > 1;
  if (warp == 0) {
    tc::tmem_alloc(&sh.tmem_base, kStreamTmemCols);
    tc::tmem_relinquish();
  }
  if (threadIdx.x == 0) {
    tc::mbar_init(&sh.mma_bar, 1);
    tc::mbar_init(&sh.never, 1);
    tc::fence_mbar_init();
    sh.more[0] = sh.more[1] = 0u;
    sh.arrived[0] = sh.arrived[1] = 0u;
    sh.decision = 0xFFFFFFFEu;
  }
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tmem = sh.tmem_base;
  // This warp's 12 accumulator columns, in its own 32 lanes.
  const uint32_t dq = tmem + (uint32_t(32 * warp) << 16) + 16u * warp;
  {
    const uint32_t z[8] = {0u, 0u, 0u, 0u, 0u, 0u, 0u, 0u};
    const uint32_t z4[4] = {0u, 0u, 0u, 0u};
    tc::tmem_st8(dq, z);
    tc::tmem_st4(dq + 8, z4);
    tc::tmem_wait_st();
  }
  constexpr uint32_t idesc = tc::instr_desc(1u, 128, kStreamN, 1u, 1u);

  // Batch metadata: lanes 0..3 load the counts and offsets of cell slot
  // `lane`; lane l loads B corner values (l >> 2) + 8i of slot l & 3.
  auto fetch_meta = [&](int bid) {
    MetaRegs r{0u, 0u, 0u, 0u, -1, {0.0f, 0.0f, 0.0f}};
    const long long cell = (long long)bid * kBatch + (lane & 3);
    if (bid < batches && cell < cells) {
      const uint32_t c = uint32_t(cell), nx = uint32_t(g.nx), ny = uint32_t(g.ny);
      const uint32_t row = c / nx;
      const int ci = int(c - row * nx), cj = int(row % ny), ck = int(row / ny);
      r.bin = g.encode(ci, cj, ck);
      if (lane < kBatch) {
        r.c0 = tp.sp[0].counts[r.bin];
        r.f0 = tp.sp[0].offsets[r.bin];
        if (two) {
          r.c1 = tp.sp[1].counts[r.bin];
          r.f1 = tp.sp[1].offsets[r.bin];
        }
      }
#pragma unroll
      for (int i = 0; i < 3; ++i) {
        const int idx = (lane >> 2) + 8 * i, a = idx / 3, comp = idx - 3 * a;
        r.corner[i] = bnode[comp * nn + g.node(ci + (a & 1), cj + ((a >> 1) & 1), ck + ((a >> 2) & 1))];
      }
    }
    return r;
  };
  // The walk: a warp-uniform cursor over this warp's batches. Per batch,
  // the eight (cell, species) ranges of its stream: lane r < 8 holds the
  // stream end of range r = 2 slot + species and its sorted-array offset
  // minus its stream start; cb1, cb2, cb3, ctot are the cell ends.
  int cbid = blockIdx.x * kCells + warp;  // current batch
  int cslot = 0;                          // its metadata slot
  uint32_t rend = 0, roff = 0;
  uint32_t cb1 = 0, cb2 = 0, cb3 = 0, ctot = 0;
  uint32_t cnonempty = 0;  // nonempty cells of the batch
  uint32_t cbase = 0;      // stream position of the next chunk
  uint32_t cdone = 0;      // cells of the batch already ended
  bool cend = cbid >= batches, cnext = false;
  // Writes a batch's metadata into its slot and sets the cursor's batch
  // state: counts and offsets, bins and the trilinear B of each cell as a
  // polynomial in the cell fractions,
  // B = c0 + c1 x + c2 y + c3 z + c4 xy + c5 xz + c6 yz + c7 xyz.
  auto enter_batch = [&](const MetaRegs& r) {
    StreamMeta& m = sh.meta[warp][cslot];
    float* tmp = sh.scratch[warp];
    const int cell_slot = (lane >> 1) & 3;
    const uint32_t c0 = __shfl_sync(0xffffffffu, r.c0, cell_slot), c1 = __shfl_sync(0xffffffffu, r.c1, cell_slot);
    const uint32_t f0 = __shfl_sync(0xffffffffu, r.f0, cell_slot), f1 = __shfl_sync(0xffffffffu, r.f1, cell_slot);
    const uint32_t n = lane < 2 * kBatch ? ((lane & 1) ? c1 : c0) : 0u;
    uint32_t incl = n;  // inclusive scan over the ranges
#pragma unroll
    for (int o = 1; o < 2 * kBatch; o <<= 1) {
      const uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += t;
    }
    rend = incl;
    roff = ((lane & 1) ? f1 : f0) - (incl - n);
    if (lane < kBatch) m.bin[lane] = r.bin;
#pragma unroll
    for (int i = 0; i < 3; ++i) tmp[(lane & 3) * 24 + (lane >> 2) + 8 * i] = r.corner[i];
    cb1 = __shfl_sync(0xffffffffu, incl, 1);
    cb2 = __shfl_sync(0xffffffffu, incl, 3);
    cb3 = __shfl_sync(0xffffffffu, incl, 5);
    ctot = __shfl_sync(0xffffffffu, incl, 7);
    cnonempty = __ballot_sync(0xffffffffu, lane < kBatch && r.c0 + r.c1 > 0u) & 0xFu;
    __syncwarp();
    if (lane < 3 * kBatch) {
      const int s = lane / 3, c = lane - 3 * s;
      float bc[8];
#pragma unroll
      for (int a = 0; a < 8; ++a) bc[a] = tmp[s * 24 + 3 * a + c];
      float* cp = m.bpoly[s] + 8 * c;
      cp[0] = bc[0];
      cp[1] = bc[1] - bc[0];
      cp[2] = bc[2] - bc[0];
      cp[3] = bc[4] - bc[0];
      cp[4] = (bc[3] - bc[2]) - (bc[1] - bc[0]);
      cp[5] = (bc[5] - bc[4]) - (bc[1] - bc[0]);
      cp[6] = (bc[6] - bc[4]) - (bc[2] - bc[0]);
      cp[7] = ((bc[7] - bc[6]) - (bc[5] - bc[4])) - ((bc[3] - bc[2]) - (bc[1] - bc[0]));
    }
    __syncwarp();
    cbase = 0;
    cdone = 0;
  };
  MetaRegs pf = fetch_meta(cbid);
  if (!cend) {
    enter_batch(pf);
    pf = fetch_meta(cbid + W);
  }
  auto walk = [&](StreamLane& L, StreamInfo& I, uint32_t chunk) {
    L = StreamLane{0u, 0u, 0u};
    I = StreamInfo{0, 0u};
    if (cnext) {  // the previous chunk finished the batch
      cnext = false;
      cbid += W;
      cslot = cslot == kMetaSlots - 1 ? 0 : cslot + 1;
      if (cbid >= batches) {
        cend = true;
      } else {
        enter_batch(pf);
        pf = fetch_meta(cbid + W);
      }
    }
    if (cend) return;
    // The chunk [cbase, end): at most 32 records of the cell of the first
    // range that ends above cbase (empty ranges end at or below it); the
    // chunk may hold the end of the cell's species-0 range and the start of
    // its species-1 range.
    const uint32_t above = __ballot_sync(0xffffffffu, lane < 2 * kBatch && rend > cbase);
    // A batch without records has no range: its one chunk is empty.
    const int cell_slot = above ? (__ffs(above) - 1) >> 1 : 0;
    const uint32_t first_end = __shfl_sync(0xffffffffu, rend, 2 * cell_slot);
    const uint32_t cell_end = __shfl_sync(0xffffffffu, rend, 2 * cell_slot + 1);
    const uint32_t end = above ? min(cbase + 32u, cell_end) : cbase;
    // Each lane's range (species) and its sorted-array offset.
    const uint32_t p = cbase + lane;
    const uint32_t second = p >= first_end ? 1u : 0u;
    const uint32_t offset = __shfl_sync(0xffffffffu, roff, 2 * cell_slot + int(second));
    // Cells ending in this chunk (empty cells at or below `end` included).
    uint32_t ended = (cb1 <= end ? 1u : 0u) | (cb2 <= end ? 2u : 0u) | (cb3 <= end ? 4u : 0u) |
                     (ctot <= end ? 8u : 0u);
    ended &= ~cdone;
    cdone |= ended;
    const bool last = end >= ctot;
    I.bid = cbid;
    I.bits = ended | (cnonempty << 4) | (1u << 13) | (uint32_t(cslot) << 14) | (uint32_t(cell_slot) << 16);
    if (p < end) {
      L.pos = p + offset;
      const uint32_t* perm = second ? tp.sp[1].perm : tp.sp[0].perm;
      uint32_t* dst = &sh.rank[warp][chunk & 3u][lane];
      if (perm)
        tc::cp_async4(dst, perm + L.pos);
      else
        *dst = L.pos;
      L.flags = 1u | (second << 1);
    }
    if (last)
      cnext = true;
    else
      cbase = end;
  };
  // The record index of a walked chunk (its rank copy has completed). Records
  // read through ranks are gathered: they are requested into L2 one chunk
  // before their loads are issued.
  auto take_rank = [&](StreamLane& L, const StreamInfo& I, uint32_t chunk) {
    L.idx = sh.rank[warp][chunk & 3u][lane];
    auto prefetch = [&](const TcSpecies& sp) {
      if (!sp.perm) return;
      const uint32_t n = L.idx;
      prefetch_l2(sp.rx + n); prefetch_l2(sp.ry + n); prefetch_l2(sp.rz + n); prefetch_l2(sp.q + n);
      prefetch_l2(sp.u + n); prefetch_l2(sp.v + n); prefetch_l2(sp.w + n); prefetch_l2(sp.key + n);
    };
    if (L.flags & 1u) {
      if (L.flags & 2u)
        prefetch(tp.sp[1]);
      else
        prefetch(tp.sp[0]);
    }
  };
  // The record of a lane (its species: bit 1 of its flags).
  auto load_rec = [&](const StreamLane& L) {
    StreamRec r{0.0, 0.0, 0.0, 0.0, 0.0f, 0.0f, 0.0f, -1, L.pos, L.flags};
    auto from = [&](const TcSpecies& sp) {
      const uint32_t n = L.idx;
      r.fx = sp.rx[n];
      r.fy = sp.ry[n];
      r.fz = sp.rz[n];
      r.q = sp.q[n];
      r.u = sp.u[n];
      r.v = sp.v[n];
      r.w = sp.w[n];
      r.key = sp.key[n];
    };
    if (L.flags & 1u) {
      if (L.flags & 2u)
        from(tp.sp[1]);
      else
        from(tp.sp[0]);
    }
    return r;
  };
  // Moments of the cells that ended in a chunk whose MMAs have completed;
  // a batch's moments are stored when its last cell (slot 3) is done.
  auto flush = [&](const StreamInfo& I) {
    const uint32_t ended = I.bits & 0xFu;
    if (!((I.bits >> 13) & 1u) || ended == 0u) return;
    const uint32_t nonempty = (I.bits >> 4) & 0xFu;
    float* hs = sh.scratch[warp];
#pragma unroll 1
    for (int s = 0; s < kBatch; ++s) {
      if (!((ended >> s) & 1u)) continue;
      float* st = sh.stage[warp][s];
      if ((nonempty >> s) & 1u) {
        uint32_t g8[8], g4[4];
        tc::tmem_ld8(dq, g8);
        tc::tmem_ld4(dq + 8u, g4);
        tc::tmem_wait_ld();
        const uint32_t z8[8] = {0u, 0u, 0u, 0u, 0u, 0u, 0u, 0u};
        const uint32_t z4[4] = {0u, 0u, 0u, 0u};
        tc::tmem_st8(dq, z8);
        tc::tmem_st4(dq + 8u, z4);
        if (lane < 27) {
#pragma unroll
          for (int e = 0; e < 8; ++e) st[lane * 9 + e] = __uint_as_float(g8[e]);
          st[lane * 9 + 8] = __uint_as_float(g4[0]);
#pragma unroll
          for (int c = 0; c < 3; ++c) hs[lane * 3 + c] = __uint_as_float(g4[1 + c]);
        }
        __syncwarp();
        if (lane < 24) {
          const int a = lane / 3, c = lane - 3 * (lane / 3);
          float sum = 0.0f;
#pragma unroll
          for (int b = 0; b < 8; ++b) sum += hs[monomial_class(a, b) * 3 + c];
          st[kMassMoments + lane] = sum;
        }
        __syncwarp();
      } else {
        for (int q = lane; q < kMoments; q += 32) st[q] = 0.0f;
      }
    }
    if ((ended >> 3) & 1u) {
      __syncwarp();
      bool bad_value = false;
      float* base = mom + (long long)I.bid * kMoments * kBatch;
      for (int q = lane; q < kMoments; q += 32) {
        float4 val = make_float4(sh.stage[warp][0][q], sh.stage[warp][1][q], sh.stage[warp][2][q],
                                 sh.stage[warp][3][q]);
        if (!isfinite(val.x + val.y + val.z + val.w)) {
          bad_value = true;
          val.x = isfinite(val.x) ? val.x : 0.0f;
          val.y = isfinite(val.y) ? val.y : 0.0f;
          val.z = isfinite(val.z) ? val.z : 0.0f;
          val.w = isfinite(val.w) ? val.w : 0.0f;
        }
        float4* dst = reinterpret_cast<float4*>(base + q * kBatch);
        if (accumulate) {
          const float4 old = *dst;
          val.x += old.x; val.y += old.y; val.z += old.z; val.w += old.w;
        }
        *dst = val;
      }
      if (bad_value) atomicAdd(invalid, 1u);
      __syncwarp();
    }
  };

  // Per-warp pipeline: chunk j + 3 walked (ranks copying), j + 2's ranks
  // read (its records requested into L2), j + 1 loaded into registers, j
  // computed.
  StreamLane la, lb, lc;
  StreamInfo ia, ib, ic;
  // One cp.async group per walked chunk (empty when no rank is copied).
  walk(la, ia, 0u);
  tc::cp_async_commit();
  walk(lb, ib, 1u);
  tc::cp_async_commit();
  walk(lc, ic, 2u);
  tc::cp_async_commit();
  tc::cp_async_wait_group<2>();
  take_rank(la, ia, 0u);
  tc::cp_async_wait_group<1>();
  take_rank(lb, ib, 1u);
  StreamRec r1 = load_rec(la);
  StreamInfo i1 = ia;
  StreamInfo ip{0, 0u};  // the previous chunk, whose cells are flushed next
  bool bad = false;
  const int kofs = (lane >> 3) * 128 + (lane & 7) * 16;  // lane's K row in a 512-byte core group
  for (uint32_t j = 0;; ++j) {
    const StreamRec r0 = r1;
    const StreamInfo i0 = i1;
    r1 = load_rec(lb);
    i1 = ib;
    StreamLane ld;
    StreamInfo id;
    walk(ld, id, j + 3u);
    tc::cp_async_commit();
    tc::cp_async_wait_group<1>();
    take_rank(lc, ic, j + 2u);
    lb = lc;
    ib = ic;
    lc = ld;
    ic = id;
    const bool have = (i0.bits >> 13) & 1u;

    // Particle phase: (s alpha, j) and the per-axis factors of one record.
    float bv[12], X[3], YZ[9];
#pragma unroll
    for (int c = 0; c < 12; ++c) bv[c] = 0.0f;
#pragma unroll
    for (int c = 0; c < 3; ++c) X[c] = 0.0f;
#pragma unroll
    for (int c = 0; c < 9; ++c) YZ[c] = 0.0f;
    if (have && (r0.flags & 1u)) {
      const int slot = int(i0.bits >> 16) & 3;
      const TcSpecies& sp = (r0.flags & 2u) ? tp.sp[1] : tp.sp[0];
      if (sp.orx) {
        const uint32_t o = r0.pos;
        sp.orx[o] = r0.fx; sp.ory[o] = r0.fy; sp.orz[o] = r0.fz;
        sp.ou[o] = r0.u; sp.ov[o] = r0.v; sp.ow[o] = r0.w;
        sp.oq[o] = r0.q; sp.okey[o] = r0.key;
      }
      const StreamMeta& m = sh.meta[warp][(i0.bits >> 14) & 3u];
      const double fx = r0.fx, fy = r0.fy, fz = r0.fz;
      bool ok = r0.key == m.bin[slot] && fx >= 0 && fx < 1 && fy >= 0 && fy < 1 && fz >= 0 && fz < 1;
      if (ok) {
        const float x = float(fx), y = float(fy), z = float(fz);
        float b[3];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          const float4 lo4 = *reinterpret_cast<const float4*>(&m.bpoly[slot][8 * c]);
          const float4 hi4 = *reinterpret_cast<const float4*>(&m.bpoly[slot][8 * c + 4]);
          const float t1 = fmaf(z, hi4.w, hi4.x);              // c4 + z c7
          const float t2 = fmaf(z, hi4.y, fmaf(y, t1, lo4.y));  // c1 + y (c4 + z c7) + z c5
          const float t3 = fmaf(z, hi4.z, lo4.z);              // c2 + z c6
          b[c] = fmaf(z, lo4.w, fmaf(y, t3, fmaf(x, t2, lo4.x)));
        }
        const float bo = sp.beta_over_c;
        const ScaledResponse r(b[0], b[1], b[2], bo);
        const float charge = float(r0.q);
        const float hx = r.a[0] * r0.u + r.a[1] * r0.v + r.a[2] * r0.w;
        const float hy = r.a[3] * r0.u + r.a[4] * r0.v + r.a[5] * r0.w;
        const float hz = r.a[6] * r0.u + r.a[7] * r0.v + r.a[8] * r0.w;
        const float qv = charge * tp.inv_volume;
        const float scale = bo * charge;
        bv[9] = qv * hx; bv[10] = qv * hy; bv[11] = qv * hz;
#pragma unroll
        for (int e = 0; e < 9; ++e) bv[e] = r.a[e] * scale;
        ok = isfinite(bv[9] + bv[10] + bv[11] + r.norm_square + scale);
        if (ok) {
          const float cx = 1.0f - x, cy = 1.0f - y, cz = 1.0f - z;
          X[0] = cx * cx; X[1] = x * cx; X[2] = x * x;
          const float Y[3] = {cy * cy, y * cy, y * y};
          const float Z[3] = {cz * cz, z * cz, z * z};
#pragma unroll
          for (int tz = 0; tz < 3; ++tz)
#pragma unroll
            for (int ty = 0; ty < 3; ++ty) YZ[ty + 3 * tz] = Y[ty] * Z[tz];
        } else {
#pragma unroll
          for (int c = 0; c < 12; ++c) bv[c] = 0.0f;
        }
      }
      if (!ok) atomicAdd(invalid, 1u);
    }

    // The MMAs of chunk j - 1 have completed: flush the cells that ended in
    // it; a warp without chunks learns whether any warp of the CTA has one.
    if (j > 0) {
      const bool stall = j == tp.stall_chunk;
      const bool done = tc::mbar_wait(stall ? &sh.never : &sh.mma_bar, stall ? 0u : (j - 1) & 1u, tp.wait_polls);
      if (__any_sync(0xffffffffu, !done)) {
        bad = true;
        break;
      }
      tc::fence_after_sync();
      flush(ip);
      if (!have) {
        // The issuer of chunk j - 1 published whether any warp has chunk j.
        uint32_t d = 0;
        bool seen = false;
        for (uint32_t i = 0; i < tp.wait_polls && !seen; ++i) {
          d = tc::ld_acquire(&sh.decision);
          seen = (d >> 1) == ((j - 1) & 0x7FFFFFFFu);
        }
        if (__any_sync(0xffffffffu, !seen)) {
          bad = true;
          break;
        }
        if (!(d & 1u)) break;
      }
    }
    if (have) {
      // B: the 12 values in columns 16w..16w+11, zeros in 16w+12..16w+15.
      uint32_t bh[6], bl[6];
#pragma unroll
      for (int e = 0; e < 6; ++e) split_pair(make_float2(bv[2 * e], bv[2 * e + 1]), bh[e], bl[e]);
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const uint32_t* w = h ? bl : bh;
        uint8_t* base = sh.b[h] + kofs;
        *reinterpret_cast<uint4*>(base + (2 * warp) * 512) = make_uint4(w[0], w[1], w[2], w[3]);
        *reinterpret_cast<uint4*>(base + (2 * warp + 1) * 512) = make_uint4(w[4], w[5], 0u, 0u);
      }
      // A: the 27 monomials m_t = X[t % 3] YZ[t / 3] of this lane's record.
      uint32_t ah[16], al[16];
#pragma unroll
      for (int i = 0; i < 14; ++i) {
        const int t0 = 2 * i, t1 = 2 * i + 1;
        const float2 f = make_float2(X[t0 % 3], t1 < 27 ? X[t1 % 3] : 0.0f);
        const float2 y = make_float2(YZ[t0 / 3], t1 < 27 ? YZ[t1 / 3] : 0.0f);
        split_pair(__fmul2_rn(f, y), ah[i], al[i]);
      }
      ah[14] = ah[15] = al[14] = al[15] = 0u;
#pragma unroll
      for (int c = 0; c < 4; ++c) {
        const int off = (4 * warp + c) * 512 + kofs;
        *reinterpret_cast<uint4*>(sh.a[0] + off) = make_uint4(ah[4 * c], ah[4 * c + 1], ah[4 * c + 2], ah[4 * c + 3]);
        *reinterpret_cast<uint4*>(sh.a[1] + off) = make_uint4(al[4 * c], al[4 * c + 1], al[4 * c + 2], al[4 * c + 3]);
      }
    }
    if (lane == 0)
      reinterpret_cast<volatile uint8_t*>(&sh.more[j & 1u])[warp] = uint8_t((i1.bits >> 13) & 1u);
    tc::tmem_wait_st();
    tc::fence_proxy_async_smem();
    tc::fence_before_sync();
    __syncwarp();
    // Arrival: the warp whose add completes the chunk's four arrivals issues
    // its MMAs (the counter of parity j & 1 has seen 4 (j >> 1) arrivals of
    // the earlier chunks of that parity).
    if (lane == 0) {
      const uint32_t old = tc::atom_add_acq_rel(&sh.arrived[j & 1u], 1u);
      if (old == 4u * (j >> 1) + 3u) {
        const uint32_t any = *reinterpret_cast<volatile uint32_t*>(&sh.more[j & 1u]) != 0u ? 1u : 0u;
        tc::st_release(&sh.decision, ((j & 0x7FFFFFFFu) << 1) | any);
        tc::fence_after_sync();
        const uint32_t ah = tc::smem_u32(sh.a[0]), al = tc::smem_u32(sh.a[1]);
        const uint32_t bh = tc::smem_u32(sh.b[0]), bl = tc::smem_u32(sh.b[1]);
#pragma unroll
        for (int s = 0; s < 2; ++s) {
          const uint64_t dah = tc::smem_desc(ah + s * 256, 128, 512), dal = tc::smem_desc(al + s * 256, 128, 512);
          const uint64_t dbh = tc::smem_desc(bh + s * 256, 128, 512), dbl = tc::smem_desc(bl + s * 256, 128, 512);
          tc::mma_f16_ss(tmem, dah, dbh, idesc, 1u);
          tc::mma_f16_ss(tmem, dah, dbl, idesc, 1u);
          tc::mma_f16_ss(tmem, dal, dbh, idesc, 1u);
        }
        tc::commit(&sh.mma_bar);
      }
    }
    ip = i0;
  }

  tc::cp_async_wait_all();
  if (bad && lane == 0) atomicAdd(invalid, 1u << 20);
  // Every warp has left the chunk loop, so no chunk is issued after this
  // barrier. The issuer publishes a chunk's index before issuing its MMAs:
  // the last published chunk is the last issued one. After a failed wait its
  // MMAs may still be in flight; one thread waits for them (with the default
  // bound, whatever tp.wait_polls is) before the tensor memory is freed. On
  // the normal path that chunk has completed and the wait returns at once.
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  if (threadIdx.x == 0) {
    const uint32_t d = tc::ld_acquire(&sh.decision);
    if (d != 0xFFFFFFFEu) tc::mbar_wait(&sh.mma_bar, (d >> 1) & 1u);
  }
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  if (warp == 0) tc::tmem_dealloc(tmem, kStreamTmemCols);
}

}  // namespace

long long moment_stride(const Geom& g) {
  const long long cells = (long long)g.nx * g.ny * g.nz;
  return (cells + kCells - 1) / kCells * kCells;
}
size_t moment_floats(const Geom& g) { return size_t(kMoments) * size_t(moment_stride(g)); }

cudaError_t launch_deposit_tc(int mass_kind, const Geom& g, int ns, const double* qom, double dt, double c,
                              const tpicb200_particles* const* p, const uint32_t* const* counts,
                              const uint32_t* const* offsets, const void* bnode, float* moments, int accumulate,
                              uint32_t* invalid, const SortedCopy* const* copies, cudaStream_t s,
                              uint32_t wait_polls, uint32_t stall_chunk) {
  if (mass_kind != TPICB200_MASS_TF32 && mass_kind != TPICB200_MASS_BF16X3) return cudaErrorNotSupported;
  if (!moments || ns < 1) return cudaErrorInvalidValue;
  int device = 0, sms = 148;
  cudaGetDevice(&device);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  const long long cells = (long long)g.nx * g.ny * g.nz;
  if (cells > (1LL << 31) - 64) return cudaErrorInvalidValue;
  const long long groups = (cells + kCells - 1) / kCells;
  const bool tf32 = mass_kind == TPICB200_MASS_TF32;
  cudaError_t e = cudaSuccess;
  // TF32: one CTA group of four cells at a time. Dynamic shared-memory
  // padding brings each CTA to ~47 KB, so at most four CTAs (4 x 128
  // tensor-memory columns = all 512) are resident per SM and no
  // tcgen05.alloc ever waits for another CTA's columns; the maximum
  // shared-memory carveout lets all four be resident.
  // BF16x3: the stream kernel, ~53 KB of dynamic shared memory per CTA (four
  // resident per SM, 128 tensor-memory columns each).
  auto kernel = tc_deposit_kernel<false>;
  const int pad = 47 * 1024 - int(sizeof(TcShared<false>));
  unsigned blocks = unsigned(std::min<long long>(groups, (long long)kCtasPerSm * sms));
  const int stream_bytes = int(sizeof(StreamShared));
  if (tf32) {
    e = cudaFuncSetAttribute(kernel, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
  } else {
    blocks = unsigned(std::min<long long>((groups + kCells - 1) / kCells, (long long)kCtasPerSm * sms));
    e = cudaFuncSetAttribute(tc_stream_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, stream_bytes);
    if (e == cudaSuccess)
      e = cudaFuncSetAttribute(tc_stream_kernel, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
  }
  if (e != cudaSuccess) return e;
  for (int first = 0; first < ns; first += kFuse) {
    TcParams tp{};
    tp.ns = std::min(kFuse, ns - first);
    tp.inv_volume = float(g.inv_volume);
    tp.wait_polls = wait_polls ? wait_polls : kDefaultWaitPolls;
    tp.stall_chunk = stall_chunk;
    for (int i = 0; i < tp.ns; ++i) {
      const tpicb200_particles* sp = p[first + i];
      const SortedCopy* cp = copies ? copies[first + i] : nullptr;
      const bool copy = cp && cp->perm && cp->out.rx;
      tp.sp[i] = TcSpecies{(const double*)sp->rx, (const double*)sp->ry, (const double*)sp->rz,
                           (const float*)sp->u, (const float*)sp->v, (const float*)sp->w, sp->q, sp->cell,
                           counts[first + i], offsets[first + i], float(qom[first + i] * dt / 2 / c),
                           cp ? cp->perm : nullptr, copy ? (double*)cp->out.rx : nullptr,
                           copy ? (double*)cp->out.ry : nullptr, copy ? (double*)cp->out.rz : nullptr,
                           copy ? (float*)cp->out.u : nullptr, copy ? (float*)cp->out.v : nullptr,
                           copy ? (float*)cp->out.w : nullptr, copy ? cp->out.q : nullptr,
                           copy ? cp->out.cell : nullptr};
    }
    const int acc = (accumulate || first > 0) ? 1 : 0;
    if (tf32)
      kernel<<<blocks, 128, pad, s>>>(g, tp, (const float*)bnode, moments, acc, invalid);
    else
      tc_stream_kernel<<<blocks, 128, stream_bytes, s>>>(g, tp, (const float*)bnode, moments, acc,
                                                         invalid, int(groups));
    count_launches(1);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
  }
  return cudaSuccess;
}

namespace {

// For every stencil: the corners a whose pair (a, a + offset) lies in one
// cell, and that pair's monomial class t.
struct StencilPairs {
  int count[14];
  int corner[14][8];
  int monomial[14][8];
};
__host__ __device__ constexpr StencilPairs make_stencil_pairs() {
  StencilPairs r{};
  for (int s = 0; s < 14; ++s)
    for (int a = 0; a < 8; ++a) {
      const int bx = (a & 1) + stencil_offset(s, 0), by = ((a >> 1) & 1) + stencil_offset(s, 1),
                bz = ((a >> 2) & 1) + stencil_offset(s, 2);
      if (bx < 0 || bx > 1 || by < 0 || by > 1 || bz < 0 || bz > 1) continue;
      const int t = ((a & 1) + bx) + 3 * (((a >> 1) & 1) + by) + 9 * (((a >> 2) & 1) + bz);
      r.corner[s][r.count[s]] = a;
      r.monomial[s][r.count[s]] = t;
      ++r.count[s];
    }
  return r;
}

// One thread per (unique node, stencil): the stencil's nine record entries
// of the node, each the sum, in increasing corner order, of the moments
// G[t][e] of the cells holding the pairs (a, a + offset_s); "stencil" 14 is
// the current, whose component c is the sum of the eight corner sums
// J[a][c] of the cells around the node. The stencil is the block index
// modulo 15 and each case is unrolled from the compile-time tables, so a thread holds
// at most nine sums and the loads of a warp are consecutive across its
// nodes. `overwrite` stores the sums (J and M were cleared and nothing else
// was deposited); otherwise they are added.
template <class T, int S>
__device__ __forceinline__ void assemble_stencil(const Geom& g, const long long (&cell)[8], long long node,
                                                 long long mvertex, const T* __restrict__ mom,
                                                 T* __restrict__ J, T* __restrict__ M, int overwrite) {
  constexpr StencilPairs pairs = make_stencil_pairs();
  if constexpr (S < 14) {
    T sum[9];
#pragma unroll
    for (int e = 0; e < 9; ++e) sum[e] = T(0);
#pragma unroll
    for (int p = 0; p < 8; ++p) {
      if (p < pairs.count[S]) {
#pragma unroll
        for (int e = 0; e < 9; ++e)
          sum[e] += __ldg(mom + moment_index(cell[pairs.corner[S][p]], pairs.monomial[S][p] * 9 + e));
      }
    }
#pragma unroll
    for (int e = 0; e < 9; ++e) {
      T* dst = M + g.mass_index(mvertex, S * 9 + e);
      *dst = overwrite ? sum[e] : *dst + sum[e];
    }
  } else {
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      T sum = T(0);
#pragma unroll
      for (int a = 0; a < 8; ++a) sum += __ldg(mom + moment_index(cell[a], kMassMoments + a * 3 + c));
      T* dst = J + c * g.nodes + node;
      *dst = overwrite ? sum : *dst + sum;
    }
  }
}

template <class T>
__global__ void __launch_bounds__(128) assemble_moments_kernel(Geom g, const T* __restrict__ mom,
                                                               T* __restrict__ J, T* __restrict__ M,
                                                               int overwrite) {
  const int nx = g.nx, ny = g.ny;
  const long long unique = (long long)nx * ny * g.nz;
  // The stencil is the fast block index (see assemble_warp_quads_kernel).
  const int stencil = int(blockIdx.x % 15);
  const long long v = (blockIdx.x / 15) * (long long)blockDim.x + threadIdx.x;
  if (v >= unique) return;
  const int i = int(v % nx);
  const long long r = v / nx;
  const int j = int(r % ny), k = int(r / ny);
  // Cells of corner a: the node is corner a of cell (i - a_x, j - a_y, k - a_z).
  const int i1 = i > 0 ? i - 1 : nx - 1, j1 = j > 0 ? j - 1 : ny - 1, k1 = k > 0 ? k - 1 : g.nz - 1;
  long long cell[8];
#pragma unroll
  for (int a = 0; a < 8; ++a)
    cell[a] = ((a & 1) ? i1 : i) + (long long)nx * (((a & 2) ? j1 : j) + (long long)ny * ((a & 4) ? k1 : k));
  const long long node = g.node(i, j, k), mvertex = g.mass_vertex(i, j, k);
  switch (stencil) {
    case 0: assemble_stencil<T, 0>(g, cell, node, mvertex, mom, J, M, overwrite); break;
    case 1: assemble_stencil<T, 1>(g, cell, node, mvertex, mom, J, M, overwrite); break;
    case 2: assemble_stencil<T, 2>(g, cell, node, mvertex, mom, J, M, overwrite); break;
    case 3: assemble_stencil<T, 3>(g, cell, node, mvertex, mom, J, M, overwrite); break;
    case 4: assemble_stencil<T, 4>(g, cell, node, mvertex, mom, J, M, overwrite); break;
    case 5: assemble_stencil<T, 5>(g, cell, node, mvertex, mom, J, M, overwrite); break;
    case 6: assemble_stencil<T, 6>(g, cell, node, mvertex, mom, J, M, overwrite); break;
    case 7: assemble_stencil<T, 7>(g, cell, node, mvertex, mom, J, M, overwrite); break;
    case 8: assemble_stencil<T, 8>(g, cell, node, mvertex, mom, J, M, overwrite); break;
    case 9: assemble_stencil<T, 9>(g, cell, node, mvertex, mom, J, M, overwrite); break;
    case 10: assemble_stencil<T, 10>(g, cell, node, mvertex, mom, J, M, overwrite); break;
    case 11: assemble_stencil<T, 11>(g, cell, node, mvertex, mom, J, M, overwrite); break;
    case 12: assemble_stencil<T, 12>(g, cell, node, mvertex, mom, J, M, overwrite); break;
    case 13: assemble_stencil<T, 13>(g, cell, node, mvertex, mom, J, M, overwrite); break;
    default: assemble_stencil<T, 14>(g, cell, node, mvertex, mom, J, M, overwrite); break;
  }
}

// Rows of a multiple of four cells: one thread per (four consecutive nodes
// 4m .. 4m + 3 of an x-row, stencil), so that every 16-byte word of a
// four-cell record serves four nodes at once. Corner a_x = 0 reads the
// nodes' own group of cells (4m .. 4m + 3); corner a_x = 1 reads cells
// 4m - 1 .. 4m + 2: the last cell of the previous group (periodic in x), then
// the first three of the own group. Sums in increasing corner order, as the
// per-node kernel.
// The 16-byte (float) or two 16-byte (double) words of one moment entry of a
// group of four cells.
__device__ __forceinline__ void load_quad(const float* p, float (&v)[4]) {
  const float4 x = __ldg(reinterpret_cast<const float4*>(p));
  v[0] = x.x; v[1] = x.y; v[2] = x.z; v[3] = x.w;
}
__device__ __forceinline__ void load_quad(const double* p, double (&v)[4]) {
  const double2 x = __ldg(reinterpret_cast<const double2*>(p)), y = __ldg(reinterpret_cast<const double2*>(p) + 1);
  v[0] = x.x; v[1] = x.y; v[2] = y.x; v[3] = y.y;
}

// The moment assembly when nx is a multiple of 4: a warp takes eight consecutive
// quads (32 nodes) of one node row and one stencil; lane l works on quad
// l / 4 and on the entries e = l % 4, l % 4 + 4 (and 8 for l % 4 = 0), so
// the four lanes of a quad read four consecutive 16-byte moment words and a
// warp's load touches eight 64-byte runs instead of 32 scattered words.
// Every (node, entry) sum adds the pairs' moments in increasing corner
// order, the quad's lower neighbour group supplying the corner-1 cells of
// its first node. The sums are staged in
// shared memory and stored by node (32 consecutive nodes per entry).
template <class T, int S>
__device__ __forceinline__ void assemble_warp_quads(const Geom& g, int m0, int j, int k, const T* __restrict__ mom,
                                                    T* __restrict__ J, T* __restrict__ M, int overwrite,
                                                    T (*stage)[32]) {
  constexpr StencilPairs pairs = make_stencil_pairs();
  constexpr int kEntries = S < 14 ? 9 : 3;
  const int lane = threadIdx.x & 31, sub = lane & 3;
  const int ny = g.ny, nz = g.nz, qx = g.nx >> 2;
  const int m = m0 + (lane >> 2);
  const bool live = m < qx;
  const int j1 = j > 0 ? j - 1 : ny - 1, k1 = k > 0 ? k - 1 : nz - 1;
  const int mp = m > 0 ? m - 1 : qx - 1;
  T sum[3][4];
#pragma unroll
  for (int r = 0; r < 3; ++r)
#pragma unroll
    for (int n = 0; n < 4; ++n) sum[r][n] = T(0);
  if (live) {
#pragma unroll
    for (int a = 0; a < 8; ++a) {
      const long long row = (long long)((a & 2) ? j1 : j) + (long long)ny * ((a & 4) ? k1 : k);
      const long long own = row * qx + m, prev = row * qx + mp;
      auto add = [&](int q, int r) {
        T v[4];
        load_quad(mom + (own * kMoments + q) * 4, v);
        if (a & 1) {
          const T p3 = __ldg(mom + (prev * kMoments + q) * 4 + 3);
          sum[r][0] += p3; sum[r][1] += v[0]; sum[r][2] += v[1]; sum[r][3] += v[2];
        } else {
          sum[r][0] += v[0]; sum[r][1] += v[1]; sum[r][2] += v[2]; sum[r][3] += v[3];
        }
      };
#pragma unroll
      for (int r = 0; r < 3; ++r) {
        const int e = sub + 4 * r;
        if (e >= kEntries) continue;
        if constexpr (S < 14) {
#pragma unroll
          for (int pp = 0; pp < 8; ++pp)
            if (pp < pairs.count[S] && pairs.corner[S][pp] == a) add(pairs.monomial[S][pp] * 9 + e, r);
        } else {
          add(kMassMoments + a * 3 + e, r);
        }
      }
    }
  }
#pragma unroll
  for (int r = 0; r < 3; ++r) {
    const int e = sub + 4 * r;
    if (e < kEntries)
#pragma unroll
      for (int n = 0; n < 4; ++n) stage[e][4 * (lane >> 2) + n] = sum[r][n];
  }
  __syncwarp();
  const int i = 4 * m0 + lane;
  if (i < g.nx) {
    const long long node = g.node(i, j, k);
#pragma unroll
    for (int e = 0; e < kEntries; ++e) {
      T* dst = S < 14 ? M + g.mass_index(g.mass_vertex(i, j, k), S * 9 + e) : J + e * g.nodes + node;
      *dst = overwrite ? stage[e][lane] : *dst + stage[e][lane];
    }
  }
}

template <class T>
__global__ void __launch_bounds__(128) assemble_warp_quads_kernel(Geom g, const T* __restrict__ mom,
                                                                  T* __restrict__ J, T* __restrict__ M,
                                                                  int overwrite) {
  __shared__ T stage[4][9][32];
  const int warp = threadIdx.x >> 5;
  const int qx = g.nx >> 2, tiles = (qx + 7) / 8;
  const long long rows = (long long)g.ny * g.nz;
  // The stencil is the fast block index, so that the 15 blocks of the same
  // nodes run together and share the cell moments in L2.
  const int stencil = int(blockIdx.x % 15);
  const long long t = (blockIdx.x / 15) * 4LL + warp;
  if (t >= rows * tiles) return;
  const long long row = t / tiles;
  const int m0 = int(t - row * tiles) * 8;
  const int j = int(row % g.ny), k = int(row / g.ny);
  T (*st)[32] = stage[warp];
  switch (stencil) {
    case 0: assemble_warp_quads<T, 0>(g, m0, j, k, mom, J, M, overwrite, st); break;
    case 1: assemble_warp_quads<T, 1>(g, m0, j, k, mom, J, M, overwrite, st); break;
    case 2: assemble_warp_quads<T, 2>(g, m0, j, k, mom, J, M, overwrite, st); break;
    case 3: assemble_warp_quads<T, 3>(g, m0, j, k, mom, J, M, overwrite, st); break;
    case 4: assemble_warp_quads<T, 4>(g, m0, j, k, mom, J, M, overwrite, st); break;
    case 5: assemble_warp_quads<T, 5>(g, m0, j, k, mom, J, M, overwrite, st); break;
    case 6: assemble_warp_quads<T, 6>(g, m0, j, k, mom, J, M, overwrite, st); break;
    case 7: assemble_warp_quads<T, 7>(g, m0, j, k, mom, J, M, overwrite, st); break;
    case 8: assemble_warp_quads<T, 8>(g, m0, j, k, mom, J, M, overwrite, st); break;
    case 9: assemble_warp_quads<T, 9>(g, m0, j, k, mom, J, M, overwrite, st); break;
    case 10: assemble_warp_quads<T, 10>(g, m0, j, k, mom, J, M, overwrite, st); break;
    case 11: assemble_warp_quads<T, 11>(g, m0, j, k, mom, J, M, overwrite, st); break;
    case 12: assemble_warp_quads<T, 12>(g, m0, j, k, mom, J, M, overwrite, st); break;
    case 13: assemble_warp_quads<T, 13>(g, m0, j, k, mom, J, M, overwrite, st); break;
    default: assemble_warp_quads<T, 14>(g, m0, j, k, mom, J, M, overwrite, st); break;
  }
}



// ---------------------------------------------------------------------------
// FP64 form of the moment deposition (double precision).
//
// The same per-cell moments as the tensor-core forms, G[t][e] = sum_p m_pt
// (s_p alpha_p[e]) and H[t][c] = sum_p m_pt j_p[c], accumulated in FP64: a
// warp per cell; per chunk of 32 records each lane forms one record's B
// gather, response, s alpha and j (12 values) and its 27 pair-weight products
// m_t = (X_tx Y_ty) Z_tz into shared memory; then the warp contracts the
// chunk on the FP64 tensor cores (mma.sync m8n8k4: D[t][e] += sum_k m[k][t]
// src[k][e], t in four tiles of 8 rows (27 used), e in two of 8 columns (12
// used), four records per step). The contraction on the CUDA cores (a 3 x 4
// register block per lane, 7 shared loads per 12 fused multiply-adds) was
// bound by the shared-memory pipe (93 % of its wavefronts at 64^3); the
// fragments need 6 shared loads per 4 records and lane (128^3-cell workload:
// the FP64 deposit stage 20.0 -> 16.1 ms). The flush stores G and the corner
// currents J_a[c] = sum_b H[t(a,b)][c] into the double moment records, which
// the assembly adds into J and the mass records as for the tensor-core forms.
// Per record this is 27 x 12 multiply-adds, where the reference's scalar and
// matrix-core kernels form the 64 corner-pair products of 9 entries
// (mass_matrix_scalar_device.hpp:25-97, mass_matrix_mma_device.hpp:58-150).
struct F64Species {
  const double* rx;
  const double* ry;
  const double* rz;
  const double* u;
  const double* v;
  const double* w;
  const double* q;
  const int32_t* key;
  const uint32_t* counts;
  const uint32_t* offsets;
  double beta_over_c;
  const uint32_t* perm;  // sorted position -> record (null: records in sorted order)
  double* orx;           // sorted copy (null: none)
  double* ory;
  double* orz;
  double* ou;
  double* ov;
  double* ow;
  double* oq;
  int32_t* okey;
};

struct F64Params {
  F64Species sp[kFuse];
  int ns;
  double inv_volume;
};

// D (8 x 8) += A (8 x 4) B (4 x 8) in FP64 on the tensor cores. Per lane:
// A[lane >> 2][lane & 3], B[lane & 3][lane >> 2], D[lane >> 2][2 (lane & 3) + i].
__device__ __forceinline__ void dmma_884(double (&d)[2], double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
               : "+d"(d[0]), "+d"(d[1])
               : "d"(a), "d"(b));
}

constexpr int kF64Warps = 4;
// The products and values are stored by (t or entry, record), 36 records a
// row: a lane's stores of its record fall in consecutive words, and the 16
// lanes of a half-warp fragment load (4 rows x 4 records) hit 16 different
// bank pairs. With record-major rows of 29 and 13 words the fragment loads
// met 2-way conflicts (C3 FP64 deposit stage 16.2 ms, 15.7 ms with these rows).
constexpr int kF64Pitch = 36;
struct F64Warp {
  double bc[24];                 // B at the cell's corners, [c][a]
  double m[27][kF64Pitch];       // [t][record]: the 27 pair-weight products
  double src[12][kF64Pitch];     // [entry][record]: s alpha[9], j[3]
  double hs[27][3];              // H of the cell at the flush
};

__global__ void __launch_bounds__(kF64Warps * 32) moments_f64_kernel(Geom g, F64Params fp,
                                                                     const double* __restrict__ bnode,
                                                                     double* __restrict__ mom, int accumulate,
                                                                     uint32_t* invalid) {
  __shared__ F64Warp shared[kF64Warps];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  F64Warp& S = shared[warp];
  const int nx = g.nx, ny = g.ny;
  const long long cells = (long long)nx * ny * g.nz, nn = g.nodes;
  const int kk = lane & 3, rr = lane >> 2;  // fragment coordinates
  uint32_t bad = 0;
  for (long long cell = (long long)blockIdx.x * kF64Warps + warp; cell < cells;
       cell += (long long)gridDim.x * kF64Warps) {
    const int ci = int(cell % nx), cj = int((cell / nx) % ny), ck = int(cell / ((long long)nx * ny));
    const int32_t key = g.encode(ci, cj, ck);
    if (lane < 24) {
      const int c = lane >> 3, a = lane & 7;
      S.bc[lane] = bnode[c * nn + g.node(ci + (a & 1), cj + ((a >> 1) & 1), ck + ((a >> 2) & 1))];
    }
    __syncwarp();
    // D tiles (t: 4 x 8 rows, entry: 2 x 8 columns) of this lane.
    double acc[4][2][2];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int e = 0; e < 2; ++e) acc[i][e][0] = acc[i][e][1] = 0.0;
    for (int si = 0; si < fp.ns; ++si) {
      const F64Species& sp = fp.sp[si];
      const uint32_t begin = sp.offsets[key], n = sp.counts[key];
      for (uint32_t c0 = 0; c0 < n; c0 += 32) {
        const uint32_t m = n - c0 < 32u ? n - c0 : 32u;
        if (lane < int(m)) {
          const uint32_t pos = begin + c0 + lane;
          const uint32_t r = sp.perm ? sp.perm[pos] : pos;
          const double fx = sp.rx[r], fy = sp.ry[r], fz = sp.rz[r];
          const double u = sp.u[r], v = sp.v[r], w = sp.w[r], q = sp.q[r];
          const int32_t k0 = sp.key[r];
          if (sp.orx) {
            sp.orx[pos] = fx; sp.ory[pos] = fy; sp.orz[pos] = fz;
            sp.ou[pos] = u; sp.ov[pos] = v; sp.ow[pos] = w; sp.oq[pos] = q; sp.okey[pos] = k0;
          }
          bool ok = k0 == key && fx >= 0 && fx < 1 && fy >= 0 && fy < 1 && fz >= 0 && fz < 1;
          if (ok) {
            double wt[8];
            cic_weights<double>(fx, fy, fz, wt);
            double b[3];
#pragma unroll
            for (int c = 0; c < 3; ++c) {
              double val = 0;
#pragma unroll
              for (int a = 0; a < 8; ++a) val += wt[a] * S.bc[c * 8 + a];
              b[c] = val;
            }
            const Response<double> resp(b[0], b[1], b[2], sp.beta_over_c);
            const double scale = sp.beta_over_c * q;
            double hx, hy, hz;
            resp.apply(u, v, w, hx, hy, hz);
            const double qv = q * fp.inv_volume;
            double sv[12];
#pragma unroll
            for (int e = 0; e < 9; ++e) sv[e] = resp.a[e] * scale;
            sv[9] = qv * hx; sv[10] = qv * hy; sv[11] = qv * hz;
#pragma unroll
            for (int e = 0; e < 12; ++e) {
              ok = ok && isfinite(sv[e]);
              S.src[e][lane] = sv[e];
            }
            const double cx = 1.0 - fx, cy = 1.0 - fy, cz = 1.0 - fz;
            const double px[3] = {cx * cx, cx * fx, fx * fx};
            const double py[3] = {cy * cy, cy * fy, fy * fy};
            const double pz[3] = {cz * cz, cz * fz, fz * fz};
#pragma unroll
            for (int ty = 0; ty < 3; ++ty)
#pragma unroll
              for (int tx = 0; tx < 3; ++tx) {
                const double pxy = px[tx] * py[ty];
#pragma unroll
                for (int tz = 0; tz < 3; ++tz) S.m[tx + 3 * ty + 9 * tz][lane] = pxy * pz[tz];
              }
          }
          if (!ok) {
            ++bad;
#pragma unroll
            for (int e = 0; e < 12; ++e) S.src[e][lane] = 0.0;
#pragma unroll
            for (int t = 0; t < 27; ++t) S.m[t][lane] = 0.0;
          }
        }
        __syncwarp();
        for (uint32_t k0 = 0; k0 < m; k0 += 4) {
          const uint32_t k = k0 + kk;
          const bool in = k < m;
          double av[4], bv[2];
#pragma unroll
          for (int i = 0; i < 4; ++i) av[i] = in && 8 * i + rr < 27 ? S.m[8 * i + rr][k] : 0.0;
#pragma unroll
          for (int e = 0; e < 2; ++e) bv[e] = in && 8 * e + rr < 12 ? S.src[8 * e + rr][k] : 0.0;
#pragma unroll
          for (int i = 0; i < 4; ++i)
#pragma unroll
            for (int e = 0; e < 2; ++e) dmma_884(acc[i][e], av[i], bv[e]);
        }
        __syncwarp();
      }
    }
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int e = 0; e < 2; ++e)
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const int t = 8 * i + rr, entry = 8 * e + 2 * kk + h;
          if (t >= 27 || entry >= 12) continue;
          if (entry < 9) {
            double* dst = mom + moment_index(cell, t * 9 + entry);
            *dst = accumulate ? *dst + acc[i][e][h] : acc[i][e][h];
          } else {
            S.hs[t][entry - 9] = acc[i][e][h];
          }
        }
    __syncwarp();
    if (lane < 24) {
      const int a = lane / 3, c = lane % 3;
      double sum = 0.0;
#pragma unroll
      for (int b = 0; b < 8; ++b) sum += S.hs[monomial_class(a, b)][c];
      double* dst = mom + moment_index(cell, kMassMoments + a * 3 + c);
      *dst = accumulate ? *dst + sum : sum;
    }
    __syncwarp();
  }
  bad = warp_sum(bad);
  if (bad && lane == 0) atomicAdd(invalid, bad);
}

}  // namespace

cudaError_t launch_assemble_moments(int precision, const Geom& g, const void* moments, void* j, void* mass,
                                    int overwrite, cudaStream_t s) {
  const long long unique = (long long)g.nx * g.ny * g.nz;
  // nx a multiple of 4: warps of eight quads (4 warps a block); otherwise one
  // node per thread.
  const long long warp_tiles = (long long)g.ny * g.nz * (((g.nx >> 2) + 7) / 8);
  const long long items = g.nx % 4 == 0 ? warp_tiles * 32 : unique;
  const long long blocks = (items + 127) / 128 * 15;
  if (blocks > 0x7FFFFFFFLL) return cudaErrorInvalidValue;
  if (precision == TPICB200_PRECISION_DOUBLE) {
    if (g.nx % 4 == 0)
      assemble_warp_quads_kernel<double><<<unsigned(blocks), 128, 0, s>>>(g, (const double*)moments, (double*)j,
                                                                         (double*)mass, overwrite);
    else
      assemble_moments_kernel<double><<<unsigned(blocks), 128, 0, s>>>(g, (const double*)moments, (double*)j,
                                                                      (double*)mass, overwrite);
  } else if (g.nx % 4 == 0) {
    assemble_warp_quads_kernel<float><<<unsigned(blocks), 128, 0, s>>>(g, (const float*)moments, (float*)j,
                                                                      (float*)mass, overwrite);
  } else {
    assemble_moments_kernel<float><<<unsigned(blocks), 128, 0, s>>>(g, (const float*)moments, (float*)j,
                                                                   (float*)mass, overwrite);
  }
  count_launches(1);
  return cudaGetLastError();
}

cudaError_t launch_deposit_moments_f64(const Geom& g, int ns, const double* qom, double dt, double c,
                                       const tpicb200_particles* const* p, const uint32_t* const* counts,
                                       const uint32_t* const* offsets, const void* bnode, double* moments,
                                       int accumulate, uint32_t* invalid, const SortedCopy* const* copies,
                                       cudaStream_t s) {
  if (!moments || ns < 1) return cudaErrorInvalidValue;
  const long long cells = (long long)g.nx * g.ny * g.nz;
  const unsigned blocks = unsigned(std::min<long long>((cells + kF64Warps - 1) / kF64Warps, 148LL * 16));
  for (int first = 0; first < ns; first += kFuse) {
    F64Params fp{};
    fp.ns = std::min(kFuse, ns - first);
    fp.inv_volume = g.inv_volume;
    for (int i = 0; i < fp.ns; ++i) {
      const tpicb200_particles* sp = p[first + i];
      const SortedCopy* cp = copies ? copies[first + i] : nullptr;
      const bool copy = cp && cp->perm && cp->out.rx;
      fp.sp[i] = F64Species{(const double*)sp->rx, (const double*)sp->ry, (const double*)sp->rz,
                            (const double*)sp->u, (const double*)sp->v, (const double*)sp->w, sp->q, sp->cell,
                            counts[first + i], offsets[first + i], qom[first + i] * dt / 2 / c,
                            cp ? cp->perm : nullptr, copy ? (double*)cp->out.rx : nullptr,
                            copy ? (double*)cp->out.ry : nullptr, copy ? (double*)cp->out.rz : nullptr,
                            copy ? (double*)cp->out.u : nullptr, copy ? (double*)cp->out.v : nullptr,
                            copy ? (double*)cp->out.w : nullptr, copy ? cp->out.q : nullptr,
                            copy ? cp->out.cell : nullptr};
    }
    moments_f64_kernel<<<blocks, kF64Warps * 32, 0, s>>>(g, fp, (const double*)bnode, moments,
                                                        (accumulate || first > 0) ? 1 : 0, invalid);
    count_launches(1);
    if (cudaError_t e = cudaGetLastError()) return e;
  }
  return cudaSuccess;
}

}  // namespace tpicb200
