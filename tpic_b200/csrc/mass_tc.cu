// Tensor-core (tcgen05) mass-matrix assembly with the implicit current on
// CUDA cores, one species of sorted records per launch.
//
// The mass block of a corner pair is K_ab = sum_p s_p alpha_p W_pa W_pb with
// s = (beta/c) q (ecsim/mass_matrix/mass_matrix_scalar_device.hpp:25-97). With
// CIC weights W_pa = X_p(a_x) Y_p(a_y) Z_p(a_z), the pair weight factors per
// axis into one of three products, (1-x)^2, x(1-x) or x^2, so W_pa W_pb is the
// monomial m_pt of the per-axis class t = (a_x+b_x) + 3(a_y+b_y) + 9(a_z+b_z).
// A cell's 36 canonical pair blocks are therefore 27 monomial moments
//   G[t][c] = sum_p m_pt (s_p alpha_p[c]),  t < 27, c < 9,
// a dense contraction over the cell's particles: D = A^T B with K = particles.
//
// Tensor-core mapping (one CTA of four warps works on four cells at once):
//   A (tensor memory, M = 128 lanes x K columns): lane 32w + t holds m_pt of
//     cell w's particles (rows 27..31 of each quadrant are zero);
//   B (shared memory, K x N, no swizzle): columns 12w..12w+8 (TF32, N = 48,
//     K-major core matrices of 8 N-rows x 4 K-values) or 16w..16w+8 (BF16,
//     N = 64, MN-major core matrices of 8 K-rows x 8 N-values) hold
//     s_p alpha_p of cell w's particle p (the rest zero);
//   D (tensor memory, 128 x 48 FP32): D[32w + t][12w + c] = G_w[t][c]; the
//     off-diagonal blocks are never read.
// Each 32-particle chunk is four tcgen05.mma.kind::tf32 (K = 8) issued by one
// thread; A and B are double-buffered so the next chunk is produced while the
// tensor core consumes the previous one (tcgen05.commit -> mbarrier).
// Operands are rounded to TF32 with round-to-nearest (cvt.rna) so the
// rounding is unbiased; accumulation is FP32. The epilogue reads G with
// tcgen05.ld and stores it, with the cell's 8x3 current corner sums, as the
// cell's moments (27x9 + 8x3 values, entry-major arrays over the unique
// cells; a later species adds to them in place). No atomics: the reference's
// flush issues up to 324 atomics per cell (mass_matrix_mma_device.hpp:141-150).
// assemble_moments_kernel then forms every record entry of a unique node as
// the sum of the 1, 2, 4 or 8 cell moments that share it, in a fixed order.
// J-hat is accumulated in FP32 on the CUDA cores exactly as the scalar form.
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
constexpr int kFacStride = 36;     // floats per factor row (padded against bank conflicts)
constexpr uint32_t kTmemCols = 128;
constexpr int kMassMoments = 27 * 9;                  // G[t][c] per cell
constexpr int kMoments = kMassMoments + 24;           // + J corner sums [a][c]
constexpr uint32_t kDcol = 64;
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

// Canonical pairs sharing each monomial class: corner a and stencil s.
struct MonomialPairs {
  int count[27];
  int corner[27][4];
  int stencil[27][4];
};
constexpr MonomialPairs make_monomial_pairs() {
  MonomialPairs r{};
  for (int a = 0; a < 8; ++a)
    for (int b = 0; b < 8; ++b) {
      const int s = pair_stencil(a, b);
      if (s < 0) continue;
      const int t = ((a & 1) + (b & 1)) + 3 * (((a >> 1) & 1) + ((b >> 1) & 1)) + 9 * (((a >> 2) & 1) + ((b >> 2) & 1));
      r.corner[t][r.count[t]] = a;
      r.stencil[t][r.count[t]] = s;
      ++r.count[t];
    }
  return r;
}
__constant__ MonomialPairs c_pairs = make_monomial_pairs();

struct TcParams {
  float beta_over_c;
  float inv_volume;
};

template <bool Bf16> struct __align__(128) TcShared {
  uint8_t btile[2][Form<Bf16>::tiles][Form<Bf16>::tile_bytes];
  float fac[kCells][12][kFacStride];
  float bcache[kCells][24];
  float stage[kMoments][kCells];
  uint64_t mbar[2];
  uint32_t tmem_base;
  uint32_t count[kCells];
};

__device__ __forceinline__ uint32_t pack_bf16(float lo_elem, float hi_elem) {
  const __nv_bfloat162 v = __floats2bfloat162_rn(lo_elem, hi_elem);  // .x (low half) = first element
  return *reinterpret_cast<const uint32_t*>(&v);
}
__device__ __forceinline__ void split_bf16(float v, float& hi, float& lo) {
  hi = __bfloat162float(__float2bfloat16_rn(v));
  lo = v - hi;
}

template <bool Bf16>
__global__ void __launch_bounds__(128, 1) tc_deposit_kernel(Geom g, TcParams tp,
    const double* __restrict__ rx, const double* __restrict__ ry, const double* __restrict__ rz,
    const float* __restrict__ u, const float* __restrict__ v, const float* __restrict__ w,
    const double* __restrict__ q, const int32_t* __restrict__ key, const uint32_t* __restrict__ counts,
    const uint32_t* __restrict__ offsets, const float* __restrict__ bnode, float* __restrict__ mom,
    long long mom_stride, int accumulate, uint32_t* invalid) {
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
    tc::fence_mbar_init();
  }
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tmem = sh.tmem_base;
  const uint32_t lane_base = uint32_t(32 * warp) << 16;
  constexpr uint32_t idesc = tc::instr_desc(Bf16 ? 1u : 2u, 128, kN, Bf16 ? 1u : 0u);
  uint32_t phase[2] = {0, 0};
  bool pending[2] = {false, false};
  int buf = 0;
  bool failed = false;

  const long long cells = (long long)g.nx * g.ny * g.nz;
  const long long groups = (cells + kCells - 1) / kCells;
  // Monomial row of this thread in its warp's quadrant.
  const int t_row = lane;
  const int tx = t_row % 3, tyz = t_row / 3;

  // Software pipeline: the metadata and B corners of the next group and the
  // records of the next chunk (possibly the next group's first) are loaded
  // while the current chunk is produced and consumed.
  struct Meta {
    int ci, cj, ck;
    uint32_t count, first;
    int32_t bin;
    bool live;
    float bval;  // lane < 24: B corner (lane / 3) component (lane % 3)
  };
  struct Rec {
    double fx, fy, fz, q;
    float u, v, w;
    int32_t key;
    bool present;
  };
  auto load_meta = [&](long long grp_) {
    Meta m{0, 0, 0, 0u, 0u, -1, false, 0.0f};
    const long long cell = grp_ * kCells + warp;
    if (grp_ < groups && cell < cells) {
      m.live = true;
      m.ci = int(cell % g.nx); m.cj = int((cell / g.nx) % g.ny); m.ck = int(cell / ((long long)g.nx * g.ny));
      m.bin = g.encode(m.ci, m.cj, m.ck);
      m.count = counts[m.bin];
      m.first = offsets[m.bin];
      if (lane < 24) {
        const int a = lane / 3, c = lane % 3;
        m.bval = bnode[c * nn + g.node(m.ci + (a & 1), m.cj + ((a >> 1) & 1), m.ck + ((a >> 2) & 1))];
      }
    }
    return m;
  };
  auto load_rec = [&](const Meta& m, uint32_t k) {
    Rec r{0.0, 0.0, 0.0, 0.0, 0.0f, 0.0f, 0.0f, -1, false};
    if (k < m.count) {
      const uint32_t n = m.first + k;
      r.present = true;
      r.fx = rx[n]; r.fy = ry[n]; r.fz = rz[n]; r.q = q[n];
      r.u = u[n]; r.v = v[n]; r.w = w[n]; r.key = key[n];
    }
    return r;
  };
  Meta cur = load_meta(blockIdx.x);
  Rec pre = load_rec(cur, lane);

  for (long long grp = blockIdx.x; grp < groups && !failed; grp += gridDim.x) {
    const Meta nxt = load_meta(grp + gridDim.x);
    const bool live = cur.live;
    const int ci = cur.ci, cj = cur.cj, ck = cur.ck;
    const uint32_t count = cur.count;
    const int32_t bin = cur.bin;
    if (live && lane < 24) sh.bcache[warp][lane] = cur.bval;
    if (lane == 0) sh.count[warp] = count;
    __syncthreads();
    uint32_t maxc = sh.count[0];
#pragma unroll
    for (int c = 1; c < kCells; ++c) maxc = max(maxc, sh.count[c]);
    float jsum[24];
#pragma unroll
    for (int t = 0; t < 24; ++t) jsum[t] = 0.0f;
    if (maxc == 0) pre = load_rec(nxt, lane);

    for (uint32_t chunk = 0; chunk < maxc; chunk += kChunk) {
      // The buffer is free once the MMAs that read it have completed.
      bool bad = false;
      if (pending[buf]) {
        bad = !tc::mbar_wait(&sh.mbar[buf], phase[buf]);
        phase[buf] ^= 1u;
        pending[buf] = false;
      }
      const Rec rec = pre;
      pre = chunk + kChunk < maxc ? load_rec(cur, chunk + kChunk + lane) : load_rec(nxt, lane);
      // Particle phase: one record per lane.
      float bv[kCols];
      float fac[12];
#pragma unroll
      for (int c = 0; c < kCols; ++c) bv[c] = 0.0f;
#pragma unroll
      for (int f = 0; f < 12; ++f) fac[f] = 0.0f;
      if (rec.present) {
        const double fx = rec.fx, fy = rec.fy, fz = rec.fz;
        if (rec.key == bin && fx >= 0 && fx < 1 && fy >= 0 && fy < 1 && fz >= 0 && fz < 1) {
          const float x = float(fx), y = float(fy), z = float(fz);
          float wt[8];
          cic_weights<float>(x, y, z, wt);
          float b[3];
#pragma unroll
          for (int c = 0; c < 3; ++c) {
            float val = 0.0f;
#pragma unroll
            for (int a = 0; a < 8; ++a) val += wt[a] * sh.bcache[warp][a * 3 + c];
            b[c] = val;
          }
          const Response<float> r(b[0], b[1], b[2], tp.beta_over_c);
          const float charge = float(rec.q);
          float hx, hy, hz;
          r.apply(rec.u, rec.v, rec.w, hx, hy, hz);
          const float qv = charge * tp.inv_volume;
          const float jc[3] = {qv * hx, qv * hy, qv * hz};
          const float scale = tp.beta_over_c * charge;
          if (isfinite(jc[0]) && isfinite(jc[1]) && isfinite(jc[2]) && isfinite(r.norm_square) && isfinite(scale)) {
#pragma unroll
            for (int a = 0; a < 8; ++a)
#pragma unroll
              for (int c = 0; c < 3; ++c) jsum[a * 3 + c] += __fmul_rn(jc[c], wt[a]);
#pragma unroll
            for (int e = 0; e < 9; ++e) bv[e] = r.a[e] * scale;
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
            atomicAdd(invalid, 1u);
          }
        } else {
          atomicAdd(invalid, 1u);
        }
      }
      // B tile (MN-major core matrices: 8 K-rows x 16 bytes of N-values,
      // K-groups 128 B apart, 16-byte N-chunks 512 B apart).
      if constexpr (!Bf16) {
        // K-major: value (n, k) at (n%8)*16 + (n/8)*128 + (k/4)*784 + (k%4)*4.
        uint8_t* bt = sh.btile[buf][0] + (lane >> 2) * kTf32KChunk + (lane & 3) * 4;
#pragma unroll
        for (int c = 0; c < kCols; ++c) {
          const int nn = kCols * warp + c;
          *reinterpret_cast<uint32_t*>(bt + (nn & 7) * 16 + (nn >> 3) * 128) = tc::to_tf32(bv[c]);
        }
      } else {
        float hi[kCols], lo[kCols];
#pragma unroll
        for (int c = 0; c < kCols; ++c) split_bf16(bv[c], hi[c], lo[c]);
#pragma unroll
        for (int j = 0; j < 2; ++j) {
          const uint4 ph = make_uint4(pack_bf16(hi[8 * j + 0], hi[8 * j + 1]), pack_bf16(hi[8 * j + 2], hi[8 * j + 3]),
                                      pack_bf16(hi[8 * j + 4], hi[8 * j + 5]), pack_bf16(hi[8 * j + 6], hi[8 * j + 7]));
          const uint4 pl = make_uint4(pack_bf16(lo[8 * j + 0], lo[8 * j + 1]), pack_bf16(lo[8 * j + 2], lo[8 * j + 3]),
                                      pack_bf16(lo[8 * j + 4], lo[8 * j + 5]), pack_bf16(lo[8 * j + 6], lo[8 * j + 7]));
          const int off = (2 * warp + j) * 512 + (lane >> 3) * 128 + (lane & 7) * 16;
          *reinterpret_cast<uint4*>(sh.btile[buf][0] + off) = ph;
          *reinterpret_cast<uint4*>(sh.btile[buf][1] + off) = pl;
        }
      }
#pragma unroll
      for (int f = 0; f < 12; ++f) sh.fac[warp][f][lane] = fac[f];
      __syncwarp();
      // A: lane t of warp w writes m_pt of the chunk's 32 particles into
      // tensor-memory lane 32w + t (TF32: columns 32*buf .. +31; BF16: the
      // hi pairs in columns 32*buf .. +15 and the lo pairs in +16 .. +31).
      const bool row = t_row < 27;
      const float* xrow = sh.fac[warp][row ? tx : 0];
      const float* yzrow = sh.fac[warp][row ? 3 + tyz : 0];
      if constexpr (!Bf16) {
#pragma unroll
        for (int q8 = 0; q8 < 4; ++q8) {
          uint32_t m[8];
#pragma unroll
          for (int h = 0; h < 2; ++h) {
            const float4 xf = *reinterpret_cast<const float4*>(xrow + 8 * q8 + 4 * h);
            const float4 yzf = *reinterpret_cast<const float4*>(yzrow + 8 * q8 + 4 * h);
            m[4 * h + 0] = row ? tc::to_tf32(xf.x * yzf.x) : 0u;
            m[4 * h + 1] = row ? tc::to_tf32(xf.y * yzf.y) : 0u;
            m[4 * h + 2] = row ? tc::to_tf32(xf.z * yzf.z) : 0u;
            m[4 * h + 3] = row ? tc::to_tf32(xf.w * yzf.w) : 0u;
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
            float v4[4] = {xf.x * yzf.x, xf.y * yzf.y, xf.z * yzf.z, xf.w * yzf.w};
            float hi4[4], lo4[4];
#pragma unroll
            for (int e = 0; e < 4; ++e) {
              split_bf16(row ? v4[e] : 0.0f, hi4[e], lo4[e]);
            }
            mh[2 * h + 0] = pack_bf16(hi4[0], hi4[1]);
            mh[2 * h + 1] = pack_bf16(hi4[2], hi4[3]);
            ml[2 * h + 0] = pack_bf16(lo4[0], lo4[1]);
            ml[2 * h + 1] = pack_bf16(lo4[2], lo4[3]);
          }
          tc::tmem_st8(tmem + lane_base + (buf ? 32u : 0u) + 8 * q16, mh);
          tc::tmem_st8(tmem + lane_base + (buf ? 32u : 0u) + 16 + 8 * q16, ml);
        }
      }
      tc::tmem_wait_st();
      tc::fence_proxy_async_smem();
      tc::fence_before_sync();
      if (__syncthreads_or(bad)) {
        failed = true;
        break;
      }
      if (threadIdx.x == 0) {
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
      pending[buf] = true;
      buf ^= 1;
    }
    if (failed) break;

    // J-hat corner sums of this warp's cell: reduce-scatter of the 24 lane
    // sums, staged for the coalesced moment store.
    {
      const bool b4 = lane & 16, b3 = lane & 8, b2 = lane & 4;
      float h12[12];
#pragma unroll
      for (int t = 0; t < 12; ++t) {
        const float keep = b4 ? jsum[t + 12] : jsum[t];
        const float send = b4 ? jsum[t] : jsum[t + 12];
        h12[t] = keep + __shfl_xor_sync(0xffffffffu, send, 16);
      }
      float h6[6];
#pragma unroll
      for (int t = 0; t < 6; ++t) {
        const float keep = b3 ? h12[t + 6] : h12[t];
        const float send = b3 ? h12[t] : h12[t + 6];
        h6[t] = keep + __shfl_xor_sync(0xffffffffu, send, 8);
      }
      float h3[3];
#pragma unroll
      for (int t = 0; t < 3; ++t) {
        const float keep = b2 ? h6[t + 3] : h6[t];
        const float send = b2 ? h6[t] : h6[t + 3];
        h3[t] = keep + __shfl_xor_sync(0xffffffffu, send, 4);
      }
#pragma unroll
      for (int t = 0; t < 3; ++t) {
        h3[t] += __shfl_xor_sync(0xffffffffu, h3[t], 2);
        h3[t] += __shfl_xor_sync(0xffffffffu, h3[t], 1);
      }
      if ((lane & 3) == 0) {
        const int index0 = (b4 ? 12 : 0) + (b3 ? 6 : 0) + (b2 ? 3 : 0);
#pragma unroll
        for (int t = 0; t < 3; ++t) {
          float value = live ? h3[t] : 0.0f;
          if (!isfinite(value)) {
            atomicAdd(invalid, 1u);
            value = 0.0f;
          }
          sh.stage[kMassMoments + index0 + t][warp] = value;
        }
      }
    }

    // Mass moments: wait for the group's last MMA and read G_w.
    if (maxc > 0) {
      const int last = buf ^ 1;
      const bool ok = tc::mbar_wait(&sh.mbar[last], phase[last]);
      phase[last] ^= 1u;
      pending[last] = false;
      tc::fence_after_sync();
      if (__syncthreads_or(!ok)) {
        failed = true;
        break;
      }
      uint32_t gbits[8], g8;
      tc::tmem_ld8(tmem + lane_base + kDcol + kCols * warp, gbits);
      tc::tmem_ld1(tmem + lane_base + kDcol + kCols * warp + 8, g8);
      tc::tmem_wait_ld();
      if (t_row < 27) {
        float G[9];
#pragma unroll
        for (int e = 0; e < 8; ++e) G[e] = __uint_as_float(gbits[e]);
        G[8] = __uint_as_float(g8);
#pragma unroll
        for (int e = 0; e < 9; ++e) {
          float value = (live && count > 0) ? G[e] : 0.0f;
          if (!isfinite(value)) {
            atomicAdd(invalid, 1u);
            value = 0.0f;
          }
          sh.stage[t_row * 9 + e][warp] = value;
        }
      }
    } else if (t_row < 27) {
#pragma unroll
      for (int e = 0; e < 9; ++e) sh.stage[t_row * 9 + e][warp] = 0.0f;
    }
    __syncthreads();
    // Coalesced moment store: entry q of the group's four cells is 16 bytes.
    for (int qi = threadIdx.x; qi < kMoments; qi += blockDim.x) {
      float4 val = make_float4(sh.stage[qi][0], sh.stage[qi][1], sh.stage[qi][2], sh.stage[qi][3]);
      float4* dst = reinterpret_cast<float4*>(mom + qi * mom_stride + grp * kCells);
      if (accumulate) {
        const float4 old = *dst;
        val.x += old.x; val.y += old.y; val.z += old.z; val.w += old.w;
      }
      *dst = val;
    }
    // D is overwritten by the next group's first MMA only after every warp
    // has read it.
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    cur = nxt;
  }

  if (failed && threadIdx.x == 0) atomicAdd(invalid, 1u << 20);
  // Retire in-flight MMAs (bounded) before freeing tensor memory.
#pragma unroll
  for (int b = 0; b < 2; ++b)
    if (pending[b]) tc::mbar_wait(&sh.mbar[b], phase[b]);
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  if (warp == 0) tc::tmem_dealloc(tmem, kTmemCols);
}

}  // namespace

long long moment_stride(const Geom& g) {
  const long long cells = (long long)g.nx * g.ny * g.nz;
  return (cells + kCells - 1) / kCells * kCells;
}
size_t moment_floats(const Geom& g) { return size_t(kMoments) * size_t(moment_stride(g)); }

cudaError_t launch_deposit_tc(int mass_kind, const Geom& g, double qom, double dt, double c,
                              const tpicb200_particles* p, const uint32_t* counts, const uint32_t* offsets,
                              const void* bnode, float* moments, int accumulate, uint32_t* invalid,
                              cudaStream_t s) {
  if (mass_kind != TPICB200_MASS_TF32 && mass_kind != TPICB200_MASS_BF16X3) return cudaErrorNotSupported;
  if (!moments) return cudaErrorInvalidValue;
  TcParams tp{float(qom * dt / 2 / c), float(g.inv_volume)};
  int device = 0, sms = 148;
  cudaGetDevice(&device);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  const long long cells = (long long)g.nx * g.ny * g.nz;
  const long long groups = (cells + kCells - 1) / kCells;
  const unsigned blocks = unsigned(std::min<long long>(groups, 4LL * sms));
  // Dynamic shared-memory padding brings each CTA to ~47 KB, so at most four
  // CTAs (4 x 128 tensor-memory columns = all 512) are resident per SM and
  // no tcgen05.alloc ever waits for another CTA's columns.
  const bool tf32 = mass_kind == TPICB200_MASS_TF32;
  auto kernel = tf32 ? tc_deposit_kernel<false> : tc_deposit_kernel<true>;
  const int pad = 47 * 1024 - int(tf32 ? sizeof(TcShared<false>) : sizeof(TcShared<true>));
  kernel<<<blocks, 128, pad, s>>>(g, tp, (const double*)p->rx, (const double*)p->ry,
      (const double*)p->rz, (const float*)p->u, (const float*)p->v, (const float*)p->w, p->q, p->cell, counts,
      offsets, (const float*)bnode, moments, moment_stride(g), accumulate, invalid);
  count_launches(1);
  return cudaGetLastError();
}

namespace {

// For every stencil: the corners a whose pair (a, a + offset) lies in one
// cell, and that pair's monomial class t.
struct StencilPairs {
  int count[14];
  int corner[14][8];
  int monomial[14][8];
};
constexpr StencilPairs make_stencil_pairs() {
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
__constant__ StencilPairs c_stencil_pairs = make_stencil_pairs();

// Record entry k < 126 (stencil k/9, component k%9) and current component
// k - 126 of every unique node, summed over the cells that share it in
// increasing corner order, added to M and J.
__global__ void __launch_bounds__(256) assemble_moments_kernel(Geom g, const float* __restrict__ mom,
                                                               long long stride, float* __restrict__ J,
                                                               float* __restrict__ M) {
  const long long unique = (long long)g.nx * g.ny * g.nz;
  const long long total = 129 * unique;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    const int k = int(t / unique);
    const long long vtx = t - k * unique;
    const int i = int(vtx % g.nx), j = int((vtx / g.nx) % g.ny), kk = int(vtx / ((long long)g.nx * g.ny));
    auto cell_of = [&](int a) {
      const int ci = wrap_index(i - (a & 1), g.nx), cj = wrap_index(j - ((a >> 1) & 1), g.ny),
                ck = wrap_index(kk - ((a >> 2) & 1), g.nz);
      return ci + (long long)g.nx * (cj + (long long)g.ny * ck);
    };
    const long long node = g.node(i, j, kk);
    if (k < 126) {
      const int s = k / 9, e = k - 9 * (k / 9);
      float sum = 0.0f;
      const int n = c_stencil_pairs.count[s];
      for (int p = 0; p < n; ++p)
        sum += mom[(c_stencil_pairs.monomial[s][p] * 9 + e) * stride + cell_of(c_stencil_pairs.corner[s][p])];
      if (sum != 0.0f) M[g.mass_index(node, k)] += sum;
    } else {
      const int c = k - 126;
      float sum = 0.0f;
#pragma unroll
      for (int a = 0; a < 8; ++a) sum += mom[(kMassMoments + a * 3 + c) * stride + cell_of(a)];
      if (sum != 0.0f) J[c * g.nodes + node] += sum;
    }
  }
}

}  // namespace

cudaError_t launch_assemble_moments(const Geom& g, const float* moments, void* j, void* mass, cudaStream_t s) {
  const long long total = 129LL * g.nx * g.ny * g.nz;
  assemble_moments_kernel<<<grid_for(total, 256, 148u * 16u), 256, 0, s>>>(g, moments, moment_stride(g),
                                                                           (float*)j, (float*)mass);
  count_launches(1);
  return cudaGetLastError();
}

}  // namespace tpicb200
