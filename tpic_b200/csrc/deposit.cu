// Implicit current (J-hat) and mass-matrix deposition on CUDA cores, and the
// periodic fold of both.
//
// Sorted form: one warp per interior cell bin (the records of a cell are
// contiguous after the sort). The warp caches the cell's eight nodal B
// corners in shared memory, every lane samples one record per 32-record
// chunk (CIC weights, gathered B, response alpha), and
//   * J-hat: each lane keeps 24 corner/component sums of its records, the
//     warp reduce-scatters them (27 shuffles) and 8 lane groups add 24 values
//     with atomics; every product is rounded on its own before its addition
//     (deposit_product, ecsim/deposition/current_deposition_device.hpp:44-58);
//   * mass: lanes own two of the 64 ordered corner pairs (lane/4, 2*(lane%4)+slot)
//     and accumulate alpha*scale*(W_a*W_b) for all nine tensor components by
//     shuffling each record's fractions and scaled response, as the reference's
//     sorted scalar kernel (ecsim/mass_matrix/mass_matrix_scalar_device.hpp:121-232);
//     the 36 canonical pairs are flushed with 9 atomics each.
// Deposits target the periodic unique node (index n wraps to 0), so the fold
// afterwards only replicates unique nodes into duplicates and ghosts.
//
// Unsorted form: one thread per record with global atomics
// (current_deposition_device.hpp:150-161, mass_matrix_scalar_device.hpp:107-116).
#include "kernels.cuh"

namespace tpicb200 {
namespace {

template <class C> __device__ __forceinline__ C mul_rn(C a, C b);
template <> __device__ __forceinline__ float mul_rn<float>(float a, float b) { return __fmul_rn(a, b); }
template <> __device__ __forceinline__ double mul_rn<double>(double a, double b) { return __dmul_rn(a, b); }

template <class C>
__device__ __forceinline__ C corner_weight(int a, C x, C y, C z) {
  return ((a & 1) ? x : C(1) - x) * ((a & 2) ? y : C(1) - y) * ((a & 4) ? z : C(1) - z);
}

struct DepositParams {
  double beta_over_c;  // (q/m) dt / (2c)
  double inv_volume;
};

__device__ __forceinline__ long long wrapped_node(const Geom& g, int i, int j, int k) {
  return g.node(i == g.nx ? 0 : i, j == g.ny ? 0 : j, k == g.nz ? 0 : k);
}
__device__ __forceinline__ long long wrapped_mass_vertex(const Geom& g, int i, int j, int k) {
  return g.mass_vertex(i == g.nx ? 0 : i, j == g.ny ? 0 : j, k == g.nz ? 0 : k);
}

// ---------------------------------------------------------------------------
// Unsorted per-record deposition.
template <class P, class MC>
__global__ void __launch_bounds__(128) unsorted_deposit_kernel(Geom g, DepositParams dp,
    const double* __restrict__ rx, const double* __restrict__ ry, const double* __restrict__ rz,
    const typename P::Vel* __restrict__ u, const typename P::Vel* __restrict__ v,
    const typename P::Vel* __restrict__ w, const double* __restrict__ q,
    const int32_t* __restrict__ key, uint32_t count, const typename P::Fld* __restrict__ bnode,
    typename P::Fld* __restrict__ J, typename P::Mass* __restrict__ M, uint32_t* invalid) {
  using C = typename P::VC;
  using Cur = typename P::Fld;
  using Mass = typename P::Mass;
  const long long nn = g.nodes;
  for (uint32_t n = blockIdx.x * blockDim.x + threadIdx.x; n < count; n += gridDim.x * blockDim.x) {
    const int32_t k0 = key[n];
    int ci, cj, ck;
    bool ok = k0 >= 0 && (long long)k0 < g.bins;
    if (ok) {
      g.decode(k0, ci, cj, ck);
      ok = g.interior_cell(ci, cj, ck);
    }
    const double fx = rx[n], fy = ry[n], fz = rz[n];
    ok = ok && fx >= 0 && fx < 1 && fy >= 0 && fy < 1 && fz >= 0 && fz < 1;
    if (!ok) { atomicAdd(invalid, 1u); continue; }
    long long nodes[8];
#pragma unroll
    for (int a = 0; a < 8; ++a)
      nodes[a] = wrapped_node(g, ci + (a & 1), cj + ((a >> 1) & 1), ck + ((a >> 2) & 1));
    const long long base = g.node(ci, cj, ck);
    const long long off[8] = {0, 1, g.NX, g.NX + 1, (long long)g.NX * g.NY, (long long)g.NX * g.NY + 1,
                              (long long)g.NX * g.NY + g.NX, (long long)g.NX * g.NY + g.NX + 1};
    if (J) {
      C wt[8];
      cic_weights<C>(C(fx), C(fy), C(fz), wt);
      C b[3];
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        C val = 0;
#pragma unroll
        for (int a = 0; a < 8; ++a) val += wt[a] * C(bnode[c * nn + base + off[a]]);
        b[c] = val;
      }
      const Response<C> r(b[0], b[1], b[2], C(dp.beta_over_c));
      C hx, hy, hz;
      r.apply(C(u[n]), C(v[n]), C(w[n]), hx, hy, hz);
      const C qv = C(q[n]) * C(dp.inv_volume);
      const C jc[3] = {qv * hx, qv * hy, qv * hz};
      if (!isfinite(jc[0]) || !isfinite(jc[1]) || !isfinite(jc[2])) { atomicAdd(invalid, 1u); continue; }
#pragma unroll
      for (int a = 0; a < 8; ++a) {
        if (wt[a] == C(0)) continue;
#pragma unroll
        for (int c = 0; c < 3; ++c) atomicAdd(J + c * nn + nodes[a], Cur(mul_rn(jc[c], wt[a])));
      }
    }
    if (M) {
      MC wt[8];
      cic_weights<MC>(MC(fx), MC(fy), MC(fz), wt);
      MC b[3];
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        MC val = 0;
#pragma unroll
        for (int a = 0; a < 8; ++a) val += wt[a] * MC(bnode[c * nn + base + off[a]]);
        b[c] = val;
      }
      const Response<MC> r(b[0], b[1], b[2], MC(dp.beta_over_c));
      const MC scale = MC(dp.beta_over_c) * MC(q[n]);
      MC as[9];
      bool fin = true;
#pragma unroll
      for (int e = 0; e < 9; ++e) { as[e] = r.a[e] * scale; fin = fin && isfinite(as[e]); }
      if (!fin) { atomicAdd(invalid, 1u); continue; }
#pragma unroll
      for (int a = 0; a < 8; ++a)
#pragma unroll
        for (int bb = 0; bb < 8; ++bb) {
          const int s = pair_stencil(a, bb);
          if (s < 0) continue;
          const MC pw = wt[a] * wt[bb];
          if (pw == MC(0)) continue;
#pragma unroll
          for (int e = 0; e < 9; ++e) {
            const Mass amount = Mass(as[e] * pw);
            if (amount != Mass(0))
              atomicAdd(M + g.mass_index(wrapped_mass_vertex(g, ci + (a & 1), cj + ((a >> 1) & 1),
                                                             ck + ((a >> 2) & 1)),
                                         s * 9 + e),
                        amount);
          }
        }
    }
  }
}

// ---------------------------------------------------------------------------
// Sorted warp-per-cell deposition. MC is the mass arithmetic/accumulator type
// (the precision's compute type for SCALAR, double for SCALAR_F64).
template <class P, class MC>
__global__ void __launch_bounds__(128) sorted_deposit_kernel(Geom g, DepositParams dp,
    const double* __restrict__ rx, const double* __restrict__ ry, const double* __restrict__ rz,
    const typename P::Vel* __restrict__ u, const typename P::Vel* __restrict__ v,
    const typename P::Vel* __restrict__ w, const double* __restrict__ q,
    const int32_t* __restrict__ key, const uint32_t* __restrict__ counts,
    const uint32_t* __restrict__ offsets, const typename P::Fld* __restrict__ bnode,
    typename P::Fld* __restrict__ J, typename P::Mass* __restrict__ M, uint32_t* invalid,
    const uint32_t* __restrict__ perm, double* __restrict__ orx, double* __restrict__ ory,
    double* __restrict__ orz, typename P::Vel* __restrict__ ou, typename P::Vel* __restrict__ ov,
    typename P::Vel* __restrict__ ow, double* __restrict__ oq, int32_t* __restrict__ okey) {
  using C = typename P::VC;
  using Cur = typename P::Fld;
  using Mass = typename P::Mass;
  __shared__ C bcache[4][24];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const long long nn = g.nodes;
  const int corner_a = lane >> 2;
  const int lanes_per_corner = 4;
  int corner_b[2], stencil[2];
#pragma unroll
  for (int slot = 0; slot < 2; ++slot) {
    corner_b[slot] = 2 * (lane & 3) + slot;
    stencil[slot] = pair_stencil(corner_a, corner_b[slot]);
  }
  const long long cells = (long long)g.nx * g.ny * g.nz;
  for (long long cell = (long long)blockIdx.x * 4 + warp; cell < cells; cell += (long long)gridDim.x * 4) {
    const int ci = int(cell % g.nx), cj = int((cell / g.nx) % g.ny), ck = int(cell / ((long long)g.nx * g.ny));
    const int32_t bin = g.encode(ci, cj, ck);
    const uint32_t count = counts[bin];
    if (count == 0) continue;
    const uint32_t first = offsets[bin];
    if (lane < 24) {
      const int a = lane / 3, c = lane % 3;
      bcache[warp][lane] = C(bnode[c * nn + g.node(ci + (a & 1), cj + ((a >> 1) & 1), ck + ((a >> 2) & 1))]);
    }
    __syncwarp();
    Cur jsum[24];
#pragma unroll
    for (int t = 0; t < 24; ++t) jsum[t] = Cur(0);
    MC macc[2][9];
#pragma unroll
    for (int slot = 0; slot < 2; ++slot)
#pragma unroll
      for (int e = 0; e < 9; ++e) macc[slot][e] = MC(0);
    for (uint32_t chunk = 0; chunk < count; chunk += 32) {
      MC mx = 0, my = 0, mz = 0;
      MC as[9];
#pragma unroll
      for (int e = 0; e < 9; ++e) as[e] = MC(0);
      const uint32_t offset = chunk + lane;
      if (offset < count) {
        // With perm, the record at sorted position `pos` is read through it
        // and copied to that position of the sorted slot.
        const uint32_t pos = first + offset;
        const uint32_t n = perm ? perm[pos] : pos;
        const double fx = rx[n], fy = ry[n], fz = rz[n];
        if (orx) {
          orx[pos] = fx; ory[pos] = fy; orz[pos] = fz;
          ou[pos] = u[n]; ov[pos] = v[n]; ow[pos] = w[n];
          oq[pos] = q[n]; okey[pos] = key[n];
        }
        bool ok = key[n] == bin && fx >= 0 && fx < 1 && fy >= 0 && fy < 1 && fz >= 0 && fz < 1;
        if (ok) {
          const double charge = q[n];
          if (J) {
            C wt[8];
            cic_weights<C>(C(fx), C(fy), C(fz), wt);
            C b[3];
#pragma unroll
            for (int c = 0; c < 3; ++c) {
              C val = 0;
#pragma unroll
              for (int a = 0; a < 8; ++a) val += wt[a] * bcache[warp][a * 3 + c];
              b[c] = val;
            }
            const Response<C> r(b[0], b[1], b[2], C(dp.beta_over_c));
            C hx, hy, hz;
            r.apply(C(u[n]), C(v[n]), C(w[n]), hx, hy, hz);
            const C qv = C(charge) * C(dp.inv_volume);
            const C jc[3] = {qv * hx, qv * hy, qv * hz};
            if (isfinite(jc[0]) && isfinite(jc[1]) && isfinite(jc[2])) {
#pragma unroll
              for (int a = 0; a < 8; ++a)
#pragma unroll
                for (int c = 0; c < 3; ++c) jsum[a * 3 + c] += Cur(mul_rn(jc[c], wt[a]));
            } else {
              ok = false;
            }
          }
          if (M) {
            MC wt[8];
            cic_weights<MC>(MC(fx), MC(fy), MC(fz), wt);
            MC b[3];
#pragma unroll
            for (int c = 0; c < 3; ++c) {
              MC val = 0;
#pragma unroll
              for (int a = 0; a < 8; ++a) val += wt[a] * MC(bcache[warp][a * 3 + c]);
              b[c] = val;
            }
            const Response<MC> r(b[0], b[1], b[2], MC(dp.beta_over_c));
            const MC scale = MC(dp.beta_over_c) * MC(charge);
            if (isfinite(r.norm_square) && isfinite(scale)) {
#pragma unroll
              for (int e = 0; e < 9; ++e) as[e] = r.a[e] * scale;
              mx = MC(fx); my = MC(fy); mz = MC(fz);
            } else {
              ok = false;
            }
          }
        }
        if (!ok) {
          atomicAdd(invalid, 1u);
          mx = my = mz = MC(0);
#pragma unroll
          for (int e = 0; e < 9; ++e) as[e] = MC(0);
        }
      }
      if (M) {
        const uint32_t populated = count - chunk < 32u ? count - chunk : 32u;
        for (uint32_t src = 0; src < populated; ++src) {
          const MC x = __shfl_sync(0xffffffffu, mx, src);
          const MC y = __shfl_sync(0xffffffffu, my, src);
          const MC z = __shfl_sync(0xffffffffu, mz, src);
          const MC wa = corner_weight(corner_a, x, y, z);
          MC pw[2];
#pragma unroll
          for (int slot = 0; slot < 2; ++slot)
            pw[slot] = wa * __shfl_sync(0xffffffffu, wa, corner_b[slot] * lanes_per_corner);
#pragma unroll
          for (int e = 0; e < 9; ++e) {
            const MC alpha = __shfl_sync(0xffffffffu, as[e], src);
#pragma unroll
            for (int slot = 0; slot < 2; ++slot) {
              if constexpr (sizeof(MC) == sizeof(Mass))
                macc[slot][e] += MC(Mass(alpha * pw[slot]));
              else
                macc[slot][e] += alpha * pw[slot];
            }
          }
        }
      }
    }
    if (J) {
      // Reduce-scatter of the 24 sums: after the xor-16/8/4 halvings each lane
      // holds 3 partial sums of index 12*b4 + 6*b3 + 3*b2 + t; xor 2 and 1 finish.
      const bool b4 = lane & 16, b3 = lane & 8, b2 = lane & 4;
      Cur h12[12];
#pragma unroll
      for (int t = 0; t < 12; ++t) {
        const Cur keep = b4 ? jsum[t + 12] : jsum[t];
        const Cur send = b4 ? jsum[t] : jsum[t + 12];
        h12[t] = keep + __shfl_xor_sync(0xffffffffu, send, 16);
      }
      Cur h6[6];
#pragma unroll
      for (int t = 0; t < 6; ++t) {
        const Cur keep = b3 ? h12[t + 6] : h12[t];
        const Cur send = b3 ? h12[t] : h12[t + 6];
        h6[t] = keep + __shfl_xor_sync(0xffffffffu, send, 8);
      }
      Cur h3[3];
#pragma unroll
      for (int t = 0; t < 3; ++t) {
        const Cur keep = b2 ? h6[t + 3] : h6[t];
        const Cur send = b2 ? h6[t] : h6[t + 3];
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
          const int index = index0 + t, a = index / 3, c = index % 3;
          const Cur value = h3[t];
          if (!isfinite(value)) atomicAdd(invalid, 1u);
          else if (value != Cur(0))
            atomicAdd(J + c * nn + wrapped_node(g, ci + (a & 1), cj + ((a >> 1) & 1), ck + ((a >> 2) & 1)), value);
        }
      }
    }
    if (M) {
      const long long vertex = wrapped_mass_vertex(g, ci + (corner_a & 1), cj + ((corner_a >> 1) & 1),
                                                   ck + ((corner_a >> 2) & 1));
#pragma unroll
      for (int slot = 0; slot < 2; ++slot) {
        if (stencil[slot] < 0) continue;
#pragma unroll
        for (int e = 0; e < 9; ++e) {
          const Mass amount = Mass(macc[slot][e]);
          if (!isfinite(amount)) atomicAdd(invalid, 1u);
          else if (amount != Mass(0)) atomicAdd(M + g.mass_index(vertex, stencil[slot] * 9 + e), amount);
        }
      }
    }
    __syncwarp();
  }
}

// ---------------------------------------------------------------------------
// Fold: duplicates (index n) and ghosts (-1, n+1) take their unique node's
// value. Only the shell of non-unique vertices is visited.
// Component blockIdx.y; the shell index in 32-bit arithmetic (launch_fold
// checks that the shell holds fewer than 2^31 vertices).
template <class T>
__global__ void __launch_bounds__(256) fold_field_kernel(Geom g, T* __restrict__ f) {
  const uint32_t shell = uint32_t(shell_count(g));
  T* fc = f + (long long)blockIdx.y * g.nodes;
  for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < shell; t += gridDim.x * blockDim.x) {
    int i, j, k;
    shell_coordinates32(g, t, i, j, k);
    fc[g.node(i, j, k)] = fc[g.node(wrap_index(i, g.nx), wrap_index(j, g.ny), wrap_index(k, g.nz))];
  }
}

// Stencil-major and tiled layouts: a thread copies kFoldEntries entries
// (group blockIdx.y of the 126) of one shell vertex, each entry a coalesced
// row across the warp's vertices; the vertex is decoded once (32-bit
// arithmetic, checked by launch_fold). One thread per vertex and all 126
// entries took 342 us at 512 x 512 x 1, where the ghost planes hold three
// times the interior vertices.
constexpr int kFoldEntries = 9;
template <class T>
__global__ void __launch_bounds__(256) fold_mass_rows_kernel(Geom g, T* __restrict__ m) {
  const uint32_t shell = uint32_t(shell_count(g));
  const int e0 = int(blockIdx.y) * kFoldEntries;
  for (uint32_t sv = blockIdx.x * blockDim.x + threadIdx.x; sv < shell; sv += gridDim.x * blockDim.x) {
    int i, j, k;
    shell_coordinates32(g, sv, i, j, k);
    const long long to = g.mass_vertex(i, j, k),
                    from = g.mass_vertex(wrap_index(i, g.nx), wrap_index(j, g.ny), wrap_index(k, g.nz));
    T v[kFoldEntries];
#pragma unroll
    for (int e = 0; e < kFoldEntries; ++e) v[e] = m[g.mass_index(from, e0 + e)];
#pragma unroll
    for (int e = 0; e < kFoldEntries; ++e) m[g.mass_index(to, e0 + e)] = v[e];
  }
}

template <class T>
__global__ void __launch_bounds__(256) fold_mass_kernel(Geom g, T* __restrict__ m) {
  const long long total = shell_count(g) * 126;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    // Records: consecutive threads copy consecutive entries of one record;
    // stencil-major: consecutive threads copy one entry of consecutive vertices.
    const long long shell = shell_count(g);
    long long sv, e;
    if (g.mes == 1) { sv = t / 126; e = t - sv * 126; }
    else { e = t / shell; sv = t - e * shell; }
    int i, j, k;
    shell_coordinates(g, sv, i, j, k);
    m[g.mass_index(g.mass_vertex(i, j, k), int(e))] =
        m[g.mass_index(g.mass_vertex(wrap_index(i, g.nx), wrap_index(j, g.ny), wrap_index(k, g.nz)), int(e))];
  }
}

template <class P, class MC>
cudaError_t launch_typed(const Geom& g, DepositParams dp, const tpicb200_particles* p, const uint32_t* counts,
                         const uint32_t* offsets, const void* bnode, void* j, void* mass, uint32_t* invalid,
                         const SortedCopy* copy, cudaStream_t s) {
  using Vel = typename P::Vel;
  using Fld = typename P::Fld;
  using Mass = typename P::Mass;
  if (counts && offsets) {
    const long long cells = (long long)g.nx * g.ny * g.nz;
    const unsigned blocks = grid_for((cells + 3) / 4, 1, 148u * 64u);
    const bool c = copy && copy->perm && copy->out.rx;
    sorted_deposit_kernel<P, MC><<<blocks, 128, 0, s>>>(g, dp, (const double*)p->rx, (const double*)p->ry,
        (const double*)p->rz, (const Vel*)p->u, (const Vel*)p->v, (const Vel*)p->w, p->q, p->cell,
        counts, offsets, (const Fld*)bnode, (Fld*)j, (Mass*)mass, invalid, copy ? copy->perm : nullptr,
        c ? (double*)copy->out.rx : nullptr, c ? (double*)copy->out.ry : nullptr,
        c ? (double*)copy->out.rz : nullptr, c ? (Vel*)copy->out.u : nullptr, c ? (Vel*)copy->out.v : nullptr,
        c ? (Vel*)copy->out.w : nullptr, c ? copy->out.q : nullptr, c ? copy->out.cell : nullptr);
    count_launches(1);
  } else if (p->count) {
    unsorted_deposit_kernel<P, MC><<<grid_for(p->count, 128, 148u * 16u), 128, 0, s>>>(g, dp,
        (const double*)p->rx, (const double*)p->ry, (const double*)p->rz, (const Vel*)p->u,
        (const Vel*)p->v, (const Vel*)p->w, p->q, p->cell, p->count, (const Fld*)bnode, (Fld*)j,
        (Mass*)mass, invalid);
    count_launches(1);
  }
  return cudaGetLastError();
}

}  // namespace

cudaError_t launch_deposit(int precision, int mass_kind, const Geom& g, double qom, double dt,
                           double c, const tpicb200_particles* p, const uint32_t* counts,
                           const uint32_t* offsets, const void* bnode, void* j, void* mass,
                           uint32_t* invalid, const SortedCopy* copy, cudaStream_t s) {
  DepositParams dp{qom * dt / 2 / c, g.inv_volume};
  if (precision == TPICB200_PRECISION_DOUBLE)
    return launch_typed<PDouble, double>(g, dp, p, counts, offsets, bnode, j, mass, invalid, copy, s);
  if (mass_kind == TPICB200_MASS_SCALAR_F64)
    return launch_typed<PMixed, double>(g, dp, p, counts, offsets, bnode, j, mass, invalid, copy, s);
  return launch_typed<PMixed, float>(g, dp, p, counts, offsets, bnode, j, mass, invalid, copy, s);
}

namespace {
__global__ void __launch_bounds__(256) copy_ids_kernel(const uint32_t* __restrict__ perm,
                                                       const uint64_t* __restrict__ in, uint64_t* __restrict__ out,
                                                       uint32_t count) {
  for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < count; p += gridDim.x * blockDim.x)
    out[p] = in[perm[p]];
}
}  // namespace

cudaError_t launch_copy_ids(const tpicb200_particles* in, const SortedCopy* copy, cudaStream_t s) {
  if (!copy || !copy->perm || !copy->out.rx || !in->id || !copy->out.id || in->count == 0) return cudaSuccess;
  copy_ids_kernel<<<grid_for(in->count, 256, 148u * 8u), 256, 0, s>>>(copy->perm, in->id, copy->out.id, in->count);
  count_launches(1);
  return cudaGetLastError();
}

cudaError_t launch_fold(int precision, const Geom& g, void* j, void* mass, cudaStream_t s) {
  if (shell_count(g) >= (1LL << 31)) return cudaErrorInvalidValue;
  if (j) {
    const dim3 blocks(grid_for(shell_count(g), 256), 3);
    if (precision == TPICB200_PRECISION_DOUBLE) fold_field_kernel<double><<<blocks, 256, 0, s>>>(g, (double*)j);
    else fold_field_kernel<float><<<blocks, 256, 0, s>>>(g, (float*)j);
    count_launches(1);
  }
  if (mass) {
    if (g.mes != 1) {
      const dim3 blocks(grid_for(shell_count(g), 256), 126 / kFoldEntries);
      if (precision == TPICB200_PRECISION_DOUBLE) fold_mass_rows_kernel<double><<<blocks, 256, 0, s>>>(g, (double*)mass);
      else fold_mass_rows_kernel<float><<<blocks, 256, 0, s>>>(g, (float*)mass);
    } else {
      const unsigned blocks = grid_for(126 * shell_count(g), 256, 148u * 8u);
      if (precision == TPICB200_PRECISION_DOUBLE) fold_mass_kernel<double><<<blocks, 256, 0, s>>>(g, (double*)mass);
      else fold_mass_kernel<float><<<blocks, 256, 0, s>>>(g, (float*)mass);
    }
    count_launches(1);
  }
  return cudaGetLastError();
}

}  // namespace tpicb200
