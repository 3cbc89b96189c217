// Field kernels of the cycle: periodic node/cell ghost fills, cell-to-node
// B, the Maxwell right-hand side, the E/B advance and the energy reductions.
// All are HBM-streaming stencils, one thread per target sample.
#include "kernels.cuh"
#include "stencils.cuh"

namespace tpicb200 {
namespace {

// Ghost nodes take their periodic images; component blockIdx.y. The shell
// index is decoded in 32-bit arithmetic (launch_node_ghosts checks that the
// shell holds fewer than 2^31 nodes): on a grid one cell thick the ghost
// planes hold three times the interior, and 64-bit division per node took
// 23 us per fill at 512 x 512 x 1.
template <class T>
__global__ void __launch_bounds__(256) node_fill_kernel(Geom g, T* __restrict__ f) {
  wait_for_predecessor();
  const uint32_t shell = uint32_t(shell_count(g));
  T* fc = f + (long long)blockIdx.y * g.nodes;
  for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < shell; t += gridDim.x * blockDim.x) {
    int i, j, k;
    shell_coordinates32(g, t, i, j, k);
    fc[g.node(i, j, k)] = fc[g.node(wrap_index(i, g.nx), wrap_index(j, g.ny), wrap_index(k, g.nz))];
  }
}

// Ghost cells -1 and n per axis take cells n-1 and 0.
template <class T>
__global__ void __launch_bounds__(256) cell_fill_kernel(Geom g, T* __restrict__ f) {
  const long long zs = (long long)g.CX * g.CY, ys = (long long)g.CX * g.nz, xs = (long long)g.ny * g.nz;
  const long long shell = 2 * (zs + ys + xs), total = 3 * shell;
  for (long long t0 = blockIdx.x * (long long)blockDim.x + threadIdx.x; t0 < total;
       t0 += (long long)gridDim.x * blockDim.x) {
    const long long c = t0 / shell;
    long long t = t0 - c * shell;
    int i, j, k;
    if (t < 2 * zs) {
      const int p = int(t / zs);
      const long long r = t - p * zs;
      k = p == 0 ? -1 : g.nz;
      i = int(r % g.CX) - 1;
      j = int(r / g.CX) - 1;
    } else if ((t -= 2 * zs) < 2 * ys) {
      const int p = int(t / ys);
      const long long r = t - p * ys;
      j = p == 0 ? -1 : g.ny;
      i = int(r % g.CX) - 1;
      k = int(r / g.CX);
    } else {
      t -= 2 * ys;
      const int p = int(t / xs);
      const long long r = t - p * xs;
      i = p == 0 ? -1 : g.nx;
      j = int(r % g.ny);
      k = int(r / g.ny);
    }
    f[c * g.cells + g.cell(i, j, k)] =
        f[c * g.cells + g.cell(wrap_index(i, g.nx), wrap_index(j, g.ny), wrap_index(k, g.nz))];
  }
}

// cell_to_node_average in Compute::Magnetic (ecsim/fields/cell_to_node.hpp:19-32,
// ecsim/fields/cell_to_node_device.hpp:17-38), interior nodes.
template <class C, class T>
__global__ void __launch_bounds__(256) cell_to_node_kernel(Geom g, const T* __restrict__ cellf, T* __restrict__ node) {
  const long long total = 3 * g.interior;
  for (long long t0 = blockIdx.x * (long long)blockDim.x + threadIdx.x; t0 < total;
       t0 += (long long)gridDim.x * blockDim.x) {
    const long long c = t0 / g.interior;
    int i, j, k;
    interior_node_coordinates(g, t0 - c * g.interior, i, j, k);
    const T* f = cellf + c * g.cells;
    const C v = (C(f[g.cell(i - 1, j - 1, k - 1)]) + C(f[g.cell(i, j - 1, k - 1)]) +
                 C(f[g.cell(i - 1, j, k - 1)]) + C(f[g.cell(i, j, k - 1)]) +
                 C(f[g.cell(i - 1, j - 1, k)]) + C(f[g.cell(i, j - 1, k)]) +
                 C(f[g.cell(i - 1, j, k)]) + C(f[g.cell(i, j, k)])) * C(0.125);
    node[c * g.nodes + g.node(i, j, k)] = T(v);
  }
}

// rhs = ((1*E + delta*curl_C2N(B)) + (-k)*J) in Compute::Electric
// (MaxwellOperator::complete_rhs, ecsim/maxwell/maxwell_device.hpp:152-172).
template <class C, class T, class TJ>
__global__ void __launch_bounds__(256) rhs_kernel(Geom g, C delta, C kfac, const T* __restrict__ e,
                                                  const T* __restrict__ bcell, const TJ* __restrict__ j,
                                                  double* __restrict__ rhs) {
  const C inv[3] = {C(g.inv[0]), C(g.inv[1]), C(g.inv[2])};
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < g.interior;
       t += (long long)gridDim.x * blockDim.x) {
    int i, jj, k;
    interior_node_coordinates(g, t, i, jj, k);
    C cb[3];
    curl_c2n_at<C>(g, bcell, i, jj, k, inv, cb);
    const long long at = g.node(i, jj, k);
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const long long p = c * g.nodes + at;
      rhs[p] = double((C(1) * C(e[p]) + delta * cb[c]) + (-kfac) * C(j[p]));
    }
  }
}

// E update over interior nodes (field_vector_linear_combination, two terms).
template <class C, class T>
__global__ void __launch_bounds__(256) e_update_kernel(Geom g, C a, C b, bool copy, T* __restrict__ e,
                                                       const double* __restrict__ th, uint32_t* invalid) {
  const long long total = 3 * g.interior;
  for (long long t0 = blockIdx.x * (long long)blockDim.x + threadIdx.x; t0 < total;
       t0 += (long long)gridDim.x * blockDim.x) {
    const long long c = t0 / g.interior;
    int i, j, k;
    interior_node_coordinates(g, t0 - c * g.interior, i, j, k);
    const long long p = c * g.nodes + g.node(i, j, k);
    const T value = copy ? T(th[p]) : T(a * C(th[p]) + b * C(e[p]));
    e[p] = value;
    if (!isfinite(value)) atomicAdd(invalid, 1u);
  }
}

// Faraday: next = 1*B + faraday*curl_N2C(theta) in Compute::Magnetic over all
// cells (faraday_update_kernel, ecsim/maxwell/field_update_device.hpp:25-44).
template <class C, class T>
__global__ void __launch_bounds__(256) faraday_kernel(Geom g, C faraday, const T* __restrict__ b,
                                                      const double* __restrict__ th, T* __restrict__ next,
                                                      uint32_t* invalid) {
  const C inv[3] = {C(g.inv[0]), C(g.inv[1]), C(g.inv[2])};
  const long long cells = (long long)g.nx * g.ny * g.nz;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < cells;
       t += (long long)gridDim.x * blockDim.x) {
    const int i = int(t % g.nx), j = int((t / g.nx) % g.ny), k = int(t / ((long long)g.nx * g.ny));
    C cu[3];
    curl_n2c_at<C>(g, th, i, j, k, inv, cu);
    const long long at = g.cell(i, j, k);
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const long long p = c * g.cells + at;
      const T value = T(C(1) * C(b[p]) + faraday * cu[c]);
      next[p] = value;
      if (!isfinite(value)) atomicAdd(invalid, 1u);
    }
  }
}

template <class T>
__global__ void __launch_bounds__(256) field_energy_kernel(Geom g, const T* __restrict__ e,
                                                           const T* __restrict__ b, double* partials) {
  __shared__ double scratch[2][8];
  const long long unique = (long long)g.nx * g.ny * g.nz;
  double we = 0, wb = 0;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < unique;
       t += (long long)gridDim.x * blockDim.x) {
    const int i = int(t % g.nx), j = int((t / g.nx) % g.ny), k = int(t / ((long long)g.nx * g.ny));
    const long long n = g.node(i, j, k), c = g.cell(i, j, k);
    const double ex = e[n], ey = e[g.nodes + n], ez = e[2 * g.nodes + n];
    const double bx = b[c], by = b[g.cells + c], bz = b[2 * g.cells + c];
    we += ex * ex + ey * ey + ez * ez;
    wb += bx * bx + by * by + bz * bz;
  }
  we = block_sum<256>(we, scratch[0]);
  wb = block_sum<256>(wb, scratch[1]);
  if (threadIdx.x == 0) {
    partials[blockIdx.x] = we;
    partials[gridDim.x + blockIdx.x] = wb;
  }
}

template <class Vel>
__global__ void __launch_bounds__(256) species_kernel(const Vel* __restrict__ u, const Vel* __restrict__ v,
                                                      const Vel* __restrict__ w, const double* __restrict__ q,
                                                      uint32_t count, double inverse_qom, double* partials) {
  __shared__ double scratch[5][8];
  double s[5] = {0, 0, 0, 0, 0};
  for (uint32_t n = blockIdx.x * blockDim.x + threadIdx.x; n < count; n += gridDim.x * blockDim.x) {
    const double weight = q[n], mass = weight * inverse_qom;
    const double vx = u[n], vy = v[n], vz = w[n];
    s[0] += 0.5 * mass * (vx * vx + vy * vy + vz * vz);
    s[1] += weight;
    s[2] += mass * vx;
    s[3] += mass * vy;
    s[4] += mass * vz;
  }
#pragma unroll
  for (int r = 0; r < 5; ++r) {
    const double total = block_sum<256>(s[r], scratch[r]);
    if (threadIdx.x == 0) partials[r * gridDim.x + blockIdx.x] = total;
  }
}

// One block per row: out[row] = sum of the row's `count` partials; rows at or
// above `filled` store zero (reduce_block_partials_kernel,
// device/block_reduction_device.hpp:23-44).
__global__ void __launch_bounds__(256) reduce_rows_kernel(const double* __restrict__ partials, double* out,
                                                          int row_stride, int count, int filled) {
  wait_for_predecessor();
  __shared__ double scratch[8];
  const int row = blockIdx.x;
  if (row >= filled) {
    if (threadIdx.x == 0) out[row] = 0;
    return;
  }
  double sum = 0;
  for (int i = threadIdx.x; i < count; i += blockDim.x) sum += partials[(long long)row * row_stride + i];
  sum = block_sum<256>(sum, scratch);
  if (threadIdx.x == 0) out[row] = sum;
}

template <class T>
__global__ void __launch_bounds__(256) copy_node_kernel(long long total, const T* __restrict__ in,
                                                        double* __restrict__ out) {
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x)
    out[t] = double(in[t]);
}

}  // namespace

cudaError_t launch_node_ghosts(const Geom& g, double* f, int components, cudaStream_t s, bool programmatic) {
  if (shell_count(g) >= (1LL << 31)) return cudaErrorInvalidValue;
  const dim3 blocks(grid_for(shell_count(g), 256), unsigned(components));
  count_launches(1);
  if (programmatic) return launch_programmatic(node_fill_kernel<double>, blocks, 256, 0, s, g, f);
  node_fill_kernel<double><<<blocks, 256, 0, s>>>(g, f);
  return cudaGetLastError();
}

cudaError_t launch_cell_ghosts(int precision, const Geom& g, void* f, cudaStream_t s) {
  const long long shell = 2 * ((long long)g.CX * g.CY + (long long)g.CX * g.nz + (long long)g.ny * g.nz);
  const unsigned blocks = grid_for(3 * shell, 256);
  if (precision == TPICB200_PRECISION_DOUBLE) cell_fill_kernel<double><<<blocks, 256, 0, s>>>(g, (double*)f);
  else cell_fill_kernel<float><<<blocks, 256, 0, s>>>(g, (float*)f);
  count_launches(1);
  return cudaGetLastError();
}

cudaError_t launch_cell_to_node(int precision, const Geom& g, const void* cellf, void* node, cudaStream_t s) {
  const unsigned blocks = grid_for(3 * g.interior, 256);
  if (precision == TPICB200_PRECISION_DOUBLE) {
    cell_to_node_kernel<double, double><<<blocks, 256, 0, s>>>(g, (const double*)cellf, (double*)node);
    node_fill_kernel<double><<<dim3(grid_for(shell_count(g), 256), 3), 256, 0, s>>>(g, (double*)node);
  } else {
    cell_to_node_kernel<float, float><<<blocks, 256, 0, s>>>(g, (const float*)cellf, (float*)node);
    node_fill_kernel<float><<<dim3(grid_for(shell_count(g), 256), 3), 256, 0, s>>>(g, (float*)node);
  }
  count_launches(2);
  return cudaGetLastError();
}

cudaError_t launch_rhs(int precision, const Geom& g, double delta, double kfac, const void* e,
                       const void* bcell, const void* j, double* rhs, cudaStream_t s, bool j_double) {
  const unsigned blocks = grid_for(g.interior, 256);
  if (precision == TPICB200_PRECISION_DOUBLE)
    rhs_kernel<double, double, double><<<blocks, 256, 0, s>>>(g, delta, kfac, (const double*)e,
                                                             (const double*)bcell, (const double*)j, rhs);
  else if (j_double)
    rhs_kernel<float, float, double><<<blocks, 256, 0, s>>>(g, float(delta), float(kfac), (const float*)e,
                                                           (const float*)bcell, (const double*)j, rhs);
  else
    rhs_kernel<float, float, float><<<blocks, 256, 0, s>>>(g, float(delta), float(kfac), (const float*)e,
                                                          (const float*)bcell, (const float*)j, rhs);
  count_launches(1);
  return cudaGetLastError();
}

// Energy-conserving smoothing, one pass (node_smoothing_kernel,
// ecsim/fields/node_smoothing_device.hpp:17-36, with the operator of
// ecsim/fields/node_smoothing.hpp:24-52): every interior node 0..n of the
// three components, from a double node field with filled ghosts into a
// double node field, in arithmetic C with each product and sum rounded on
// its own (no contraction) in the reference's order. Op 0 Face7: alpha *
// centre + beta * faces; op 1 Binomial27: (8 centre + 4 faces + 2 edges +
// corners) * (1/64). A nonfinite result counts in *invalid (when given), as
// the reference's kernel flags it (node_smoothing_device.hpp:30-36).
__device__ __forceinline__ float rn_mul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double rn_mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float rn_add(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ double rn_add(double a, double b) { return __dadd_rn(a, b); }

template <class C, int Op>
__global__ void __launch_bounds__(256) smooth_kernel(Geom g, C alpha, C beta, const double* __restrict__ src,
                                                     double* __restrict__ dst, uint32_t* invalid) {
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < 3 * g.interior;
       t += (long long)gridDim.x * blockDim.x) {
    const int c = int(t / g.interior);
    int i, j, k;
    interior_node_coordinates(g, t - c * g.interior, i, j, k);
    const double* f = src + c * g.nodes;
    auto v = [&](int a, int b, int d) { return C(f[g.node(a, b, d)]); };
    const C face = rn_add(rn_add(rn_add(rn_add(rn_add(v(i - 1, j, k), v(i + 1, j, k)), v(i, j - 1, k)),
                                        v(i, j + 1, k)), v(i, j, k - 1)), v(i, j, k + 1));
    C value;
    if constexpr (Op == 0) {
      value = rn_add(rn_mul(alpha, v(i, j, k)), rn_mul(beta, face));
    } else {
      C edge = rn_add(v(i - 1, j - 1, k), v(i + 1, j - 1, k));
      edge = rn_add(edge, v(i - 1, j + 1, k)); edge = rn_add(edge, v(i + 1, j + 1, k));
      edge = rn_add(edge, v(i - 1, j, k - 1)); edge = rn_add(edge, v(i + 1, j, k - 1));
      edge = rn_add(edge, v(i - 1, j, k + 1)); edge = rn_add(edge, v(i + 1, j, k + 1));
      edge = rn_add(edge, v(i, j - 1, k - 1)); edge = rn_add(edge, v(i, j + 1, k - 1));
      edge = rn_add(edge, v(i, j - 1, k + 1)); edge = rn_add(edge, v(i, j + 1, k + 1));
      C corner = rn_add(v(i - 1, j - 1, k - 1), v(i + 1, j - 1, k - 1));
      corner = rn_add(corner, v(i - 1, j + 1, k - 1)); corner = rn_add(corner, v(i + 1, j + 1, k - 1));
      corner = rn_add(corner, v(i - 1, j - 1, k + 1)); corner = rn_add(corner, v(i + 1, j - 1, k + 1));
      corner = rn_add(corner, v(i - 1, j + 1, k + 1)); corner = rn_add(corner, v(i + 1, j + 1, k + 1));
      const C sum = rn_add(rn_add(rn_add(rn_mul(C(8), v(i, j, k)), rn_mul(C(4), face)), rn_mul(C(2), edge)), corner);
      value = rn_mul(sum, C(1) / C(64));
    }
    dst[c * g.nodes + g.node(i, j, k)] = double(value);
    if (invalid && !isfinite(value)) atomicAdd(invalid, 1u);
  }
}

// S^n(src) into out with its ghosts filled (complete_smoothing,
// ecsim/maxwell/maxwell_device.hpp:455-487 on a periodic domain): src's
// ghosts must be filled; the passes alternate between out and tmp so that
// the last lands in out, with the ghosts refilled between passes. Neither
// out nor tmp may alias src. double_arithmetic selects the pass arithmetic
// (the reference's Arithmetic / Compute::Electric). invalid (may be null)
// counts nonfinite smoothed values.
cudaError_t launch_smooth(bool double_arithmetic, const Geom& g, int niter, int op, double alpha,
                          const double* src, double* out, double* tmp, uint32_t* invalid, cudaStream_t s) {
  if (niter <= 0 || src == out || src == tmp || out == tmp) return cudaErrorInvalidValue;
  const unsigned blocks = grid_for(3 * g.interior, 256);
  const double* from = src;
  for (int pass = 1; pass <= niter; ++pass) {
    double* to = (niter - pass) % 2 == 0 ? out : tmp;
    if (double_arithmetic) {
      const double beta = (1.0 - alpha) / 6.0;
      if (op == 0) smooth_kernel<double, 0><<<blocks, 256, 0, s>>>(g, alpha, beta, from, to, invalid);
      else smooth_kernel<double, 1><<<blocks, 256, 0, s>>>(g, alpha, beta, from, to, invalid);
    } else {
      const float a = float(alpha), beta = (1.0f - a) / 6.0f;
      if (op == 0) smooth_kernel<float, 0><<<blocks, 256, 0, s>>>(g, a, beta, from, to, invalid);
      else smooth_kernel<float, 1><<<blocks, 256, 0, s>>>(g, a, beta, from, to, invalid);
    }
    count_launches(1);
    launch_node_ghosts(g, to, 3, s);
    from = to;
  }
  return cudaGetLastError();
}

// A node field of float or double into double (every entry, ghosts included).
__global__ void __launch_bounds__(256) widen_kernel(const float* __restrict__ in, double* __restrict__ out,
                                                    long long n) {
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x)
    out[t] = double(in[t]);
}
cudaError_t launch_widen(int precision, const Geom& g, const void* in, double* out, cudaStream_t s) {
  const long long n = 3 * g.nodes;
  if (precision == TPICB200_PRECISION_DOUBLE)
    return cudaMemcpyAsync(out, in, size_t(n) * 8, cudaMemcpyDeviceToDevice, s);
  widen_kernel<<<grid_for(n, 256), 256, 0, s>>>((const float*)in, out, n);
  count_launches(1);
  return cudaGetLastError();
}

cudaError_t launch_field_advance(int precision, const Geom& g, double theta_value, double faraday,
                                 void* e, const void* bcell, const double* etheta, void* bnext,
                                 uint32_t* invalid, cudaStream_t s) {
  const bool copy = fabs(theta_value - 1.0) < 1e-10;
  const unsigned eb = grid_for(3 * g.interior, 256);
  const unsigned fb = grid_for((long long)g.nx * g.ny * g.nz, 256);
  if (precision == TPICB200_PRECISION_DOUBLE) {
    const double a = 1.0 / theta_value, b = -(1.0 - theta_value) / theta_value;
    e_update_kernel<double, double><<<eb, 256, 0, s>>>(g, a, b, copy, (double*)e, etheta, invalid);
    faraday_kernel<double, double><<<fb, 256, 0, s>>>(g, faraday, (const double*)bcell, etheta,
                                                     (double*)bnext, invalid);
  } else {
    const float th = float(theta_value);
    const float a = 1.0f / th, b = -(1.0f - th) / th;
    e_update_kernel<float, float><<<eb, 256, 0, s>>>(g, a, b, copy, (float*)e, etheta, invalid);
    faraday_kernel<float, float><<<fb, 256, 0, s>>>(g, float(faraday), (const float*)bcell, etheta,
                                                   (float*)bnext, invalid);
  }
  count_launches(2);
  return cudaGetLastError();
}

cudaError_t launch_field_energy(int precision, const Geom& g, const void* e, const void* bcell,
                                double* partials, int blocks, cudaStream_t s) {
  if (precision == TPICB200_PRECISION_DOUBLE)
    field_energy_kernel<double><<<blocks, 256, 0, s>>>(g, (const double*)e, (const double*)bcell, partials);
  else
    field_energy_kernel<float><<<blocks, 256, 0, s>>>(g, (const float*)e, (const float*)bcell, partials);
  count_launches(1);
  return cudaGetLastError();
}

cudaError_t launch_species_scalars(int precision, const tpicb200_particles* p, double qom,
                                   double* partials, int blocks, cudaStream_t s) {
  if (precision == TPICB200_PRECISION_DOUBLE)
    species_kernel<double><<<blocks, 256, 0, s>>>((const double*)p->u, (const double*)p->v,
                                                  (const double*)p->w, p->q, p->count, 1.0 / qom, partials);
  else
    species_kernel<float><<<blocks, 256, 0, s>>>((const float*)p->u, (const float*)p->v,
                                                 (const float*)p->w, p->q, p->count, 1.0 / qom, partials);
  count_launches(1);
  return cudaGetLastError();
}

cudaError_t launch_reduce_rows(const double* partials, double* out, int rows, int row_stride, int count,
                               int filled, cudaStream_t s, bool programmatic) {
  count_launches(1);
  if (programmatic)
    return launch_programmatic(reduce_rows_kernel, unsigned(rows), 256, 0, s, partials, out, row_stride, count,
                               filled);
  reduce_rows_kernel<<<rows, 256, 0, s>>>(partials, out, row_stride, count, filled);
  return cudaGetLastError();
}

cudaError_t launch_copy_node_field(const Geom& g, const void* in, int in_double, double* out, cudaStream_t s) {
  const long long total = 3 * g.nodes;
  if (in_double) copy_node_kernel<double><<<grid_for(total, 256), 256, 0, s>>>(total, (const double*)in, out);
  else copy_node_kernel<float><<<grid_for(total, 256), 256, 0, s>>>(total, (const float*)in, out);
  count_launches(1);
  return cudaGetLastError();
}

}  // namespace tpicb200
