// Gauss-law residual of the committed states (diagnostics/gauss_residual_device.hpp,
// docs/developer/gauss_diagnostic.md): a sample begun at state n stores per cell
// s = divC(E^n)/2 - c, with c = 4 pi times the 8-node mean of the charge density
// rho = sum(q W)/V of the state's records (the positions x^{n+1/2} of the
// staggered cycle), passed through the run's smoothing; finishing at state n+1
// gives r = s + divC(E^{n+1})/2. divC is the solver's node-to-cell divergence
// (ecsim/fields/node_cell_curl.hpp:129-141: the curl's edge differences,
// summed in the same order). Every quantity is FP64 (the reduction type of
// both precision profiles). On a fully periodic grid there is no wall: the
// dual volume of every node is the cell volume and the wall sum is zero.
//
// The sums of a sample (residual r^2, drift (r - r_first)^2, wall r^2, charge
// c^2) are block partials of a fixed grid, added in a fixed order: the sums
// of the same inputs are reproducible. The charge itself is deposited with
// FP64 atomics (any order), as TPIC's.
#include "kernels.cuh"

#include <cmath>

namespace tpicb200 {
namespace {

constexpr int kGaussThreads = 256;
constexpr int kGaussBlocks = 4 * 148;  // partials per sum
constexpr double kPi = 3.14159265358979323846;

__device__ __forceinline__ void block_partials(double (&v)[3], int count, double* partials) {
  __shared__ double red[3][kGaussThreads / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int c = 0; c < count; ++c) {
    double x = v[c];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
    if (lane == 0) red[c][warp] = x;
  }
  __syncthreads();
  if (threadIdx.x < count) {
    double sum = 0.0;
    for (int w = 0; w < kGaussThreads / 32; ++w) sum += red[threadIdx.x][w];
    partials[threadIdx.x * kGaussBlocks + blockIdx.x] = sum;
  }
}

// h = divC(E)/2 per cell; finish: r = stash + h into residual and the sums of
// r^2 and of the drift (first = r on the first finished sample); begin:
// stash = h, after the finish has read it.
template <class F>
__global__ void __launch_bounds__(kGaussThreads) gauss_field_kernel(Geom g, const F* __restrict__ e,
                                                                   double* __restrict__ stash,
                                                                   double* __restrict__ first,
                                                                   double* __restrict__ residual, int begin,
                                                                   int finish, int set_first, double* partials) {
  const uint32_t nx = uint32_t(g.nx), ny = uint32_t(g.ny);
  const uint32_t cells = nx * ny * uint32_t(g.nz);
  const long long nn = g.nodes;
  double v[3] = {0.0, 0.0, 0.0};
  for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < cells; t += gridDim.x * blockDim.x) {
    const int i = int(t % nx), j = int((t / nx) % ny), k = int(t / (nx * ny));
    // The cell's corner samples: base, x, y, z, xy, xz, yz, xyz.
    auto samples = [&](int c, double (&q)[8]) {
      const F* f = e + c * nn;
      q[0] = double(f[g.node(i, j, k)]);
      q[1] = double(f[g.node(i + 1, j, k)]);
      q[2] = double(f[g.node(i, j + 1, k)]);
      q[3] = double(f[g.node(i, j, k + 1)]);
      q[4] = double(f[g.node(i + 1, j + 1, k)]);
      q[5] = double(f[g.node(i + 1, j, k + 1)]);
      q[6] = double(f[g.node(i, j + 1, k + 1)]);
      q[7] = double(f[g.node(i + 1, j + 1, k + 1)]);
    };
    double q[8];
    samples(0, q);
    const double dx = 0.25 * g.inv[0] * ((((q[1] - q[0]) + (q[5] - q[3])) + (q[4] - q[2])) + (q[7] - q[6]));
    samples(1, q);
    const double dy = 0.25 * g.inv[1] * ((((q[2] - q[0]) + (q[6] - q[3])) + (q[4] - q[1])) + (q[7] - q[5]));
    samples(2, q);
    const double dz = 0.25 * g.inv[2] * ((((q[3] - q[0]) + (q[5] - q[1])) + (q[6] - q[2])) + (q[7] - q[4]));
    const double h = 0.5 * ((dx + dy) + dz);
    if (finish) {
      const double r = stash[t] + h;
      residual[t] = r;
      v[0] += r * r;
      if (set_first) {
        first[t] = r;
      } else {
        const double drift = r - first[t];
        v[1] += drift * drift;
      }
    }
    if (begin) stash[t] = h;
  }
  if (finish) block_partials(v, 3, partials);
}

// rho of the unique nodes into component 0 of a node field (ghosts and end
// nodes the periodic copies), components 1 and 2 zero.
__global__ void __launch_bounds__(kGaussThreads) gauss_expand_kernel(Geom g, const double* __restrict__ unique,
                                                                    double* __restrict__ field) {
  const long long nn = g.nodes;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < nn;
       t += (long long)gridDim.x * blockDim.x) {
    const int NX = g.NX, NY = g.NY;
    const int i = int(t % NX) - 1, j = int((t / NX) % NY) - 1, k = int(t / ((long long)NX * NY)) - 1;
    const int ui = wrap_index(i, g.nx), uj = wrap_index(j, g.ny), uk = wrap_index(k, g.nz);
    field[t] = unique[ui + (long long)g.nx * (uj + (long long)g.ny * uk)];
    field[nn + t] = 0.0;
    field[2 * nn + t] = 0.0;
  }
}

// c = 4 pi times the 8-node mean of the charge density (component 0 of a
// node field), stash -= c, and the sum of c^2.
__global__ void __launch_bounds__(kGaussThreads) gauss_charge_kernel(Geom g, const double* __restrict__ charge,
                                                                    double* __restrict__ stash, double* partials) {
  const uint32_t nx = uint32_t(g.nx), ny = uint32_t(g.ny);
  const uint32_t cells = nx * ny * uint32_t(g.nz);
  double v[3] = {0.0, 0.0, 0.0};
  for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < cells; t += gridDim.x * blockDim.x) {
    const int i = int(t % nx), j = int((t / nx) % ny), k = int(t / (nx * ny));
    const double c = kPi / 2 *
                     (((((((charge[g.node(i, j, k)] + charge[g.node(i + 1, j, k)]) + charge[g.node(i, j + 1, k)]) +
                          charge[g.node(i + 1, j + 1, k)]) +
                         charge[g.node(i, j, k + 1)]) +
                        charge[g.node(i + 1, j, k + 1)]) +
                       charge[g.node(i, j + 1, k + 1)]) +
                      charge[g.node(i + 1, j + 1, k + 1)]);
    stash[t] -= c;
    v[0] += c * c;
  }
  block_partials(v, 1, partials);
}

// sums[offset + c] = the partials of sum c in block order.
__global__ void gauss_sum_kernel(const double* __restrict__ partials, int count, double* sums, int offset) {
  if (threadIdx.x >= count) return;
  double sum = 0.0;
  for (int b = 0; b < kGaussBlocks; ++b) sum += partials[threadIdx.x * kGaussBlocks + b];
  sums[offset + threadIdx.x] = sum;
}

int launch_failure(const char* what, cudaError_t e) {
  return report_error(TPICB200_BACKEND_FAILURE, std::string(what) + ": " + cudaGetErrorString(e));
}

}  // namespace
}  // namespace tpicb200

using namespace tpicb200;

extern "C" {

int tpicb200_gauss_field(tpicb200_context* ctx, const void* e, double* stash, double* first, double* residual,
                         int begin, int finish, int set_first, double* sums, tpicb200_stream stream) {
  if (!ctx) return report_error(TPICB200_INVALID_ARGUMENT, "null context");
  if (!e || !stash || (finish && (!first || !residual || !sums)))
    return report_error(TPICB200_INVALID_ARGUMENT, "gauss field: null buffer");
  if (!begin && !finish) return report_error(TPICB200_INVALID_ARGUMENT, "gauss field: neither begin nor finish");
  const Geom& g = context_geom(ctx);
  cudaStream_t s = (cudaStream_t)stream;
  double* partials = nullptr;
  cudaError_t err = cudaSuccess;
  if (finish && (err = cudaMallocAsync((void**)&partials, 3 * kGaussBlocks * sizeof(double), s)) != cudaSuccess)
    return launch_failure("gauss field scratch", err);
  if (context_options(ctx).precision == TPICB200_PRECISION_DOUBLE)
    gauss_field_kernel<double><<<kGaussBlocks, kGaussThreads, 0, s>>>(g, (const double*)e, stash, first, residual,
                                                                     begin, finish, set_first, partials);
  else
    gauss_field_kernel<float><<<kGaussBlocks, kGaussThreads, 0, s>>>(g, (const float*)e, stash, first, residual,
                                                                    begin, finish, set_first, partials);
  count_launches(1);
  if (finish) {
    gauss_sum_kernel<<<1, 32, 0, s>>>(partials, 2, sums, 0);
    count_launches(1);
    if ((err = cudaMemsetAsync(sums + 2, 0, sizeof(double), s)) == cudaSuccess) err = cudaFreeAsync(partials, s);
    if (err != cudaSuccess) return launch_failure("gauss field sums", err);
  }
  if ((err = cudaGetLastError()) != cudaSuccess) return launch_failure("gauss field launch failed", err);
  return TPICB200_SUCCESS;
}

int tpicb200_gauss_charge(tpicb200_context* ctx, int ns, const tpicb200_particles* species, double* stash,
                          double* sums, tpicb200_stream stream) {
  if (!ctx) return report_error(TPICB200_INVALID_ARGUMENT, "null context");
  if (ns < 0 || ns > TPICB200_MAX_SPECIES || (ns > 0 && !species) || !stash || !sums)
    return report_error(TPICB200_INVALID_ARGUMENT, "gauss charge: bad arguments");
  const Geom& g = context_geom(ctx);
  const tpicb200_options& opt = context_options(ctx);
  cudaStream_t s = (cudaStream_t)stream;
  const long long unique = (long long)g.nx * g.ny * g.nz;
  const bool smooth = opt.smooth_iterations > 0;
  // unique rho, the node field (and two more for the smoothing passes), partials.
  const size_t words = size_t(unique) + size_t(3 * g.nodes) * (smooth ? 3 : 1) + size_t(kGaussBlocks) * 3;
  double* scratch = nullptr;
  cudaError_t err = cudaMallocAsync((void**)&scratch, words * sizeof(double), s);
  if (err != cudaSuccess) return launch_failure("gauss charge scratch", err);
  double* rho = scratch;
  double* field = rho + unique;
  double* partials = field + 3 * g.nodes * (smooth ? 3 : 1);
  err = cudaMemsetAsync(rho, 0, size_t(unique) * sizeof(double), s);
  for (int sp = 0; sp < ns && err == cudaSuccess; ++sp)
    err = launch_output_moments(opt.precision, g, species[sp], 1.0, 1.0, rho, nullptr, nullptr,
                                context_invalid(ctx), s);
  if (err != cudaSuccess) {
    cudaFreeAsync(scratch, s);
    return launch_failure("gauss charge deposition", err);
  }
  gauss_expand_kernel<<<grid_for(g.nodes, kGaussThreads), kGaussThreads, 0, s>>>(g, rho, field);
  count_launches(1);
  const double* charge = field;
  if (smooth) {
    // The run's smoothing in FP64 arithmetic, the last pass into the second field.
    err = launch_smooth(true, g, opt.smooth_iterations, opt.smooth_operator, opt.smooth_alpha, field,
                        field + 3 * g.nodes, field + 6 * g.nodes, nullptr, s);
    charge = field + 3 * g.nodes;
  }
  if (err == cudaSuccess) {
    gauss_charge_kernel<<<kGaussBlocks, kGaussThreads, 0, s>>>(g, charge, stash, partials);
    gauss_sum_kernel<<<1, 32, 0, s>>>(partials, 1, sums, 3);
    count_launches(2);
    err = cudaGetLastError();
  }
  const cudaError_t freed = cudaFreeAsync(scratch, s);
  if (err == cudaSuccess) err = freed;
  if (err != cudaSuccess) return launch_failure("gauss charge", err);
  return TPICB200_SUCCESS;
}

}  // extern "C"
