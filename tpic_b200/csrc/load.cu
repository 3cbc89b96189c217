// Device particle loading and velocity centring.
//
// One thread per record, grid-stride: TPIC's dense load order
// (initialization/particles/particle_loading_device.hpp:75-160) with a
// counter-based Philox-4x32-10 stream (Salmon, Moraes, Dror, Shaw, SC'11), so
// that any chunk [first, first+count) of a species is loaded independently
// and the records equal the host generator's (positions, keys and ids bit for
// bit; velocities and charges to the last bits of log/cos/sin/cosh). The
// position arithmetic is compiled without FMA contraction (-fmad=false).
//
// Centring (initialization/particles/particle_centering_device.hpp:36-100):
// one pass removes the drift and writes per-block FP64 sums of q, q u, q v,
// q w; reduce_rows sums the partials in a fixed order; a second pass
// subtracts the charge-weighted mean and restores the drift.
#include "cases.cuh"
#include "kernels.cuh"

namespace tpicb200 {
namespace {

constexpr uint32_t kM0 = 0xD2511F53u, kM1 = 0xCD9E8D57u;
constexpr uint32_t kW0 = 0x9E3779B9u, kW1 = 0xBB67AE85u;
constexpr double kTwoPi = 6.283185307179586;  // 2 pi in double (the product 2.0 * pi)

__device__ __forceinline__ void philox(uint32_t (&c)[4], uint32_t k0, uint32_t k1) {
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    const uint32_t hi0 = __umulhi(kM0, c[0]), lo0 = kM0 * c[0];
    const uint32_t hi1 = __umulhi(kM1, c[2]), lo1 = kM1 * c[2];
    const uint32_t n0 = hi1 ^ c[1] ^ k0, n2 = hi0 ^ c[3] ^ k1;
    c[0] = n0;
    c[1] = lo1;
    c[2] = n2;
    c[3] = lo0;
    k0 += kW0;
    k1 += kW1;
  }
}

__device__ __forceinline__ double uniform(uint32_t r) { return double(r) * 0x1p-32 + 0x1p-33; }

template <class V> __device__ __forceinline__ V narrow(double v);
template <> __device__ __forceinline__ double narrow<double>(double v) { return v; }
template <> __device__ __forceinline__ float narrow<float>(double v) { return __double2float_rn(v); }

template <class V>
__global__ void __launch_bounds__(256) load_species_kernel(LoadPlan plan, CaseProfile prof, Geom g,
                                                           tpicb200_particles p, uint32_t* invalid) {
  double* rx = (double*)p.rx;
  double* ry = (double*)p.ry;
  double* rz = (double*)p.rz;
  V* u = (V*)p.u;
  V* v = (V*)p.v;
  V* w = (V*)p.w;
  uint32_t bad = 0;
  for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < p.count; t += gridDim.x * blockDim.x) {
    const uint64_t n = plan.first + t;
    uint32_t a[4] = {uint32_t(n), uint32_t(n >> 32), plan.species, 0u};
    uint32_t b[4] = {uint32_t(n), uint32_t(n >> 32), plan.species, 1u};
    philox(a, plan.key0, plan.key1);
    philox(b, plan.key0, plan.key1);
    const uint64_t cellno = n / plan.ppc;
    const uint32_t sub = uint32_t(n - cellno * plan.ppc);
    const uint32_t sub_idx[3] = {sub % uint32_t(plan.npc[0]), (sub / uint32_t(plan.npc[0])) % uint32_t(plan.npc[1]),
                                 sub / uint32_t(plan.npc[0] * plan.npc[1])};
    int cell[3] = {int(cellno % uint64_t(g.nx)), int((cellno / uint64_t(g.nx)) % uint64_t(g.ny)),
                   int(cellno / (uint64_t(g.nx) * uint64_t(g.ny)))};
    const int extent[3] = {g.nx, g.ny, g.nz};
    double f[3];
#pragma unroll
    for (int axis = 0; axis < 3; ++axis) {
      const double off = plan.quiet ? 0.5 : uniform(a[axis]);
      double fr = (double(sub_idx[axis]) + off) * plan.inverse_npc[axis];
      if (fr >= 1.0) {
        fr = 0.0;
        cell[axis] += 1;
      }
      if (cell[axis] >= extent[axis]) cell[axis] -= extent[axis];
      f[axis] = fr;
    }
    const double u1 = uniform(a[3]), u2 = uniform(b[0]), u3 = uniform(b[1]), u4 = uniform(b[2]);
    const double r12 = sqrt(-2.0 * log(u1));
    const double r34 = sqrt(-2.0 * log(u3));
    const double normal[3] = {r12 * cos(kTwoPi * u2), r12 * sin(kTwoPi * u2), r34 * cos(kTwoPi * u4)};
    const double x = (cell[0] + f[0]) * g.dx;
    const double y = (cell[1] + f[1]) * g.dy;
    double dens, mult, drift[3];
    prof.evaluate(x, y, cell[1], dens, mult, drift);
    const double q = (plan.q_factor * dens) * mult;
    const V vel[3] = {narrow<V>(drift[0] + plan.vth[0] * normal[0]), narrow<V>(drift[1] + plan.vth[1] * normal[1]),
                      narrow<V>(drift[2] + plan.vth[2] * normal[2])};
    if (!isfinite(double(vel[0])) || !isfinite(double(vel[1])) || !isfinite(double(vel[2])) || !isfinite(q)) ++bad;
    rx[t] = f[0];
    ry[t] = f[1];
    rz[t] = f[2];
    u[t] = vel[0];
    v[t] = vel[1];
    w[t] = vel[2];
    p.q[t] = q;
    p.cell[t] = g.encode(cell[0], cell[1], cell[2]);
    if (p.id) p.id[t] = n;
  }
  bad = warp_sum(bad);
  if (bad && (threadIdx.x & 31) == 0) atomicAdd(invalid, bad);
}

// The drift a record was loaded with: the profile at its stored position.
__device__ __forceinline__ void loaded_drift(const CaseProfile& prof, const Geom& g, int32_t key, double ry,
                                             double drift[3]) {
  int i, j, k;
  g.decode(key, i, j, k);
  prof.drift_at((j + ry) * g.dy, drift);
}

// Removes the loaded drift and writes the block's sums of q, q u, q v, q w
// (rows of `partials`, stride gridDim.x).
template <class V>
__global__ void __launch_bounds__(256) center_remove_kernel(CaseProfile prof, Geom g, tpicb200_particles p,
                                                            double* partials, uint32_t* invalid) {
  __shared__ double scratch[8];
  V* vel[3] = {(V*)p.u, (V*)p.v, (V*)p.w};
  const double* ry = (const double*)p.ry;
  double sums[4] = {0, 0, 0, 0};
  uint32_t bad = 0;
  for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < p.count; t += gridDim.x * blockDim.x) {
    double drift[3];
    loaded_drift(prof, g, p.cell[t], ry[t], drift);
    const double q = p.q[t];
    sums[0] += q;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      const V rest = narrow<V>((double(vel[a][t]) - 0.0) + -1.0 * drift[a]);
      if (!isfinite(double(rest))) ++bad;
      vel[a][t] = rest;
      sums[a + 1] += q * double(rest);
    }
  }
#pragma unroll
  for (int r = 0; r < 4; ++r) {
    const double s = block_sum<256>(sums[r], scratch);
    if (threadIdx.x == 0) partials[r * gridDim.x + blockIdx.x] = s;
  }
  bad = warp_sum(bad);
  if (bad && (threadIdx.x & 31) == 0) atomicAdd(invalid, bad);
}

// Subtracts the charge-weighted mean sums[1..3] / sums[0] and restores the drift.
template <class V>
__global__ void __launch_bounds__(256) center_restore_kernel(CaseProfile prof, Geom g, tpicb200_particles p,
                                                             const double* sums, uint32_t* invalid) {
  double mean[3] = {0.0, 0.0, 0.0};
  bool finite = isfinite(sums[0]) && isfinite(sums[1]) && isfinite(sums[2]) && isfinite(sums[3]);
  if (finite && sums[0] != 0.0)
    for (int a = 0; a < 3; ++a) mean[a] = sums[a + 1] / sums[0];
  finite = finite && isfinite(mean[0]) && isfinite(mean[1]) && isfinite(mean[2]);
  if (!finite) {
    if (blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(invalid, 1u);
    return;
  }
  V* vel[3] = {(V*)p.u, (V*)p.v, (V*)p.w};
  const double* ry = (const double*)p.ry;
  uint32_t bad = 0;
  for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < p.count; t += gridDim.x * blockDim.x) {
    double drift[3];
    loaded_drift(prof, g, p.cell[t], ry[t], drift);
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      const V next = narrow<V>((double(vel[a][t]) - mean[a]) + 1.0 * drift[a]);
      if (!isfinite(double(next))) ++bad;
      else vel[a][t] = next;
    }
  }
  bad = warp_sum(bad);
  if (bad && (threadIdx.x & 31) == 0) atomicAdd(invalid, bad);
}

int load_blocks(uint32_t count) {
  const uint32_t blocks = (count + 255u) / 256u;
  return int(blocks < 148u * 16u ? (blocks ? blocks : 1u) : 148u * 16u);
}

}  // namespace

cudaError_t launch_load_species(int precision, const Geom& g, const LoadPlan& plan, const CaseProfile& prof,
                                tpicb200_particles* p, uint32_t* invalid, cudaStream_t s) {
  if (p->count == 0) return cudaSuccess;
  const int blocks = load_blocks(p->count);
  if (precision == TPICB200_PRECISION_DOUBLE)
    load_species_kernel<double><<<blocks, 256, 0, s>>>(plan, prof, g, *p, invalid);
  else
    load_species_kernel<float><<<blocks, 256, 0, s>>>(plan, prof, g, *p, invalid);
  count_launches(1);
  return cudaGetLastError();
}

cudaError_t launch_center_velocities(int precision, const Geom& g, const CaseProfile& prof, tpicb200_particles* p,
                                     double* partials, int blocks, double* sums, uint32_t* invalid,
                                     cudaStream_t s) {
  if (precision == TPICB200_PRECISION_DOUBLE)
    center_remove_kernel<double><<<blocks, 256, 0, s>>>(prof, g, *p, partials, invalid);
  else
    center_remove_kernel<float><<<blocks, 256, 0, s>>>(prof, g, *p, partials, invalid);
  if (cudaError_t e = cudaGetLastError()) return e;
  if (cudaError_t e = launch_reduce_rows(partials, sums, 4, blocks, blocks, 4, s)) return e;
  if (precision == TPICB200_PRECISION_DOUBLE)
    center_restore_kernel<double><<<blocks, 256, 0, s>>>(prof, g, *p, sums, invalid);
  else
    center_restore_kernel<float><<<blocks, 256, 0, s>>>(prof, g, *p, sums, invalid);
  count_launches(2);
  return cudaGetLastError();
}

}  // namespace tpicb200
