// Implicit theta-scheme particle mover, one thread per record.
//
// Restates push_and_classify_particle (ecsim/particles/particle_mover_device.hpp:37-122)
// with the whole-domain periodic wrap of classify_particle_point
// (communication/particles/particle_boundaries.hpp:112-135). This file is
// compiled with -fmad=false: every multiply and add rounds on its own, as the
// reference's expressions evaluate under strict IEEE rules, so new fractions,
// velocities and cell keys are bit-identical to the CPU oracle.
//
// HBM-bound: per record it reads key (4 B), charge (8 B), three double
// fractions (24 B) and three velocities, and writes the fractions, the
// velocities and the key; the 48 field gathers hit L1/L2 because records are
// sorted by cell.
#include "kernels.cuh"

#include <climits>

namespace tpicb200 {
namespace {

template <class P>
struct MoverParams {
  typename P::VC beta, beta_over_c;
  double dt, inv[3];
};

template <class C, class F>
__device__ __forceinline__ C gather8(const F* __restrict__ f, long long base, const long long* off,
                                     const C w[8]) {
  C value = 0;
#pragma unroll
  for (int a = 0; a < 8; ++a) value += w[a] * C(__ldg(f + base + off[a]));
  return value;
}

template <class P>
__global__ void __launch_bounds__(256) mover_kernel(Geom g, MoverParams<P> mp,
    typename P::Pos* __restrict__ rx, typename P::Pos* __restrict__ ry,
    typename P::Pos* __restrict__ rz, typename P::Vel* __restrict__ u,
    typename P::Vel* __restrict__ v, typename P::Vel* __restrict__ w,
    const double* __restrict__ q, int32_t* __restrict__ key, uint32_t count,
    const double* __restrict__ theta, const typename P::Fld* __restrict__ bnode,
    uint32_t* __restrict__ invalid) {
  using C = typename P::VC;
  using Pos = typename P::Pos;
  using Vel = typename P::Vel;
  const long long nn = g.nodes;
  const long long off[8] = {0, 1, g.NX, g.NX + 1, (long long)g.NX * g.NY,
                            (long long)g.NX * g.NY + 1, (long long)g.NX * g.NY + g.NX,
                            (long long)g.NX * g.NY + g.NX + 1};
  for (uint32_t n = blockIdx.x * blockDim.x + threadIdx.x; n < count;
       n += gridDim.x * blockDim.x) {
    const int32_t k0 = key[n];
    const double charge = q[n];
    const Pos fx = rx[n], fy = ry[n], fz = rz[n];
    int ci, cj, ck;
    bool ok = k0 >= 0 && (long long)k0 < g.bins;
    if (ok) {
      g.decode(k0, ci, cj, ck);
      ok = g.interior_cell(ci, cj, ck) && isfinite(charge) && fx >= Pos(0) && fx < Pos(1) &&
           fy >= Pos(0) && fy < Pos(1) && fz >= Pos(0) && fz < Pos(1);
    }
    if (!ok) {
      atomicAdd(invalid, 1u);
      continue;
    }
    C wt[8];
    cic_weights<C>(C(fx), C(fy), C(fz), wt);
    const long long base = g.node(ci, cj, ck);
    const C bx = gather8<C>(bnode, base, off, wt);
    const C by = gather8<C>(bnode + nn, base, off, wt);
    const C bz = gather8<C>(bnode + 2 * nn, base, off, wt);
    const C ex = gather8<C>(theta, base, off, wt);
    const C ey = gather8<C>(theta + nn, base, off, wt);
    const C ez = gather8<C>(theta + 2 * nn, base, off, wt);
    const Response<C> r(bx, by, bz, mp.beta_over_c);
    const C uu = C(u[n]), vv = C(v[n]), ww = C(w[n]);
    C hx, hy, hz, ax, ay, az;
    r.apply(uu, vv, ww, hx, hy, hz);
    r.apply(ex, ey, ez, ax, ay, az);
    const C px = hx + mp.beta * ax, py = hy + mp.beta * ay, pz = hz + mp.beta * az;
    const Vel vel[3] = {Vel(C(2) * px - uu), Vel(C(2) * py - vv), Vel(C(2) * pz - ww)};
    long long cell[3] = {ci, cj, ck};
    Pos frac[3] = {fx, fy, fz};
    const int ext[3] = {g.nx, g.ny, g.nz};
#pragma unroll
    for (int axis = 0; axis < 3; ++axis) {
      if (!isfinite(vel[axis])) { ok = false; break; }
      const Pos displacement = Pos(mp.dt * double(vel[axis]) * mp.inv[axis]);
      const Pos moved = frac[axis] + displacement;
      const double shift = floor(double(moved));
      if (!(shift >= double(INT_MIN) && shift <= double(INT_MAX))) { ok = false; break; }
      cell[axis] += (long long)shift;
      frac[axis] = moved - Pos(shift);
      if (frac[axis] == Pos(1)) {  // a tiny negative crossing rounded up to the endpoint
        ++cell[axis];
        frac[axis] = Pos(0);
      }
    }
    if (!ok) {
      atomicAdd(invalid, 1u);
      continue;
    }
#pragma unroll
    for (int axis = 0; axis < 3; ++axis) {
      const long long e = ext[axis];
      if (cell[axis] < 0 || cell[axis] >= e) {
        const long long m = cell[axis] % e;
        cell[axis] = m < 0 ? m + e : m;
      }
    }
    key[n] = g.encode(int(cell[0]), int(cell[1]), int(cell[2]));
    rx[n] = frac[0]; ry[n] = frac[1]; rz[n] = frac[2];
    u[n] = vel[0]; v[n] = vel[1]; w[n] = vel[2];
  }
}

template <class P>
cudaError_t launch(const Geom& g, double qom, double dt, double c, tpicb200_particles* p,
                   const double* theta, const void* bnode, uint32_t* invalid, cudaStream_t s) {
  MoverParams<P> mp;
  const double beta = qom * dt / 2;  // prepare_particle_mover_parameters: double, converted once
  mp.beta = typename P::VC(beta);
  mp.beta_over_c = typename P::VC(beta / c);
  mp.dt = dt;
  for (int a = 0; a < 3; ++a) mp.inv[a] = 1.0 / (a == 0 ? g.dx : a == 1 ? g.dy : g.dz);
  if (p->count == 0) return cudaSuccess;
  const unsigned blocks = grid_for(p->count, 256, 148u * 8u);
  mover_kernel<P><<<blocks, 256, 0, s>>>(g, mp, (typename P::Pos*)p->rx, (typename P::Pos*)p->ry,
      (typename P::Pos*)p->rz, (typename P::Vel*)p->u, (typename P::Vel*)p->v,
      (typename P::Vel*)p->w, p->q, p->cell, p->count, theta,
      (const typename P::Fld*)bnode, invalid);
  count_launches(1);
  return cudaGetLastError();
}

}  // namespace

cudaError_t launch_mover(int precision, const Geom& g, double qom, double dt, double c,
                         tpicb200_particles* p, const double* theta, const void* bnode,
                         uint32_t* invalid, cudaStream_t s) {
  if (precision == TPICB200_PRECISION_DOUBLE)
    return launch<PDouble>(g, qom, dt, c, p, theta, bnode, invalid, s);
  return launch<PMixed>(g, qom, dt, c, p, theta, bnode, invalid, s);
}

}  // namespace tpicb200
