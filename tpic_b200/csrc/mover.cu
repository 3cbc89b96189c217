// Implicit theta-scheme particle mover, one thread per record. Ahead of the
// binned sort it also emits each record's direction code and the per-cell
// transfer counts (the sort then skips its own classification pass).
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
__device__ __forceinline__ C gather8(const F* __restrict__ f, long long base, const int* off,
                                     const C w[8]) {
  C value = 0;
#pragma unroll
  for (int a = 0; a < 8; ++a) value += w[a] * C(__ldg(f + base + off[a]));
  return value;
}

// Direction codes and transfer counts of a mover that feeds the binned sort.
struct MoveCodes {
  uint8_t* code;        // per record: direction code, 0xff when not a neighbour move
  uint32_t* transfer;   // [27][interior cells], added into
  uint32_t* fallback;   // raised when any record did not move to a neighbour
  long long cells;
};

// Resident CTAs per SM the mover is compiled for (register budget).
#ifndef TPICB200_MOVER_MIN_BLOCKS
#define TPICB200_MOVER_MIN_BLOCKS 4
#endif

template <class P, bool Coded>
__global__ void __launch_bounds__(256, TPICB200_MOVER_MIN_BLOCKS) mover_kernel(Geom g, MoverParams<P> mp,
    typename P::Pos* __restrict__ rx, typename P::Pos* __restrict__ ry,
    typename P::Pos* __restrict__ rz, typename P::Vel* __restrict__ u,
    typename P::Vel* __restrict__ v, typename P::Vel* __restrict__ w,
    const double* __restrict__ q, int32_t* __restrict__ key, uint32_t count,
    const double* __restrict__ theta, const typename P::Fld* __restrict__ bnode,
    uint32_t* __restrict__ invalid, MoveCodes mc) {
  using C = typename P::VC;
  using Pos = typename P::Pos;
  using Vel = typename P::Vel;
  const long long nn = g.nodes;
  // Corner offsets of the node box (an x-y plane of nodes is far below 2^31).
  const int plane = g.NX * g.NY;
  const int off[8] = {0, 1, g.NX, g.NX + 1, plane, plane + 1, plane + g.NX, plane + g.NX + 1};
  // Moves record n; returns its direction code (-1: invalid record, or a
  // move beyond the 27 neighbouring cells) and its old interior cell.
  auto move = [&](uint32_t n, long long& old_cell) -> int {
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
      return -1;
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
      return -1;
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
    old_cell = ci + (long long)g.nx * (cj + (long long)g.ny * ck);
    return Coded ? move_code(g, ci, cj, ck, int(cell[0]), int(cell[1]), int(cell[2])) : 0;
  };
  const int lane = threadIdx.x & 31;
  const uint32_t stride = gridDim.x * blockDim.x;
  // Warp-uniform loop: lane l of a warp takes record base + l.
  for (uint32_t base = blockIdx.x * blockDim.x + (threadIdx.x & ~31u); base < count; base += stride) {
    const uint32_t n = base + lane;
    long long old_cell = 0;
    const int d = n < count ? move(n, old_cell) : -1;
    if constexpr (Coded) {
      if (n < count) mc.code[n] = uint8_t(d < 0 ? 0xff : d);
      // Transfer counts: one atomic per run of consecutive lanes with the same
      // (old cell, direction); records are sorted by old cell, so a warp holds
      // few runs.
      const long long slot = d < 0 ? -1 : old_cell * 27 + d;
      const long long left = __shfl_up_sync(0xffffffffu, slot, 1);
      const unsigned heads = __ballot_sync(0xffffffffu, lane == 0 || slot != left);
      if (d >= 0 && ((heads >> lane) & 1u)) {
        const unsigned later = heads & ~((2u << lane) - 1u);
        const int next = later ? __ffs(later) - 1 : 32;
        atomicAdd(mc.transfer + d * mc.cells + old_cell, unsigned(next - lane));
      }
      if (__any_sync(0xffffffffu, n < count && d < 0) && lane == 0) atomicExch(mc.fallback, 1u);
    }
  }
}

template <class P>
cudaError_t launch(const Geom& g, double qom, double dt, double c, tpicb200_particles* p,
                   const double* theta, const void* bnode, uint32_t* invalid, const BinnedScratch* binned,
                   cudaStream_t s) {
  MoverParams<P> mp;
  const double beta = qom * dt / 2;  // prepare_particle_mover_parameters: double, converted once
  mp.beta = typename P::VC(beta);
  mp.beta_over_c = typename P::VC(beta / c);
  mp.dt = dt;
  for (int a = 0; a < 3; ++a) mp.inv[a] = 1.0 / (a == 0 ? g.dx : a == 1 ? g.dy : g.dz);
  if (p->count == 0) return cudaSuccess;
  const unsigned blocks = grid_for(p->count, 256, 148u * 8u);
  MoveCodes mc{nullptr, nullptr, nullptr, (long long)g.nx * g.ny * g.nz};
  auto kernel = mover_kernel<P, false>;
  if (binned) {
    mc.code = binned->code;
    mc.transfer = binned->transfer;
    mc.fallback = &binned->state->fallback;
    kernel = mover_kernel<P, true>;
  }
  kernel<<<blocks, 256, 0, s>>>(g, mp, (typename P::Pos*)p->rx, (typename P::Pos*)p->ry,
      (typename P::Pos*)p->rz, (typename P::Vel*)p->u, (typename P::Vel*)p->v,
      (typename P::Vel*)p->w, p->q, p->cell, p->count, theta,
      (const typename P::Fld*)bnode, invalid, mc);
  count_launches(1);
  return cudaGetLastError();
}

}  // namespace

cudaError_t launch_mover(int precision, const Geom& g, double qom, double dt, double c,
                         tpicb200_particles* p, const double* theta, const void* bnode,
                         uint32_t* invalid, const BinnedScratch* binned, cudaStream_t s) {
  if (precision == TPICB200_PRECISION_DOUBLE)
    return launch<PDouble>(g, qom, dt, c, p, theta, bnode, invalid, binned, s);
  return launch<PMixed>(g, qom, dt, c, p, theta, bnode, invalid, binned, s);
}

}  // namespace tpicb200
