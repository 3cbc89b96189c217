// Discrete adjoint of the ECSIM cycle: the transposes of the mover, the
// current and mass deposition, the field solve and the field advance.
//
// TPIC has no adjoint; these kernels transpose the library's own forward
// cycle, which follows TPIC's:
//   deposit   J_g = sum_p (q/V) W_a(x_p) R_p v_p          (current_deposition_device.hpp:167-264)
//             (M U)_g = sum_p (beta/c) q W_a R_p U(x_p)    (mass_matrix_scalar_device.hpp:121-232)
//   solve     A E_theta = E + delta C2N(B) - k J, A = I + delta^2 C2N N2C + (k/V) M
//   mover     v' = 2 R (v + beta E_theta(x)) - v, x' = x + dt v' / dx   (particle_mover_device.hpp:35-122)
//   advance   E' = E_theta/theta - (1-theta)/theta E, B' = B - c dt N2C(E_theta)
// with R = R(omega) the particle response (particle_response.hpp:16-42),
// omega = (beta/c) B(x), B at the nodes the cell-to-node average of B.
//
// The transpose of a gather at the particle positions is a scatter, so the
// backward of the mover scatters into E_theta and B, and the backward of the
// deposition gathers the gradient fields at the particles. Each thread takes
// one record; a warp's lanes reduce their corner contributions over runs of
// equal cell keys (the records are sorted by cell) before one lane per run
// adds them into the unique nodes with FP64 atomics. Adjoint arithmetic is
// FP64 in both precision modes (the forward values are read in their stored
// types). Particle adjoints are indexed by record id.
#include "kernels.cuh"
#include "stencils.cuh"

#include <cmath>

namespace tpicb200 {
namespace {

constexpr int kAdjointThreads = 256;
constexpr unsigned kFull = 0xffffffffu;

struct AdjointConstants {
  double beta, boc, dt, inv[3], inv_volume;
};

// Gradient fields a record's adjoint reads. jbar: the gradient of J (times
// jscale); mleft/mright: the mass term mscale * <mleft, M mright> (M applied
// without its 1/V row scale).
struct AdjointFields {
  const double* theta;
  const void* bnode;
  const double* jbar;
  double jscale;
  const double* mleft;
  const double* mright;
  double mscale;
};

struct AdjointRecords {
  const double* rx;
  const double* ry;
  const double* rz;
  const void* u;
  const void* v;
  const void* w;
  const double* q;
  const int32_t* cell;
  const uint64_t* id;
  uint32_t count, nid;
  double* xbar;  // [3][nid]
  double* vbar;  // [3][nid]
  double* qbar;  // [nid]
};

// A record's cell and CIC factors. Corner a of the cell has offset
// (a&1, a>>1&1, a>>2&1); its node in a consistent field (duplicates hold the
// unique values) and the unique node it scatters into are formed on the fly.
struct Loaded {
  bool ok;
  int32_t key;
  long long pid;
  int i, j, k;
  long long base;           // node (i, j, k)
  double X[2], Y[2], Z[2];  // per-axis CIC factors (1 - f, f)
  double v[3];
  __device__ __forceinline__ long long node(const Geom& g, int a) const {
    return base + (a & 1) + (long long)g.NX * (((a >> 1) & 1) + (long long)g.NY * ((a >> 2) & 1));
  }
  __device__ __forceinline__ long long unique(const Geom& g, int a) const {
    const int ci = i + (a & 1), cj = j + ((a >> 1) & 1), ck = k + ((a >> 2) & 1);
    return g.node(ci == g.nx ? 0 : ci, cj == g.ny ? 0 : cj, ck == g.nz ? 0 : ck);
  }
  // The (wx*wy)*wz grouping of cic_weights.
  __device__ __forceinline__ double weight(int a) const { return X[a & 1] * Y[(a >> 1) & 1] * Z[(a >> 2) & 1]; }
  __device__ __forceinline__ void weight_gradient(int a, double d[3]) const {
    const int bx = a & 1, by = (a >> 1) & 1, bz = (a >> 2) & 1;
    d[0] = (bx ? 1.0 : -1.0) * Y[by] * Z[bz];
    d[1] = X[bx] * (by ? 1.0 : -1.0) * Z[bz];
    d[2] = X[bx] * Y[by] * (bz ? 1.0 : -1.0);
  }
};

template <class F>
__device__ __forceinline__ void gather3(const Geom& g, const F* __restrict__ f, const Loaded& L, double out[3]) {
  out[0] = out[1] = out[2] = 0;
#pragma unroll
  for (int a = 0; a < 8; ++a) {
    const long long n = L.node(g, a);
    const double w = L.weight(a);
    out[0] += w * double(f[n]);
    out[1] += w * double(f[g.nodes + n]);
    out[2] += w * double(f[2 * g.nodes + n]);
  }
}

// sum_a dW_a/dx_axis (f_a . gv) into out[axis].
template <class F>
__device__ __forceinline__ void position_term(const Geom& g, const F* __restrict__ f, const Loaded& L,
                                              const double gv[3], double out[3]) {
#pragma unroll
  for (int a = 0; a < 8; ++a) {
    const long long n = L.node(g, a);
    const double d = double(f[n]) * gv[0] + double(f[g.nodes + n]) * gv[1] + double(f[2 * g.nodes + n]) * gv[2];
    double dw[3];
    L.weight_gradient(a, dw);
    out[0] += dw[0] * d;
    out[1] += dw[1] * d;
    out[2] += dw[2] * d;
  }
}

__device__ __forceinline__ void transpose_apply(const double r[9], const double x[3], double out[3]) {
  out[0] = r[0] * x[0] + r[3] * x[1] + r[6] * x[2];
  out[1] = r[1] * x[0] + r[4] * x[1] + r[7] * x[2];
  out[2] = r[2] * x[0] + r[5] * x[1] + r[8] * x[2];
}

// d/d omega of sum_ij ab_ij R_ij(omega): R = (I + omega omega^T + K) / D,
// D = 1 + |omega|^2, K antisymmetric (K_01 = wz, K_02 = -wy, K_12 = wx).
__device__ __forceinline__ void response_gradient(const double om[3], const double r[9], const double ab[9],
                                                  double out[3]) {
  const double inv_d = 1.0 / (1.0 + om[0] * om[0] + om[1] * om[1] + om[2] * om[2]);
  double ar = 0;
#pragma unroll
  for (int e = 0; e < 9; ++e) ar += ab[e] * r[e];
  const double kk[3] = {ab[5] - ab[7], ab[6] - ab[2], ab[1] - ab[3]};
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const double sym = (ab[3 * c] + ab[c]) * om[0] + (ab[3 * c + 1] + ab[3 + c]) * om[1] +
                       (ab[3 * c + 2] + ab[6 + c]) * om[2];
    out[c] = (sym + kk[c]) * inv_d - 2.0 * om[c] * ar * inv_d;
  }
}

// Adds w_a * val (the 8 corners of this lane's record) into the unique nodes
// of `field`. A run is a maximal group of consecutive lanes with equal keys
// (the records are sorted by cell, so a run is usually a cell's records in
// this warp); per corner, each lane sums the lanes after it within its run
// and the first lane of the run adds the run's total. Every lane of the warp
// calls it; inactive lanes pass a key no other lane has.
__device__ __forceinline__ void warp_scatter(const Geom& g, double* __restrict__ field, const Loaded& L,
                                             const double val[3]) {
  const unsigned lane = threadIdx.x & 31u;
  const int32_t before = __shfl_up_sync(kFull, L.key, 1);
  const bool head = lane == 0 || before != L.key;
  const unsigned heads = __ballot_sync(kFull, head);
  const unsigned later = heads & ~((2u << lane) - 1u);  // run heads after this lane
  const unsigned end = later ? unsigned(__ffs(later) - 1) : 32u;
#pragma unroll
  for (int a = 0; a < 8; ++a) {
    const double w = L.ok ? L.weight(a) : 0.0;
    double part[3] = {w * val[0], w * val[1], w * val[2]};
#pragma unroll
    for (unsigned off = 1; off < 32; off <<= 1) {
      const bool add = lane + off < end;
#pragma unroll
      for (int comp = 0; comp < 3; ++comp) {
        const double o = __shfl_down_sync(kFull, part[comp], off);
        if (add) part[comp] += o;
      }
    }
    if (L.ok && head) {
      const long long u = L.unique(g, a);
#pragma unroll
      for (int comp = 0; comp < 3; ++comp) atomicAdd(field + comp * g.nodes + u, part[comp]);
    }
  }
}

template <class P>
__device__ __forceinline__ void load_record(const Geom& g, const AdjointRecords& r, uint32_t n, bool active,
                                            Loaded& L) {
  using Vel = typename P::Vel;
  L.ok = false;
  L.key = -1 - int32_t(threadIdx.x & 31u);
  L.pid = 0;
  L.i = L.j = L.k = 0;
  L.base = 0;
  L.X[0] = L.X[1] = L.Y[0] = L.Y[1] = L.Z[0] = L.Z[1] = 0;
  L.v[0] = L.v[1] = L.v[2] = 0;
  if (!active) return;
  const int32_t key = r.cell[n];
  if (key < 0 || key >= g.bins) return;
  int i, j, k;
  g.decode(key, i, j, k);
  const uint64_t id = r.id[n];
  if (!g.interior_cell(i, j, k) || id >= r.nid) return;
  const double fx = r.rx[n], fy = r.ry[n], fz = r.rz[n];
  if (!(fx >= 0 && fx < 1 && fy >= 0 && fy < 1 && fz >= 0 && fz < 1)) return;
  L.v[0] = double(((const Vel*)r.u)[n]);
  L.v[1] = double(((const Vel*)r.v)[n]);
  L.v[2] = double(((const Vel*)r.w)[n]);
  L.ok = true;
  L.key = key;
  L.pid = (long long)id;
  L.i = i; L.j = j; L.k = k;
  L.base = g.node(i, j, k);
  L.X[0] = 1 - fx; L.X[1] = fx;
  L.Y[0] = 1 - fy; L.Y[1] = fy;
  L.Z[0] = 1 - fz; L.Z[1] = fz;
}

// The mover's E_theta gradient W_a beta R^T (2 (v_bar' + dt x_bar' / dx)),
// scattered into the unique nodes of etheta_bar (the pass before the
// adjoint solve; the record adjoints are read, not written).
template <class P>
__global__ void __launch_bounds__(kAdjointThreads) adjoint_theta_scatter_kernel(Geom g, AdjointConstants k,
                                                                               AdjointRecords r, const void* bnode,
                                                                               double* etheta_bar,
                                                                               uint32_t* invalid) {
  using Fld = typename P::Fld;
  const uint32_t lane = threadIdx.x & 31u;
  const uint32_t warp = blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32;
  const uint32_t warps = gridDim.x * (blockDim.x / 32);
  for (uint32_t base = warp * 32; base < r.count; base += warps * 32) {
    const uint32_t n = base + lane;
    Loaded L;
    load_record<P>(g, r, n, n < r.count, L);
    if (n < r.count && !L.ok) atomicAdd(invalid, 1u);
    double eb[3] = {0, 0, 0};
    if (L.ok) {
      double bp[3];
      gather3(g, (const Fld*)bnode, L, bp);
      const Response<double> resp(bp[0], bp[1], bp[2], k.boc);
      double gv[3];
#pragma unroll
      for (int c = 0; c < 3; ++c)
        gv[c] = 2.0 * (r.vbar[c * (long long)r.nid + L.pid] + k.dt * k.inv[c] * r.xbar[c * (long long)r.nid + L.pid]);
      transpose_apply(resp.a, gv, eb);
#pragma unroll
      for (int c = 0; c < 3; ++c) eb[c] *= k.beta;
    }
    warp_scatter(g, etheta_bar, L, eb);
  }
}

// The record adjoint. kMover: the mover's part (x_bar', v_bar' are the
// gradients of the moved record; v_bar is replaced, x_bar keeps x_bar' plus
// its terms). kDeposit: the current and mass part (terms added). The B
// gradient is scattered into bnode_bar; with kScatterTheta the mover's E_theta
// gradient into etheta_bar too.
template <class P, bool kMover, bool kDeposit, bool kScatterTheta>
__global__ void __launch_bounds__(kAdjointThreads) adjoint_record_kernel(Geom g, AdjointConstants k,
                                                                        AdjointRecords r, AdjointFields fl,
                                                                        double* bnode_bar, double* etheta_bar,
                                                                        uint32_t* invalid) {
  using Fld = typename P::Fld;
  const uint32_t lane = threadIdx.x & 31u;
  const uint32_t warp = blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32;
  const uint32_t warps = gridDim.x * (blockDim.x / 32);
  const long long nid = r.nid;
  for (uint32_t base = warp * 32; base < r.count; base += warps * 32) {
    const uint32_t n = base + lane;
    Loaded L;
    load_record<P>(g, r, n, n < r.count, L);
    if (n < r.count && !L.ok) atomicAdd(invalid, 1u);
    double bb[3] = {0, 0, 0}, eb[3] = {0, 0, 0};
    if (L.ok) {
      const long long pid = L.pid;
      double bp[3];
      gather3(g, (const Fld*)fl.bnode, L, bp);
      const Response<double> resp(bp[0], bp[1], bp[2], k.boc);
      const double om[3] = {k.boc * bp[0], k.boc * bp[1], k.boc * bp[2]};
      double ab[9];
#pragma unroll
      for (int e = 0; e < 9; ++e) ab[e] = 0;
      double xb[3], vn[3], t[3];
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        xb[c] = r.xbar[c * nid + pid];
        vn[c] = r.vbar[c * nid + pid];
      }
      if constexpr (kMover) {
        // v' = 2 R (v + beta E_theta) - v, x' = x + dt v' / dx.
        double ep[3], gv[3];
        gather3(g, fl.theta, L, ep);
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          const double vt = vn[c] + k.dt * k.inv[c] * xb[c];
          gv[c] = 2.0 * vt;
          vn[c] = -vt;
        }
        transpose_apply(resp.a, gv, t);
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          vn[c] += t[c];
          eb[c] = k.beta * t[c];
        }
        const double uu[3] = {L.v[0] + k.beta * ep[0], L.v[1] + k.beta * ep[1], L.v[2] + k.beta * ep[2]};
#pragma unroll
        for (int a = 0; a < 3; ++a)
#pragma unroll
          for (int b = 0; b < 3; ++b) ab[3 * a + b] += gv[a] * uu[b];
        position_term(g, fl.theta, L, eb, xb);
      }
      if constexpr (kDeposit) {
        double qb = 0;
        const double q = r.q[n];
        if (fl.jbar) {
          // J = sum (q/V) W R v: gradient jscale * jbar gathered.
          double jp[3], h[3];
          gather3(g, fl.jbar, L, jp);
#pragma unroll
          for (int c = 0; c < 3; ++c) jp[c] *= fl.jscale;
          resp.apply(L.v[0], L.v[1], L.v[2], h[0], h[1], h[2]);
          const double qv = q * k.inv_volume;
          transpose_apply(resp.a, jp, t);
#pragma unroll
          for (int c = 0; c < 3; ++c) vn[c] += qv * t[c];
#pragma unroll
          for (int a = 0; a < 3; ++a)
#pragma unroll
            for (int b = 0; b < 3; ++b) ab[3 * a + b] += qv * jp[a] * L.v[b];
          qb += k.inv_volume * (jp[0] * h[0] + jp[1] * h[1] + jp[2] * h[2]);
          const double gj[3] = {fl.jscale * qv * h[0], fl.jscale * qv * h[1], fl.jscale * qv * h[2]};
          position_term(g, fl.jbar, L, gj, xb);
        }
        if (fl.mleft) {
          // mscale * sum_p s lambda_p^T R u_p, s = (beta/c) q.
          double lp[3], up[3], ru[3], rl[3];
          gather3(g, fl.mleft, L, lp);
          gather3(g, fl.mright, L, up);
          resp.apply(up[0], up[1], up[2], ru[0], ru[1], ru[2]);
          transpose_apply(resp.a, lp, rl);
          const double cs = fl.mscale * k.boc * q;
          qb += fl.mscale * k.boc * (lp[0] * ru[0] + lp[1] * ru[1] + lp[2] * ru[2]);
#pragma unroll
          for (int a = 0; a < 3; ++a)
#pragma unroll
            for (int b = 0; b < 3; ++b) ab[3 * a + b] += cs * lp[a] * up[b];
          const double g1[3] = {cs * ru[0], cs * ru[1], cs * ru[2]};
          const double g2[3] = {cs * rl[0], cs * rl[1], cs * rl[2]};
          position_term(g, fl.mleft, L, g1, xb);
          position_term(g, fl.mright, L, g2, xb);
        }
        r.qbar[pid] += qb;
      }
      // The response's dependence on B at the record.
      double ob[3];
      response_gradient(om, resp.a, ab, ob);
#pragma unroll
      for (int c = 0; c < 3; ++c) bb[c] = k.boc * ob[c];
      position_term(g, (const Fld*)fl.bnode, L, bb, xb);
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        r.xbar[c * nid + pid] = xb[c];
        r.vbar[c * nid + pid] = vn[c];
      }
    }
    warp_scatter(g, bnode_bar, L, bb);
    if constexpr (kScatterTheta) warp_scatter(g, etheta_bar, L, eb);
  }
}

// Advance adjoint over the interior nodes 0..n: etheta_bar = a ebar' + far
// C2N(bbar'), ebar = b ebar' (in place); a = 1/theta, b = -(1-theta)/theta
// (1 and 0 at theta = 1), far = -c dt.
__global__ void __launch_bounds__(256) adjoint_advance_kernel(Geom g, double a, double b, double far,
                                                             double* __restrict__ ebar,
                                                             const double* __restrict__ bbar,
                                                             double* __restrict__ etheta_bar) {
  const double inv[3] = {g.inv[0], g.inv[1], g.inv[2]};
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < g.interior;
       t += (long long)gridDim.x * blockDim.x) {
    int i, j, k;
    interior_node_coordinates(g, t, i, j, k);
    double cn[3];
    curl_c2n_at<double>(g, bbar, i, j, k, inv, cn);
    const long long at = g.node(i, j, k);
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const double e = ebar[c * g.nodes + at];
      etheta_bar[c * g.nodes + at] = a * e + far * cn[c];
      ebar[c * g.nodes + at] = b * e;
    }
  }
}

// ebar += lambda over the interior nodes.
__global__ void __launch_bounds__(256) adjoint_add_nodes_kernel(Geom g, const double* __restrict__ lambda,
                                                               double* __restrict__ ebar) {
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < 3 * g.interior;
       t += (long long)gridDim.x * blockDim.x) {
    const long long c = t / g.interior;
    int i, j, k;
    interior_node_coordinates(g, t - c * g.interior, i, j, k);
    const long long at = c * g.nodes + g.node(i, j, k);
    ebar[at] += lambda[at];
  }
}

// bbar += delta N2C(lambda) (when lambda is given) + cell_to_node^T(bnode_bar)
// (when given) over the unique cells: a cell receives 1/8 of each of its 8
// corner nodes' gradient (consistent fields: duplicates hold the unique values).
__global__ void __launch_bounds__(256) adjoint_cells_kernel(Geom g, double delta, const double* __restrict__ lambda,
                                                           const double* __restrict__ bnode_bar,
                                                           double* __restrict__ bbar) {
  const double inv[3] = {g.inv[0], g.inv[1], g.inv[2]};
  const long long cells = (long long)g.nx * g.ny * g.nz;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < cells;
       t += (long long)gridDim.x * blockDim.x) {
    const int i = int(t % g.nx), j = int((t / g.nx) % g.ny), k = int(t / ((long long)g.nx * g.ny));
    double add[3] = {0, 0, 0};
    if (lambda) {
      curl_n2c_at<double>(g, lambda, i, j, k, inv, add);
#pragma unroll
      for (int c = 0; c < 3; ++c) add[c] *= delta;
    }
    if (bnode_bar) {
      const long long b = g.node(i, j, k), sy = g.NX, sz = (long long)g.NX * g.NY;
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const double* p = bnode_bar + c * g.nodes + b;
        const double s = ((p[0] + p[1]) + (p[sy] + p[1 + sy])) + ((p[sz] + p[1 + sz]) + (p[sy + sz] + p[1 + sy + sz]));
        add[c] += 0.125 * s;
      }
    }
    const long long at = g.cell(i, j, k);
#pragma unroll
    for (int c = 0; c < 3; ++c) bbar[c * g.cells + at] += add[c];
  }
}

// Gradient of we W_E + wb W_B: ebar = we V/(4 pi) E at the unique nodes,
// bbar = wb V/(4 pi) B at the cells (the energies sum over exactly those).
template <class T>
__global__ void __launch_bounds__(256) energy_gradient_kernel(Geom g, double ce, double cb, const T* __restrict__ e,
                                                             const T* __restrict__ bcell, double* __restrict__ ebar,
                                                             double* __restrict__ bbar) {
  const long long cells = (long long)g.nx * g.ny * g.nz;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < 3 * cells;
       t += (long long)gridDim.x * blockDim.x) {
    const long long c = t / cells, r = t - c * cells;
    const int i = int(r % g.nx), j = int((r / g.nx) % g.ny), k = int(r / ((long long)g.nx * g.ny));
    const long long n = c * g.nodes + g.node(i, j, k), cl = c * g.cells + g.cell(i, j, k);
    ebar[n] = ce * double(e[n]);
    bbar[cl] = cb * double(bcell[cl]);
  }
}

AdjointConstants constants(const Geom& g, double qom, double dt, double c) {
  AdjointConstants k;
  k.beta = qom * dt / 2;
  k.boc = k.beta / c;
  k.dt = dt;
  k.inv[0] = g.inv[0];
  k.inv[1] = g.inv[1];
  k.inv[2] = g.inv[2];
  k.inv_volume = g.inv_volume;
  return k;
}

AdjointRecords records(const tpicb200_particles* p, uint32_t nid, double* xbar, double* vbar, double* qbar) {
  return AdjointRecords{(const double*)p->rx, (const double*)p->ry, (const double*)p->rz, p->u, p->v, p->w, p->q,
                        p->cell, p->id, p->count, nid, xbar, vbar, qbar};
}

unsigned record_blocks(uint32_t count) {
  return grid_for((long long)(count + 31) / 32 * 32, kAdjointThreads, 148u * 8u);
}

}  // namespace

cudaError_t launch_adjoint_theta_scatter(int precision, const Geom& g, double qom, double dt, double c,
                                         const tpicb200_particles* p, uint32_t nid, const double* xbar,
                                         const double* vbar, const void* bnode, double* etheta_bar,
                                         uint32_t* invalid, cudaStream_t s) {
  if (p->count == 0) return cudaSuccess;
  const AdjointConstants k = constants(g, qom, dt, c);
  const AdjointRecords r = records(p, nid, const_cast<double*>(xbar), const_cast<double*>(vbar), nullptr);
  if (precision == TPICB200_PRECISION_DOUBLE)
    adjoint_theta_scatter_kernel<PDouble><<<record_blocks(p->count), kAdjointThreads, 0, s>>>(g, k, r, bnode,
                                                                                            etheta_bar, invalid);
  else
    adjoint_theta_scatter_kernel<PMixed><<<record_blocks(p->count), kAdjointThreads, 0, s>>>(g, k, r, bnode,
                                                                                           etheta_bar, invalid);
  count_launches(1);
  return cudaGetLastError();
}

cudaError_t launch_adjoint_records(int precision, int mode, const Geom& g, double qom, double dt, double c,
                                   const tpicb200_particles* p, uint32_t nid, double* xbar, double* vbar,
                                   double* qbar, const double* theta, const void* bnode, const double* jbar,
                                   double jscale, const double* mleft, const double* mright, double mscale,
                                   double* bnode_bar, double* etheta_bar, uint32_t* invalid, cudaStream_t s) {
  if (p->count == 0) return cudaSuccess;
  const AdjointConstants k = constants(g, qom, dt, c);
  const AdjointRecords r = records(p, nid, xbar, vbar, qbar);
  const AdjointFields fl{theta, bnode, jbar, jscale, mleft, mright, mscale};
  const unsigned blocks = record_blocks(p->count);
  auto go = [&](auto kernel) {
    kernel<<<blocks, kAdjointThreads, 0, s>>>(g, k, r, fl, bnode_bar, etheta_bar, invalid);
  };
  const bool dbl = precision == TPICB200_PRECISION_DOUBLE;
  switch (mode) {
    case kAdjointMover:
      if (dbl) go(adjoint_record_kernel<PDouble, true, false, true>);
      else go(adjoint_record_kernel<PMixed, true, false, true>);
      break;
    case kAdjointDeposit:
      if (dbl) go(adjoint_record_kernel<PDouble, false, true, false>);
      else go(adjoint_record_kernel<PMixed, false, true, false>);
      break;
    case kAdjointCycle:
      if (dbl) go(adjoint_record_kernel<PDouble, true, true, false>);
      else go(adjoint_record_kernel<PMixed, true, true, false>);
      break;
    default:
      return cudaErrorInvalidValue;
  }
  count_launches(1);
  return cudaGetLastError();
}

cudaError_t launch_adjoint_advance(const Geom& g, double theta, double c, double dt, double* ebar, const double* bbar,
                                   double* etheta_bar, cudaStream_t s) {
  const bool one = fabs(theta - 1.0) < 1e-10;
  const double a = one ? 1.0 : 1.0 / theta, b = one ? 0.0 : -(1.0 - theta) / theta;
  adjoint_advance_kernel<<<grid_for(g.interior, 256), 256, 0, s>>>(g, a, b, -c * dt, ebar, bbar, etheta_bar);
  count_launches(1);
  launch_node_ghosts(g, ebar, 3, s);
  launch_node_ghosts(g, etheta_bar, 3, s);
  return cudaGetLastError();
}

cudaError_t launch_adjoint_add_nodes(const Geom& g, const double* lambda, double* ebar, cudaStream_t s) {
  adjoint_add_nodes_kernel<<<grid_for(3 * g.interior, 256), 256, 0, s>>>(g, lambda, ebar);
  count_launches(1);
  launch_node_ghosts(g, ebar, 3, s);
  return cudaGetLastError();
}

cudaError_t launch_adjoint_cells(const Geom& g, double delta, const double* lambda, const double* bnode_bar,
                                 double* bbar, cudaStream_t s) {
  adjoint_cells_kernel<<<grid_for((long long)g.nx * g.ny * g.nz, 256), 256, 0, s>>>(g, delta, lambda, bnode_bar,
                                                                                     bbar);
  count_launches(1);
  return launch_cell_ghosts(TPICB200_PRECISION_DOUBLE, g, bbar, s);
}

cudaError_t launch_energy_gradient(int precision, const Geom& g, double we, double wb, const void* e,
                                   const void* bcell, double* ebar, double* bbar, cudaStream_t s) {
  const double norm = g.volume / (4 * 3.14159265358979323846);
  cudaError_t err = cudaMemsetAsync(ebar, 0, size_t(3) * g.nodes * sizeof(double), s);
  if (err == cudaSuccess) err = cudaMemsetAsync(bbar, 0, size_t(3) * g.cells * sizeof(double), s);
  if (err != cudaSuccess) return err;
  const unsigned blocks = grid_for(3LL * g.nx * g.ny * g.nz, 256);
  if (precision == TPICB200_PRECISION_DOUBLE)
    energy_gradient_kernel<double><<<blocks, 256, 0, s>>>(g, we * norm, wb * norm, (const double*)e,
                                                          (const double*)bcell, ebar, bbar);
  else
    energy_gradient_kernel<float><<<blocks, 256, 0, s>>>(g, we * norm, wb * norm, (const float*)e,
                                                         (const float*)bcell, ebar, bbar);
  count_launches(1);
  launch_node_ghosts(g, ebar, 3, s);
  return launch_cell_ghosts(TPICB200_PRECISION_DOUBLE, g, bbar, s);
}

}  // namespace tpicb200
