// CPU oracle of the single-GPU ECSIM particle cycle.
//
// TEST INFRASTRUCTURE ONLY. This file is the scalar restatement of TPIC's
// algorithm that the tests, the smoke check and the CPU baseline of the bench
// use as the checker. The product (tpic_b200/) never links, loads or calls it.
//
// Build: oracle/Makefile (g++ -O2 -ffp-contract=off: strict IEEE evaluation of
// every expression as written, which is how the reference's own host numerics
// compile; the GPU mover is built with -fmad=false so that the two agree bit
// for bit).
//
// Each function names the reference file:line it restates (paths relative to
// the TPIC source tree). Layouts are the ones of include/tpicb200.h:
//   node field  : component-major, extent (n+3) per axis, index (i+1)+NX*((j+1)+NY*(k+1))
//   cell field  : component-major, extent (n+2) per axis, index (i+1)+CX*((j+1)+CY*(k+1))
//   mass records: 126 scalars per node-field vertex, [stencil][row-major 3x3]
//   particle key: (i+2)+(nx+4)*((j+2)+(ny+4)*(k+2))
//   GMRES vector: 3 x (nx+1)(ny+1)(nz+1) interior nodes, component-major, x fastest
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <vector>

struct oracle_gmres_result {
  int converged, iterations;
  double initial_residual, residual, rhs_norm, relative_residual;
};

namespace {

constexpr double kPi = 3.14159265358979323846264338327950288;

struct Grid {
  int nx, ny, nz;
  double dx, dy, dz;
};

struct Layout {
  int nx, ny, nz;
  long NX, NY, NZ;   // node extents with one-node halo
  long CX, CY, CZ;   // cell extents with one-cell halo
  long nodes, cells;
  int ex, ey;        // particle key extents (halo 2)
  long bins;
  long inx, iny, inz, interior;  // interior nodes (cells + 1)
  explicit Layout(const Grid& g)
      : nx(g.nx), ny(g.ny), nz(g.nz), NX(g.nx + 3), NY(g.ny + 3), NZ(g.nz + 3),
        CX(g.nx + 2), CY(g.ny + 2), CZ(g.nz + 2), nodes((g.nx + 3L) * (g.ny + 3L) * (g.nz + 3L)),
        cells((g.nx + 2L) * (g.ny + 2L) * (g.nz + 2L)), ex(g.nx + 4), ey(g.ny + 4),
        bins((g.nx + 4L) * (g.ny + 4L) * (g.nz + 4L)), inx(g.nx + 1), iny(g.ny + 1), inz(g.nz + 1),
        interior((g.nx + 1L) * (g.ny + 1L) * (g.nz + 1L)) {}
  long node(int i, int j, int k) const { return (i + 1) + NX * ((j + 1) + NY * (long)(k + 1)); }
  long cell(int i, int j, int k) const { return (i + 1) + CX * ((j + 1) + CY * (long)(k + 1)); }
  int32_t encode(int i, int j, int k) const { return (i + 2) + ex * ((j + 2) + ey * (k + 2)); }
  void decode(int32_t key, int& i, int& j, int& k) const {
    const int yz = key / ex;
    i = key % ex - 2;
    j = yz % ey - 2;
    k = yz / ey - 2;
  }
  bool interior_cell(int i, int j, int k) const {
    return i >= 0 && i < nx && j >= 0 && j < ny && k >= 0 && k < nz;
  }
};

// mass_stencil_offset, data/mass_matrix/mass_matrix_layout.hpp:17-24.
constexpr int kStencil[14][3] = {{0, 0, 0}, {1, 0, 0}, {0, 1, 0}, {0, 0, 1}, {1, 1, 0},
                                 {1, -1, 0}, {1, 0, 1}, {1, 0, -1}, {0, 1, 1}, {0, 1, -1},
                                 {1, -1, 1}, {1, 1, -1}, {-1, 1, 1}, {1, 1, 1}};

// make_mass_pair_stencils, ecsim/mass_matrix/mass_matrix_stencil.hpp:13-33.
int pair_stencil(int a, int b) {
  const int d[3] = {((b & 1) - (a & 1)), ((b >> 1) & 1) - ((a >> 1) & 1),
                    ((b >> 2) & 1) - ((a >> 2) & 1)};
  int index = -1;
  for (int s = 0; s < 14; ++s)
    if (kStencil[s][0] == d[0] && kStencil[s][1] == d[1] && kStencil[s][2] == d[2]) index = s;
  return index;
}

// make_cic_weights, ecsim/particles/cic.hpp:24-36: grouping (wx*wy)*wz.
template <class C> void cic(C x, C y, C z, C w[8]) {
  const C cx = C(1) - x, cy = C(1) - y, cz = C(1) - z;
  w[0] = cx * cy * cz; w[1] = x * cy * cz; w[2] = cx * y * cz; w[3] = x * y * cz;
  w[4] = cx * cy * z;  w[5] = x * cy * z;  w[6] = cx * y * z;  w[7] = x * y * z;
}

// interpolate_cic, ecsim/particles/cic.hpp:60-71: corners summed in increasing order.
template <class C, class F>
C gather(const F* field, const Layout& L, int i, int j, int k, const C w[8]) {
  C value = 0;
  for (int a = 0; a < 8; ++a)
    value += w[a] * C(field[L.node(i + (a & 1), j + ((a >> 1) & 1), k + ((a >> 2) & 1))]);
  return value;
}

// ParticleResponse, ecsim/particles/particle_response.hpp:16-42.
template <class C> struct Response {
  C a[9];
  C norm_square;
  Response(C bx, C by, C bz, C beta_over_c) {
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
  void apply(C x, C y, C z, C& ox, C& oy, C& oz) const {
    ox = a[0] * x + a[1] * y + a[2] * z;
    oy = a[3] * x + a[4] * y + a[5] * z;
    oz = a[6] * x + a[7] * y + a[8] * z;
  }
};

template <class T> bool finite(T v) {
  return v >= -std::numeric_limits<T>::max() && v <= std::numeric_limits<T>::max();
}

// Storage/compute types of the two precision modes (include/tpicb200.h):
// 0 = double everywhere; 1 = FP64 positions and charges, FP32 velocities,
// fields, moments and mass, FP32 velocity/current compute, FP64 position compute.
template <int P> struct Prec;
template <> struct Prec<0> { using Pos = double; using Vel = double; using VC = double; using Fld = double; };
template <> struct Prec<1> { using Pos = double; using Vel = float; using VC = float; using Fld = float; };

// push_and_classify_particle, ecsim/particles/particle_mover_device.hpp:37-122, with
// the whole-domain periodic wrap of classify_particle_point,
// communication/particles/particle_boundaries.hpp:112-135. Returns 1 for an
// invalid record, which keeps all of its attributes.
template <int P>
int push(const Layout& L, typename Prec<P>::VC beta, typename Prec<P>::VC beta_over_c, double dt,
         const double inv[3], typename Prec<P>::Pos* rx, typename Prec<P>::Pos* ry,
         typename Prec<P>::Pos* rz, typename Prec<P>::Vel* u, typename Prec<P>::Vel* v,
         typename Prec<P>::Vel* w, const double* q, int32_t* key, uint32_t n,
         const double* theta, const typename Prec<P>::Fld* bnode) {
  using C = typename Prec<P>::VC;
  using Pos = typename Prec<P>::Pos;
  using Vel = typename Prec<P>::Vel;
  const int32_t k0 = key[n];
  if (k0 < 0 || k0 >= L.bins) return 1;
  int ci, cj, ck;
  L.decode(k0, ci, cj, ck);
  if (!L.interior_cell(ci, cj, ck) || !finite(q[n])) return 1;
  const Pos fx = rx[n], fy = ry[n], fz = rz[n];
  if (!(fx >= Pos(0) && fx < Pos(1) && fy >= Pos(0) && fy < Pos(1) && fz >= Pos(0) && fz < Pos(1)))
    return 1;
  C wt[8];
  cic<C>(C(fx), C(fy), C(fz), wt);
  const long nn = L.nodes;
  const C bx = gather<C>(bnode, L, ci, cj, ck, wt);
  const C by = gather<C>(bnode + nn, L, ci, cj, ck, wt);
  const C bz = gather<C>(bnode + 2 * nn, L, ci, cj, ck, wt);
  const C ex = gather<C>(theta, L, ci, cj, ck, wt);
  const C ey = gather<C>(theta + nn, L, ci, cj, ck, wt);
  const C ez = gather<C>(theta + 2 * nn, L, ci, cj, ck, wt);
  const Response<C> r(bx, by, bz, beta_over_c);
  const C uu = C(u[n]), vv = C(v[n]), ww = C(w[n]);
  C hx, hy, hz, ax, ay, az;
  r.apply(uu, vv, ww, hx, hy, hz);
  r.apply(ex, ey, ez, ax, ay, az);
  const C px = hx + beta * ax, py = hy + beta * ay, pz = hz + beta * az;
  Vel vel[3] = {Vel(C(2) * px - uu), Vel(C(2) * py - vv), Vel(C(2) * pz - ww)};
  int64_t cell[3] = {ci, cj, ck};
  Pos frac[3] = {fx, fy, fz};
  const int ext[3] = {L.nx, L.ny, L.nz};
  for (int axis = 0; axis < 3; ++axis) {
    if (!finite(vel[axis])) return 1;
    const Pos displacement = Pos(dt * double(vel[axis]) * inv[axis]);
    const Pos moved = frac[axis] + displacement;
    const double shift = std::floor(double(moved));
    if (!(shift >= double(std::numeric_limits<int32_t>::min()) &&
          shift <= double(std::numeric_limits<int32_t>::max())))
      return 1;
    cell[axis] += int64_t(shift);
    frac[axis] = moved - Pos(shift);
    if (frac[axis] == Pos(1)) {
      ++cell[axis];
      frac[axis] = Pos(0);
    }
  }
  for (int axis = 0; axis < 3; ++axis) {
    const int64_t e = ext[axis];
    if (cell[axis] < 0 || cell[axis] >= e) {
      int64_t m = cell[axis] % e;
      cell[axis] = m < 0 ? m + e : m;
    }
  }
  key[n] = L.encode(int(cell[0]), int(cell[1]), int(cell[2]));
  rx[n] = frac[0]; ry[n] = frac[1]; rz[n] = frac[2];
  u[n] = vel[0]; v[n] = vel[1]; w[n] = vel[2];
  return 0;
}

// Periodic fold of a node field: every periodic copy of a node (the shared
// endpoint plane n duplicates plane 0) receives the sum of all copies, then the
// one-node ghosts copy the opposite interior plane. This is the self-periodic
// form of the shared-node addition and ghost copy of the current assembly,
// ecsim/deposition/current_assembly_device.hpp:26-53, and of the compact mass
// halo, communication/mass_halo/mass_halo_device.hpp:91-160,350-364.
template <class T> void fold_add(const Layout& L, T* field, int width, long stride) {
  // width values per vertex (1 for a field component, 126 for mass records).
  for (int k = 0; k <= L.nz; ++k)
    for (int j = 0; j <= L.ny; ++j)
      for (int i = 0; i <= L.nx; ++i) {
        if (i == L.nx || j == L.ny || k == L.nz) continue;  // visit unique nodes
        int ci[2] = {i, i + L.nx}, cj[2] = {j, j + L.ny}, ck[2] = {k, k + L.nz};
        const int ni = (i == 0) ? 2 : 1, nj = (j == 0) ? 2 : 1, nk = (k == 0) ? 2 : 1;
        for (int e = 0; e < width; ++e) {
          T sum = 0;
          for (int c = 0; c < nk; ++c)
            for (int b = 0; b < nj; ++b)
              for (int a = 0; a < ni; ++a) sum += field[L.node(ci[a], cj[b], ck[c]) * stride + e];
          for (int c = 0; c < nk; ++c)
            for (int b = 0; b < nj; ++b)
              for (int a = 0; a < ni; ++a) field[L.node(ci[a], cj[b], ck[c]) * stride + e] = sum;
        }
      }
}

// Ghost copy of a node field (one-node halo, fully periodic): plane -1 takes
// plane n-1 and plane n+1 takes plane 1, axis by axis so edges and corners fill.
template <class T> void node_ghosts(const Layout& L, T* field, int width, long stride) {
  for (int k = -1; k <= L.nz + 1; ++k)
    for (int j = -1; j <= L.ny + 1; ++j) {
      for (int e = 0; e < width; ++e) {
        field[L.node(-1, j, k) * stride + e] = field[L.node(L.nx - 1, j, k) * stride + e];
        field[L.node(L.nx + 1, j, k) * stride + e] = field[L.node(1, j, k) * stride + e];
      }
    }
  for (int k = -1; k <= L.nz + 1; ++k)
    for (int i = -1; i <= L.nx + 1; ++i)
      for (int e = 0; e < width; ++e) {
        field[L.node(i, -1, k) * stride + e] = field[L.node(i, L.ny - 1, k) * stride + e];
        field[L.node(i, L.ny + 1, k) * stride + e] = field[L.node(i, 1, k) * stride + e];
      }
  for (int j = -1; j <= L.ny + 1; ++j)
    for (int i = -1; i <= L.nx + 1; ++i)
      for (int e = 0; e < width; ++e) {
        field[L.node(i, j, -1) * stride + e] = field[L.node(i, j, L.nz - 1) * stride + e];
        field[L.node(i, j, L.nz + 1) * stride + e] = field[L.node(i, j, 1) * stride + e];
      }
}

// Periodic ghost cells of a cell field: cell -1 takes cell n-1, cell n takes cell 0.
template <class T> void cell_ghosts(const Layout& L, T* f) {
  for (int c = 0; c < 3; ++c) {
    T* g = f + c * L.cells;
    for (int k = -1; k <= L.nz; ++k)
      for (int j = -1; j <= L.ny; ++j) {
        g[L.cell(-1, j, k)] = g[L.cell(L.nx - 1, j, k)];
        g[L.cell(L.nx, j, k)] = g[L.cell(0, j, k)];
      }
    for (int k = -1; k <= L.nz; ++k)
      for (int i = -1; i <= L.nx; ++i) {
        g[L.cell(i, -1, k)] = g[L.cell(i, L.ny - 1, k)];
        g[L.cell(i, L.ny, k)] = g[L.cell(i, 0, k)];
      }
    for (int j = -1; j <= L.ny; ++j)
      for (int i = -1; i <= L.nx; ++i) {
        g[L.cell(i, j, -1)] = g[L.cell(i, j, L.nz - 1)];
        g[L.cell(i, j, L.nz)] = g[L.cell(i, j, 0)];
      }
  }
}

// NodeCellSamples::derivative, ecsim/fields/node_cell_curl.hpp:59-78: four edge
// differences summed in the written order, times 0.25 * inverse spacing.
// Node sources extend forwards (step +1, difference neighbor - anchor), cell
// sources backwards (step -1, difference anchor - neighbor).
struct Samples {
  double base, x, y, z, xy, xz, yz, xyz;
  bool node;
  double d(double anchor, double nb) const { return node ? nb - anchor : anchor - nb; }
  double dx(double inv) const { return 0.25 * inv * (d(base, x) + d(z, xz) + d(y, xy) + d(yz, xyz)); }
  double dy(double inv) const { return 0.25 * inv * (d(base, y) + d(z, yz) + d(x, xy) + d(xz, xyz)); }
  double dz(double inv) const { return 0.25 * inv * (d(base, z) + d(x, xz) + d(y, yz) + d(xy, xyz)); }
};

template <class T>
Samples node_samples(const Layout& L, const T* f, int i, int j, int k) {
  return {double(f[L.node(i, j, k)]), double(f[L.node(i + 1, j, k)]), double(f[L.node(i, j + 1, k)]),
          double(f[L.node(i, j, k + 1)]), double(f[L.node(i + 1, j + 1, k)]),
          double(f[L.node(i + 1, j, k + 1)]), double(f[L.node(i, j + 1, k + 1)]),
          double(f[L.node(i + 1, j + 1, k + 1)]), true};
}
template <class T>
Samples cell_samples(const Layout& L, const T* f, int i, int j, int k) {
  return {double(f[L.cell(i, j, k)]), double(f[L.cell(i - 1, j, k)]), double(f[L.cell(i, j - 1, k)]),
          double(f[L.cell(i, j, k - 1)]), double(f[L.cell(i - 1, j - 1, k)]),
          double(f[L.cell(i - 1, j, k - 1)]), double(f[L.cell(i, j - 1, k - 1)]),
          double(f[L.cell(i - 1, j - 1, k - 1)]), false};
}

// node_cell_curl, ecsim/fields/node_cell_curl.hpp:116-126.
void curl(const Samples& x, const Samples& y, const Samples& z, const double inv[3], double out[3]) {
  out[0] = z.dy(inv[1]) - y.dz(inv[2]);
  out[1] = x.dz(inv[2]) - z.dx(inv[0]);
  out[2] = y.dx(inv[0]) - x.dy(inv[1]);
}

// N2C curl over all cells 0..n-1 from a node field, then periodic cell ghosts.
template <class T> void curl_n2c(const Layout& L, const T* node, double* cellf, const double inv[3]) {
  for (int k = 0; k < L.nz; ++k)
    for (int j = 0; j < L.ny; ++j)
      for (int i = 0; i < L.nx; ++i) {
        double o[3];
        curl(node_samples(L, node, i, j, k), node_samples(L, node + L.nodes, i, j, k),
             node_samples(L, node + 2 * L.nodes, i, j, k), inv, o);
        for (int c = 0; c < 3; ++c) cellf[c * L.cells + L.cell(i, j, k)] = o[c];
      }
  cell_ghosts(L, cellf);
}

// C2N curl over interior nodes 0..n from a cell field with filled ghosts.
template <class T> void curl_c2n(const Layout& L, const T* cellf, double* node, const double inv[3]) {
  for (int k = 0; k <= L.nz; ++k)
    for (int j = 0; j <= L.ny; ++j)
      for (int i = 0; i <= L.nx; ++i) {
        double o[3];
        curl(cell_samples(L, cellf, i, j, k), cell_samples(L, cellf + L.cells, i, j, k),
             cell_samples(L, cellf + 2 * L.cells, i, j, k), inv, o);
        for (int c = 0; c < 3; ++c) node[c * L.nodes + L.node(i, j, k)] = o[c];
      }
}

// cell_to_node_average, ecsim/fields/cell_to_node.hpp:19-32.
template <class T, class O> void cell_to_node(const Layout& L, const T* cellf, O* node) {
  for (int c = 0; c < 3; ++c) {
    const T* g = cellf + c * L.cells;
    for (int k = 0; k <= L.nz; ++k)
      for (int j = 0; j <= L.ny; ++j)
        for (int i = 0; i <= L.nx; ++i) {
          const double v = (double(g[L.cell(i - 1, j - 1, k - 1)]) + double(g[L.cell(i, j - 1, k - 1)]) +
                            double(g[L.cell(i - 1, j, k - 1)]) + double(g[L.cell(i, j, k - 1)]) +
                            double(g[L.cell(i - 1, j - 1, k)]) + double(g[L.cell(i, j - 1, k)]) +
                            double(g[L.cell(i - 1, j, k)]) + double(g[L.cell(i, j, k)])) * 0.125;
          node[c * L.nodes + L.node(i, j, k)] = O(v);
        }
  }
  node_ghosts(L, node, 1, 1);
  node_ghosts(L, node + L.nodes, 1, 1);
  node_ghosts(L, node + 2 * L.nodes, 1, 1);
}

// apply_mass_matrix_node, ecsim/mass_matrix/mass_matrix_stencil.hpp:119-149:
// centre, then per stencil the forward neighbour with this vertex's block and
// the backward neighbour with the neighbour vertex's block, untransposed.
// transpose = true applies M^T: the same blocks, each 3x3 block transposed
// (M^T has block (g, g+s) = B(g,s)^T and (g, g-s) = B(g-s,s)^T, so the
// stencil walk is unchanged).
template <class M>
void mass_apply_node(const Layout& L, const M* mass, const double* in, int i, int j, int k,
                     double row_inverse_volume, double out[3], bool transpose = false) {
  const long nn = L.nodes;
  auto block = [&](long vertex, int s, long at, double& x, double& y, double& z) {
    const M* b = mass + vertex * 126 + s * 9;
    const double vx = in[at], vy = in[nn + at], vz = in[2 * nn + at];
    if (transpose) {
      x = vx * double(b[0]) + vy * double(b[3]) + vz * double(b[6]);
      y = vx * double(b[1]) + vy * double(b[4]) + vz * double(b[7]);
      z = vx * double(b[2]) + vy * double(b[5]) + vz * double(b[8]);
      return;
    }
    x = vx * double(b[0]) + vy * double(b[1]) + vz * double(b[2]);
    y = vx * double(b[3]) + vy * double(b[4]) + vz * double(b[5]);
    z = vx * double(b[6]) + vy * double(b[7]) + vz * double(b[8]);
  };
  const long g = L.node(i, j, k);
  double x, y, z;
  block(g, 0, g, x, y, z);
  for (int s = 1; s < 14; ++s) {
    double bx, by, bz;
    const long fwd = L.node(i + kStencil[s][0], j + kStencil[s][1], k + kStencil[s][2]);
    block(g, s, fwd, bx, by, bz);
    x += bx; y += by; z += bz;
    const long bwd = L.node(i - kStencil[s][0], j - kStencil[s][1], k - kStencil[s][2]);
    block(bwd, s, bwd, bx, by, bz);
    x += bx; y += by; z += bz;
  }
  out[0] = x * row_inverse_volume;
  out[1] = y * row_inverse_volume;
  out[2] = z * row_inverse_volume;
}

struct Physics {
  double dt, theta, c, delta, kfac, inv_volume, inv[3];
  Physics(const Grid& g, double dt_, double theta_, double c_)
      : dt(dt_), theta(theta_), c(c_), delta(c_ * theta_ * dt_), kfac(4 * kPi * (theta_ * dt_)),
        inv_volume(1.0 / ((g.dx * g.dy) * g.dz)), inv{1.0 / g.dx, 1.0 / g.dy, 1.0 / g.dz} {}
};

// One energy-conserving smoothing pass at interior node (i,j,k) of a node
// component with filled ghosts (node_smoothing_value,
// ecsim/fields/node_smoothing.hpp:24-52): op 0 Face7, alpha*centre +
// beta*faces with beta = (1-alpha)/6; op 1 Binomial27, (8*centre + 4*faces +
// 2*edges + corners)/64. Each neighbour sum runs left to right in the order
// the reference fixes; every load is promoted before any arithmetic.
template <class C>
C smooth_value(const Layout& L, const double* f, int i, int j, int k, int op, C alpha, C beta) {
  auto v = [&](int a, int b, int c) { return C(f[L.node(a, b, c)]); };
  const C face = v(i - 1, j, k) + v(i + 1, j, k) + v(i, j - 1, k) + v(i, j + 1, k) + v(i, j, k - 1) + v(i, j, k + 1);
  if (op == 0) return alpha * v(i, j, k) + beta * face;
  const C edge = v(i - 1, j - 1, k) + v(i + 1, j - 1, k) + v(i - 1, j + 1, k) + v(i + 1, j + 1, k) +
                 v(i - 1, j, k - 1) + v(i + 1, j, k - 1) + v(i - 1, j, k + 1) + v(i + 1, j, k + 1) +
                 v(i, j - 1, k - 1) + v(i, j + 1, k - 1) + v(i, j - 1, k + 1) + v(i, j + 1, k + 1);
  const C corner = v(i - 1, j - 1, k - 1) + v(i + 1, j - 1, k - 1) + v(i - 1, j + 1, k - 1) +
                   v(i + 1, j + 1, k - 1) + v(i - 1, j - 1, k + 1) + v(i + 1, j - 1, k + 1) +
                   v(i - 1, j + 1, k + 1) + v(i + 1, j + 1, k + 1);
  return (C(8) * v(i, j, k) + C(4) * face + C(2) * edge + corner) * (C(1) / C(64));
}

// S^niter of a 3-component node field in FP64 storage (complete_smoothing,
// ecsim/maxwell/maxwell_device.hpp:455-487 on a periodic domain): the ghosts
// are filled before every pass, each pass writes the interior nodes 0..n,
// and the result leaves with its ghosts filled. niter = 0 copies.
void smooth_field(const Layout& L, int niter, int op, double alpha, const double* src, double* out) {
  std::vector<double> a(src, src + 3 * L.nodes), b(3 * L.nodes, 0.0);
  const double beta = (1.0 - alpha) / 6.0;
  for (int pass = 0; pass < niter; ++pass) {
    for (int c = 0; c < 3; ++c) node_ghosts(L, a.data() + c * L.nodes, 1, 1);
    b = a;
    for (int c = 0; c < 3; ++c)
      for (int k = 0; k <= L.nz; ++k)
        for (int j = 0; j <= L.ny; ++j)
          for (int i = 0; i <= L.nx; ++i)
            b[c * L.nodes + L.node(i, j, k)] = smooth_value<double>(L, a.data() + c * L.nodes, i, j, k, op, alpha, beta);
    a.swap(b);
  }
  for (int c = 0; c < 3; ++c) node_ghosts(L, a.data() + c * L.nodes, 1, 1);
  std::copy(a.begin(), a.end(), out);
}

// MaxwellOperator::complete_apply with the unsmoothed full schedule and
// combine_image, ecsim/maxwell/maxwell_device.hpp:184-212,471-484:
// image = ((input + delta^2 * curl_C2N(curl_N2C(input))) + k * M input).
// `in` is a node field whose ghosts this function fills.
// With smoothing (niter > 0), complete_apply_smoothed and combine_image
// (maxwell_device.hpp:389-432): the mass response of S^n(input), smoothed
// n times, replaces M input.
struct Smoothing {
  int niter = 0, op = 0;
  double alpha = 1.0;
};
template <class M>
void maxwell_apply(const Layout& L, const Physics& ph, const M* mass, double* in, double* image,
                   double* curl_cell, double* curl_node, const Smoothing& sm = Smoothing{},
                   bool transpose = false) {
  node_ghosts(L, in, 1, 1);
  node_ghosts(L, in + L.nodes, 1, 1);
  node_ghosts(L, in + 2 * L.nodes, 1, 1);
  curl_n2c(L, in, curl_cell, ph.inv);
  curl_c2n(L, curl_cell, curl_node, ph.inv);
  const double d2 = ph.delta * ph.delta;
  std::vector<double> response;
  if (sm.niter > 0) {
    std::vector<double> smoothed(3 * L.nodes), mimage(3 * L.nodes, 0.0);
    smooth_field(L, sm.niter, sm.op, sm.alpha, in, smoothed.data());
    for (int k = 0; k <= L.nz; ++k)
      for (int j = 0; j <= L.ny; ++j)
        for (int i = 0; i <= L.nx; ++i) {
          double m[3];
          mass_apply_node(L, mass, smoothed.data(), i, j, k, ph.inv_volume, m);
          for (int c = 0; c < 3; ++c) mimage[c * L.nodes + L.node(i, j, k)] = m[c];
        }
    response.resize(3 * L.nodes);
    smooth_field(L, sm.niter, sm.op, sm.alpha, mimage.data(), response.data());
  }
  for (int k = 0; k <= L.nz; ++k)
    for (int j = 0; j <= L.ny; ++j)
      for (int i = 0; i <= L.nx; ++i) {
        double m[3];
        const long g = L.node(i, j, k);
        if (sm.niter > 0)
          for (int c = 0; c < 3; ++c) m[c] = response[c * L.nodes + g];
        else
          mass_apply_node(L, mass, in, i, j, k, ph.inv_volume, m, transpose);
        for (int c = 0; c < 3; ++c) {
          const long at = c * L.nodes + g;
          image[at] = (1.0 * in[at] + d2 * curl_node[at]) + ph.kfac * m[c];
        }
      }
}

// Restarted GMRES from the guess x, restating Gmres::host_blocking_solve,
// ecsim/gmres/gmres_device.hpp:355-454, with the device tails of :52-98
// (classical Gram-Schmidt, Givens rotations, true-residual acceptance).
// Returns -1 on a nonfinite estimate, else 0 (res.converged tells).
template <class Apply>
int gmres(Apply&& apply, const double* b, double* x, long N, int restart, int max_iterations, double tol,
          oracle_gmres_result& res) {
  std::vector<double> r(N), Ax(N), w(N);
  std::vector<double> V((size_t)(restart + 1) * N);
  std::vector<double> H((size_t)restart * (restart + 1)), cs(restart), sn(restart), s(restart + 1),
      y(restart);
  auto dot = [&](const double* a, const double* bb) {
    double sum = 0;
    for (long n = 0; n < N; ++n) sum += a[n] * bb[n];
    return sum;
  };
  apply(x, Ax.data());
  for (long n = 0; n < N; ++n) r[n] = b[n] - Ax[n];
  res = oracle_gmres_result{};
  res.residual = res.initial_residual = std::sqrt(dot(r.data(), r.data()));
  res.rhs_norm = std::sqrt(dot(b, b));
  const double scale = res.rhs_norm == 0 ? 1.0 : res.rhs_norm;
  const double atol = scale * tol;
  res.relative_residual = res.residual / scale;
  res.converged = res.residual <= atol;
  while (!res.converged && res.iterations < max_iterations) {
    std::fill(H.begin(), H.end(), 0.0);
    std::fill(cs.begin(), cs.end(), 0.0);
    std::fill(sn.begin(), sn.end(), 0.0);
    std::fill(s.begin(), s.end(), 0.0);
    double rn2 = dot(r.data(), r.data());
    double sc = rn2 > 0 ? 1.0 / std::sqrt(rn2) : 0.0;
    for (long n = 0; n < N; ++n) V[n] = r[n] * sc;
    s[0] = std::sqrt(rn2);
    const int columns = std::min(restart, max_iterations - res.iterations);
    int completed = 0;
    bool breakdown = false;
    for (int col = 0; col < columns; ++col) {
      apply(&V[(size_t)col * N], w.data());
      double* h = &H[(size_t)col * (restart + 1)];
      std::vector<double> dots(col + 1);
      for (int jj = 0; jj <= col; ++jj) dots[jj] = dot(&V[(size_t)jj * N], w.data());
      double n2 = 0;
      for (long n = 0; n < N; ++n) {
        double val = w[n];
        for (int jj = 0; jj <= col; ++jj) val -= dots[jj] * V[(size_t)jj * N + n];
        w[n] = val;
        n2 += val * val;
      }
      for (int jj = 0; jj <= col; ++jj) h[jj] = dots[jj];
      // ArnoldiLeastSquaresUpdate, gmres_device.hpp:62-98.
      const double sub = std::sqrt(n2);
      h[col + 1] = sub;
      for (int row = 0; row < col; ++row) {
        const double up = h[row], lo = h[row + 1];
        h[row] = cs[row] * up + sn[row] * lo;
        h[row + 1] = -sn[row] * up + cs[row] * lo;
      }
      const double diag = h[col];
      const double den = std::hypot(diag, sub);
      const double cc = den != 0 ? diag / den : 1.0;
      const double ss = den != 0 ? sub / den : 0.0;
      cs[col] = cc;
      sn[col] = ss;
      h[col] = cc * diag + ss * sub;
      h[col + 1] = 0;
      const double up = s[col], lo = s[col + 1];
      s[col] = cc * up + ss * lo;
      s[col + 1] = -ss * up + cc * lo;
      const double estimate = std::fabs(s[col + 1]);
      const double nsc = n2 > 0 ? 1.0 / std::sqrt(n2) : 0.0;
      for (long n = 0; n < N; ++n) V[(size_t)(col + 1) * N + n] = w[n] * nsc;
      completed = col + 1;
      breakdown = sub == 0;
      if (!std::isfinite(estimate)) return -1;
      if (estimate <= atol || breakdown) break;
    }
    // gmres_back_substitute_kernel, gmres_device.hpp:267-277.
    for (int row = completed - 1; row >= 0; --row) {
      double sum = 0;
      for (int col = row + 1; col < completed; ++col) sum += H[(size_t)col * (restart + 1) + row] * y[col];
      const double d = H[(size_t)row * (restart + 1) + row];
      y[row] = d != 0 ? (s[row] - sum) / d : 0.0;
    }
    for (long n = 0; n < N; ++n) {
      double val = x[n];
      for (int col = 0; col < completed; ++col) val += y[col] * V[(size_t)col * N + n];
      x[n] = val;
    }
    res.iterations += completed;
    apply(x, Ax.data());
    for (long n = 0; n < N; ++n) r[n] = b[n] - Ax[n];
    res.residual = std::sqrt(dot(r.data(), r.data()));
    res.relative_residual = res.residual / scale;
    res.converged = res.residual <= atol;
    if (breakdown && !res.converged) break;
  }
  return 0;
}

void pack(const Layout& L, const double* field, double* vec) {
  const long n = L.interior;
  for (int c = 0; c < 3; ++c)
    for (int k = 0; k <= L.nz; ++k)
      for (int j = 0; j <= L.ny; ++j)
        for (int i = 0; i <= L.nx; ++i)
          vec[c * n + i + L.inx * (j + L.iny * (long)k)] = field[c * L.nodes + L.node(i, j, k)];
}
void unpack(const Layout& L, const double* vec, double* field) {
  const long n = L.interior;
  for (int c = 0; c < 3; ++c)
    for (int k = 0; k <= L.nz; ++k)
      for (int j = 0; j <= L.ny; ++j)
        for (int i = 0; i <= L.nx; ++i)
          field[c * L.nodes + L.node(i, j, k)] = vec[c * n + i + L.inx * (j + L.iny * (long)k)];
}

}  // namespace

extern "C" {

struct oracle_grid {
  int nx, ny, nz;
  double dx, dy, dz;
};


static Grid to_grid(const oracle_grid* g) { return {g->nx, g->ny, g->nz, g->dx, g->dy, g->dz}; }

long oracle_node_count(const oracle_grid* g) { return Layout(to_grid(g)).nodes; }
long oracle_cell_count(const oracle_grid* g) { return Layout(to_grid(g)).cells; }
long oracle_bin_count(const oracle_grid* g) { return Layout(to_grid(g)).bins; }
int oracle_pair_stencil(int a, int b) { return pair_stencil(a, b); }
void oracle_stencil_offset(int s, int* out) {
  out[0] = kStencil[s][0]; out[1] = kStencil[s][1]; out[2] = kStencil[s][2];
}

void oracle_cic_weights_f64(double x, double y, double z, double* w) { cic<double>(x, y, z, w); }
void oracle_cic_weights_f32(float x, float y, float z, float* w) { cic<float>(x, y, z, w); }
void oracle_response_f64(double bx, double by, double bz, double boc, double* a) {
  Response<double> r(bx, by, bz, boc);
  std::memcpy(a, r.a, sizeof(r.a));
}
void oracle_response_f32(float bx, float by, float bz, float boc, float* a) {
  Response<float> r(bx, by, bz, boc);
  std::memcpy(a, r.a, sizeof(r.a));
}

// Mover over `count` records. beta = qom*dt/2 and beta/c and 1/spacing are
// formed in double and converted once, as prepare_particle_mover_parameters,
// ecsim/particles/particle_mover_parameters.hpp:23-53. Returns the number of
// invalid records.
long oracle_mover(int precision, const oracle_grid* gp, double qom, double dt, double c, void* rx,
                  void* ry, void* rz, void* u, void* v, void* w, const double* q, int32_t* key,
                  long count, const double* theta, const void* bnode) {
  const Grid g = to_grid(gp);
  const Layout L(g);
  const double beta = qom * dt / 2, boc = beta / c;
  const double inv[3] = {1.0 / g.dx, 1.0 / g.dy, 1.0 / g.dz};
  long invalid = 0;
  if (precision == 0) {
    for (long n = 0; n < count; ++n)
      invalid += push<0>(L, beta, boc, dt, inv, (double*)rx, (double*)ry, (double*)rz, (double*)u,
                         (double*)v, (double*)w, q, key, uint32_t(n), theta, (const double*)bnode);
  } else {
    for (long n = 0; n < count; ++n)
      invalid += push<1>(L, float(beta), float(boc), dt, inv, (double*)rx, (double*)ry, (double*)rz,
                         (float*)u, (float*)v, (float*)w, q, key, uint32_t(n), theta,
                         (const float*)bnode);
  }
  return invalid;
}

// Stable counting sort by cell key over all halo-2 bins, restating
// PreparedSerialParticleSort::run, lpfx/algorithm/particle/host/sort.hpp:205-290:
// histogram, exclusive prefix, ascending-source placement. perm[dest] = source.
// Returns -1 on an out-of-range key.
long oracle_sort(const oracle_grid* gp, const int32_t* keys, long count, uint32_t* perm,
                 uint32_t* counts, uint32_t* offsets) {
  const Layout L(to_grid(gp));
  std::vector<uint64_t> cursor(L.bins, 0);
  for (long s = 0; s < count; ++s) {
    if (keys[s] < 0 || keys[s] >= L.bins) return -1;
    ++cursor[keys[s]];
  }
  uint64_t prefix = 0;
  for (long b = 0; b < L.bins; ++b) {
    const uint64_t n = cursor[b];
    counts[b] = uint32_t(n);
    offsets[b] = uint32_t(prefix);
    cursor[b] = prefix;
    prefix += n;
  }
  offsets[L.bins] = uint32_t(prefix);
  for (long s = 0; s < count; ++s) perm[cursor[keys[s]]++] = uint32_t(s);
  return 0;
}

// Current and mass deposition of one species in FP64 (the reference values
// that the reduced-precision forms state their error against), into the
// cell-local nodes 0..n of J (node field, double) and M (mass records,
// double). Restates evaluate_current_particle / deposit_current_particle,
// ecsim/deposition/current_deposition_device.hpp:64-141, and
// deposit_mass_matrix_particle, ecsim/mass_matrix/mass_matrix_scalar_device.hpp:25-97
// (pair weight (W_a*W_b), alpha*scale with scale = beta/c * q). Either output
// may be null. No fold: call oracle_fold afterwards.
long oracle_deposit(int precision, const oracle_grid* gp, double qom, double dt, double c,
                    const void* rx, const void* ry, const void* rz, const void* u, const void* v,
                    const void* w, const double* q, const int32_t* key, long count,
                    const void* bnode, double* J, double* M) {
  const Grid g = to_grid(gp);
  const Layout L(g);
  const double boc = qom * dt / 2 / c;
  const double inv_volume = 1.0 / ((g.dx * g.dy) * g.dz);
  long invalid = 0;
  int stencil[8][8];
  for (int a = 0; a < 8; ++a)
    for (int b = 0; b < 8; ++b) stencil[a][b] = pair_stencil(a, b);
  auto load = [&](const void* p, long n) {
    return precision == 0 ? ((const double*)p)[n] : double(((const float*)p)[n]);
  };
  for (long n = 0; n < count; ++n) {
    if (key[n] < 0 || key[n] >= L.bins) { ++invalid; continue; }
    int i, j, k;
    L.decode(key[n], i, j, k);
    if (!L.interior_cell(i, j, k)) { ++invalid; continue; }
    const double fx = ((const double*)rx)[n], fy = ((const double*)ry)[n], fz = ((const double*)rz)[n];
    if (!(fx >= 0 && fx < 1 && fy >= 0 && fy < 1 && fz >= 0 && fz < 1)) { ++invalid; continue; }
    double wt[8];
    cic<double>(fx, fy, fz, wt);
    double b[3];
    for (int comp = 0; comp < 3; ++comp) {
      double val = 0;
      for (int a = 0; a < 8; ++a)
        val += wt[a] * load(bnode, comp * L.nodes + L.node(i + (a & 1), j + ((a >> 1) & 1), k + ((a >> 2) & 1)));
      b[comp] = val;
    }
    const Response<double> r(b[0], b[1], b[2], boc);
    if (J) {
      double hx, hy, hz;
      r.apply(load(u, n), load(v, n), load(w, n), hx, hy, hz);
      const double qv = q[n] * inv_volume;
      const double jc[3] = {qv * hx, qv * hy, qv * hz};
      for (int a = 0; a < 8; ++a) {
        const long node = L.node(i + (a & 1), j + ((a >> 1) & 1), k + ((a >> 2) & 1));
        for (int comp = 0; comp < 3; ++comp) J[comp * L.nodes + node] += jc[comp] * wt[a];
      }
    }
    if (M) {
      const double scale = boc * q[n];
      double as[9];
      for (int e = 0; e < 9; ++e) as[e] = r.a[e] * scale;
      for (int a = 0; a < 8; ++a) {
        const long vertex = L.node(i + (a & 1), j + ((a >> 1) & 1), k + ((a >> 2) & 1));
        for (int bb = 0; bb < 8; ++bb) {
          const int s = stencil[a][bb];
          if (s < 0) continue;
          const double pw = wt[a] * wt[bb];
          for (int e = 0; e < 9; ++e) M[vertex * 126 + s * 9 + e] += as[e] * pw;
        }
      }
    }
  }
  return invalid;
}

// Periodic fold of J (shared-node sum, then ghosts) and of the mass records
// (shared-node sum, then ghost records). Either may be null.
void oracle_fold(const oracle_grid* gp, double* J, double* M) {
  const Layout L(to_grid(gp));
  if (J)
    for (int c = 0; c < 3; ++c) {
      fold_add(L, J + c * L.nodes, 1, 1);
      node_ghosts(L, J + c * L.nodes, 1, 1);
    }
  if (M) {
    fold_add(L, M, 126, 126);
    node_ghosts(L, M, 126, 126);
  }
}

// (M*v) at the interior nodes 0..n, times inv_volume (periodic: f_g = 1).
// `in` needs filled ghosts. mass_precision 0 = double records, 1 = float.
void oracle_mass_apply(int mass_precision, const oracle_grid* gp, const void* M, const double* in,
                       double* out) {
  const Grid g = to_grid(gp);
  const Layout L(g);
  const double iv = 1.0 / ((g.dx * g.dy) * g.dz);
  for (int k = 0; k <= L.nz; ++k)
    for (int j = 0; j <= L.ny; ++j)
      for (int i = 0; i <= L.nx; ++i) {
        double o[3];
        if (mass_precision == 0) mass_apply_node(L, (const double*)M, in, i, j, k, iv, o);
        else mass_apply_node(L, (const float*)M, in, i, j, k, iv, o);
        for (int c = 0; c < 3; ++c) out[c * L.nodes + L.node(i, j, k)] = o[c];
      }
}

void oracle_curl_n2c(const oracle_grid* gp, const double* node, double* cellf) {
  const Grid g = to_grid(gp);
  const double inv[3] = {1.0 / g.dx, 1.0 / g.dy, 1.0 / g.dz};
  curl_n2c(Layout(g), node, cellf, inv);
}
void oracle_curl_c2n(const oracle_grid* gp, const double* cellf, double* node) {
  const Grid g = to_grid(gp);
  const double inv[3] = {1.0 / g.dx, 1.0 / g.dy, 1.0 / g.dz};
  curl_c2n(Layout(g), cellf, node, inv);
}
void oracle_cell_to_node(const oracle_grid* gp, const double* cellf, double* node) {
  cell_to_node(Layout(to_grid(gp)), cellf, node);
}
void oracle_node_ghosts(const oracle_grid* gp, double* node) {
  const Layout L(to_grid(gp));
  for (int c = 0; c < 3; ++c) node_ghosts(L, node + c * L.nodes, 1, 1);
}
void oracle_cell_ghosts(const oracle_grid* gp, double* cellf) { cell_ghosts(Layout(to_grid(gp)), cellf); }

// The field solve in FP64: rhs = E + delta*curl_C2N(B) - k*J, then restarted
// GMRES from the initial guess E, restating Gmres::host_blocking_solve,
// ecsim/gmres/gmres_device.hpp:355-454, with the device tails of :52-98
// (classical Gram-Schmidt, Givens rotations, true-residual acceptance).
// E, J: node fields; B: cell field with ghosts; M: double mass records with
// ghosts; theta: node field output (the solution).
// With smooth_iterations > 0 the energy-conserving smoothing of TPIC
// (ECSimSmoothing = energy_conserving): the RHS uses S^n(J) and every apply
// the smoothed schedule (maxwell_device.hpp:152-172,389-432).
int oracle_field_solve_smoothed(const oracle_grid* gp, double dt, double th, double c, const double* E,
                                const double* B, const double* J_in, const double* M, double* theta,
                                int restart, int max_iterations, double tol, int smooth_iterations,
                                double smooth_alpha, int smooth_operator, oracle_gmres_result* out) {
  const Grid g = to_grid(gp);
  const Layout L(g);
  const Physics ph(g, dt, th, c);
  const long N = 3 * L.interior;
  const Smoothing sm{smooth_iterations, smooth_operator, smooth_alpha};
  std::vector<double> curl_node(3 * L.nodes, 0.0), curl_cell(3 * L.cells, 0.0), rhs(3 * L.nodes, 0.0),
      input(3 * L.nodes, 0.0), image(3 * L.nodes, 0.0), smoothed_j;
  const double* J = J_in;
  if (sm.niter > 0) {
    smoothed_j.resize(3 * L.nodes);
    smooth_field(L, sm.niter, sm.op, sm.alpha, J_in, smoothed_j.data());
    J = smoothed_j.data();
  }
  // RHS, maxwell_device.hpp:134-172.
  curl_c2n(L, B, curl_node.data(), ph.inv);
  for (int cc = 0; cc < 3; ++cc)
    for (int k = 0; k <= L.nz; ++k)
      for (int j = 0; j <= L.ny; ++j)
        for (int i = 0; i <= L.nx; ++i) {
          const long at = cc * L.nodes + L.node(i, j, k);
          rhs[at] = (1.0 * E[at] + ph.delta * curl_node[at]) + (-ph.kfac) * J[at];
        }
  std::vector<double> x(N), b(N);
  pack(L, E, x.data());
  pack(L, rhs.data(), b.data());
  auto apply = [&](const double* vec, double* result) {
    unpack(L, vec, input.data());
    maxwell_apply(L, ph, M, input.data(), image.data(), curl_cell.data(), curl_node.data(), sm);
    pack(L, image.data(), result);
  };
  oracle_gmres_result res{};
  if (gmres(apply, b.data(), x.data(), N, restart, max_iterations, tol, res) < 0) return -1;
  // The solution fills theta (interior nodes and ghosts).
  std::fill(theta, theta + 3 * L.nodes, 0.0);
  unpack(L, x.data(), theta);
  for (int cc = 0; cc < 3; ++cc) node_ghosts(L, theta + cc * L.nodes, 1, 1);
  if (out) *out = res;
  return res.converged ? 0 : 1;
}

int oracle_field_solve(const oracle_grid* gp, double dt, double th, double c, const double* E,
                       const double* B, const double* J, const double* M, double* theta,
                       int restart, int max_iterations, double tol, oracle_gmres_result* out) {
  return oracle_field_solve_smoothed(gp, dt, th, c, E, B, J, M, theta, restart, max_iterations, tol, 0, 1.0, 0,
                                     out);
}

// S^niter of a node field (FP64), ghosts filled; the particle field of a
// smoothed run is S^n(theta) (maxwell_device.hpp:213-228).
void oracle_smooth(const oracle_grid* gp, int niter, double alpha, int op, const double* in, double* out) {
  smooth_field(Layout(to_grid(gp)), niter, op, alpha, in, out);
}
// One pass at one node, for the pin against the reference's own operator.
double oracle_smooth_node(const oracle_grid* gp, int op, double alpha, const double* in, int i, int j, int k) {
  const Layout L(to_grid(gp));
  return smooth_value<double>(L, in, i, j, k, op, alpha, (1.0 - alpha) / 6.0);
}

// Field advance, ecsim/maxwell/field_update_device.hpp:25-78 and
// maxwell_device.hpp:234-266: E_new = (1/theta)*Etheta + (-(1-theta)/theta)*E
// (a copy when theta is within 1e-10 of 1); B_next = 1*B + (-c*dt)*curl_N2C(Etheta)
// over all cells, periodic ghosts, B_node = cell_to_node(B_next).
void oracle_field_advance(const oracle_grid* gp, double dt, double th, double c, double* E,
                          const double* B, const double* theta, double* Bnext, double* Bnode) {
  const Grid g = to_grid(gp);
  const Layout L(g);
  const double inv[3] = {1.0 / g.dx, 1.0 / g.dy, 1.0 / g.dz};
  for (int cc = 0; cc < 3; ++cc)
    for (int k = 0; k <= L.nz; ++k)
      for (int j = 0; j <= L.ny; ++j)
        for (int i = 0; i <= L.nx; ++i) {
          const long at = cc * L.nodes + L.node(i, j, k);
          E[at] = std::fabs(th - 1.0) < 1e-10 ? theta[at] : (1.0 / th) * theta[at] + (-(1.0 - th) / th) * E[at];
        }
  for (int cc = 0; cc < 3; ++cc) node_ghosts(L, E + cc * L.nodes, 1, 1);
  const double far = -c * dt;
  for (int k = 0; k < L.nz; ++k)
    for (int j = 0; j < L.ny; ++j)
      for (int i = 0; i < L.nx; ++i) {
        double o[3];
        curl(node_samples(L, theta, i, j, k), node_samples(L, theta + L.nodes, i, j, k),
             node_samples(L, theta + 2 * L.nodes, i, j, k), inv, o);
        for (int cc = 0; cc < 3; ++cc) {
          const long at = cc * L.cells + L.cell(i, j, k);
          Bnext[at] = 1.0 * B[at] + far * o[cc];
        }
      }
  cell_ghosts(L, Bnext);
  cell_to_node(L, Bnext, Bnode);
}

// Energies, diagnostics/scalar_diagnostics_device.hpp:49-133 on a fully
// periodic grid: out[0] = V/(8 pi) sum over unique nodes |E|^2,
// out[1] = V/(8 pi) sum over cells |B|^2.
void oracle_field_energy(const oracle_grid* gp, const double* E, const double* B, double* out) {
  const Grid g = to_grid(gp);
  const Layout L(g);
  const double norm = ((g.dx * g.dy) * g.dz) / (8 * kPi);
  double we = 0, wb = 0;
  for (int k = 0; k < L.nz; ++k)
    for (int j = 0; j < L.ny; ++j)
      for (int i = 0; i < L.nx; ++i) {
        const long n = L.node(i, j, k), cl = L.cell(i, j, k);
        we += E[n] * E[n] + E[L.nodes + n] * E[L.nodes + n] + E[2 * L.nodes + n] * E[2 * L.nodes + n];
        wb += B[cl] * B[cl] + B[L.cells + cl] * B[L.cells + cl] + B[2 * L.cells + cl] * B[2 * L.cells + cl];
      }
  out[0] = norm * we;
  out[1] = norm * wb;
}

// Species scalars, scalar_diagnostics_device.hpp:87-107: kinetic energy,
// charge, momentum x/y/z, with particle mass q/qom.
void oracle_species_scalars(int precision, double qom, const void* u, const void* v, const void* w,
                            const double* q, long count, double* out) {
  double s[5] = {0, 0, 0, 0, 0};
  const double inverse_qom = 1.0 / qom;
  for (long n = 0; n < count; ++n) {
    const double vx = precision == 0 ? ((const double*)u)[n] : double(((const float*)u)[n]);
    const double vy = precision == 0 ? ((const double*)v)[n] : double(((const float*)v)[n]);
    const double vz = precision == 0 ? ((const double*)w)[n] : double(((const float*)w)[n]);
    const double mass = q[n] * inverse_qom;
    s[0] += 0.5 * mass * (vx * vx + vy * vy + vz * vz);
    s[1] += q[n];
    s[2] += mass * vx;
    s[3] += mass * vy;
    s[4] += mass * vz;
  }
  std::memcpy(out, s, sizeof(s));
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Discrete adjoint of one cycle (FP64). TPIC has no adjoint; these functions
// transpose the cycle the functions above restate, so that a gradient of a
// final-state objective is carried back through the cycle:
//   deposit      J_g = sum_p (q/V) W_a(x_p) (alpha_p v_p),
//                M_ab = sum_p (beta/c) q alpha_p W_a W_b     (applied as M v)
//   solve        A E_theta = E + delta C2N(B) - k J,  A = I + delta^2 C2N N2C + (k/V) M
//   mover        v' = 2 alpha (v + beta E_theta(x)) - v,  x' = x + dt v' / dx
//   advance      E' = E_theta/theta - (1-theta)/theta E,  B' = B - c dt N2C(E_theta)
// with alpha = R(omega), omega = (beta/c) B_node(x), B_node = cell_to_node(B).
// The adjoint of a gather at the particle positions is a scatter (then the
// periodic fold), the adjoint of a scatter is a gather, the adjoint of the
// solve is a solve with A^T (every 3x3 mass block transposed; the curl-curl
// part is symmetric because C2N is the transpose of N2C on the periodic
// grid), and N2C^T = C2N, C2N^T = N2C.
// Adjoint node fields are gradients with respect to the unique periodic node
// values, stored like the primal fields (duplicate endpoint nodes and ghosts
// hold copies); scatters accumulate into a zeroed raw field that oracle_fold
// turns into that form. Particle adjoints are indexed by record id, [3][count]
// for positions (per axis, in cells) and velocities, [count] for charges.
// ---------------------------------------------------------------------------

namespace {

struct AdjointParticle {
  int i, j, k;
  double f[3], v[3], w[8], dw[3][8];
};

template <int P>
bool adjoint_load(const Layout& L, const void* rx, const void* ry, const void* rz, const void* u, const void* v,
                  const void* w, const int32_t* key, long n, AdjointParticle& a) {
  using Vel = typename Prec<P>::Vel;
  if (key[n] < 0 || key[n] >= L.bins) return false;
  L.decode(key[n], a.i, a.j, a.k);
  if (!L.interior_cell(a.i, a.j, a.k)) return false;
  a.f[0] = ((const double*)rx)[n];
  a.f[1] = ((const double*)ry)[n];
  a.f[2] = ((const double*)rz)[n];
  a.v[0] = double(((const Vel*)u)[n]);
  a.v[1] = double(((const Vel*)v)[n]);
  a.v[2] = double(((const Vel*)w)[n]);
  cic<double>(a.f[0], a.f[1], a.f[2], a.w);
  for (int c = 0; c < 8; ++c) {
    const double X[2] = {1 - a.f[0], a.f[0]}, Y[2] = {1 - a.f[1], a.f[1]}, Z[2] = {1 - a.f[2], a.f[2]};
    const int bx = c & 1, by = (c >> 1) & 1, bz = (c >> 2) & 1;
    const double sx = bx ? 1.0 : -1.0, sy = by ? 1.0 : -1.0, sz = bz ? 1.0 : -1.0;
    a.dw[0][c] = sx * Y[by] * Z[bz];
    a.dw[1][c] = X[bx] * sy * Z[bz];
    a.dw[2][c] = X[bx] * Y[by] * sz;
  }
  return true;
}

template <class F>
void adjoint_gather(const Layout& L, const F* field, const AdjointParticle& a, double out[3]) {
  for (int c = 0; c < 3; ++c) {
    double val = 0;
    for (int b = 0; b < 8; ++b)
      val += a.w[b] * double(field[c * L.nodes + L.node(a.i + (b & 1), a.j + ((b >> 1) & 1), a.k + ((b >> 2) & 1))]);
    out[c] = val;
  }
}

// sum_b dW_b/dx_axis * (field_b . g) for the three axes.
template <class F>
void adjoint_position_term(const Layout& L, const F* field, const AdjointParticle& a, const double g[3],
                           double out[3]) {
  for (int b = 0; b < 8; ++b) {
    const long node = L.node(a.i + (b & 1), a.j + ((b >> 1) & 1), a.k + ((b >> 2) & 1));
    double dotv = 0;
    for (int c = 0; c < 3; ++c) dotv += double(field[c * L.nodes + node]) * g[c];
    for (int axis = 0; axis < 3; ++axis) out[axis] += a.dw[axis][b] * dotv;
  }
}

void adjoint_scatter(const Layout& L, double* field, const AdjointParticle& a, const double g[3]) {
  for (int b = 0; b < 8; ++b) {
    const long node = L.node(a.i + (b & 1), a.j + ((b >> 1) & 1), a.k + ((b >> 2) & 1));
    for (int c = 0; c < 3; ++c) field[c * L.nodes + node] += a.w[b] * g[c];
  }
}

// R^T g
void transpose_apply(const double r[9], const double g[3], double out[3]) {
  out[0] = r[0] * g[0] + r[3] * g[1] + r[6] * g[2];
  out[1] = r[1] * g[0] + r[4] * g[1] + r[7] * g[2];
  out[2] = r[2] * g[0] + r[5] * g[1] + r[8] * g[2];
}

// Gradient with respect to omega of sum_ij abar_ij R_ij(omega), R = (I +
// omega omega^T + K(omega)) / (1 + |omega|^2) with K the antisymmetric part of
// ParticleResponse (K_01 = wz, K_02 = -wy, K_12 = wx).
void response_omega_gradient(const double om[3], const double r[9], const double ab[9], double out[3]) {
  const double D = 1 + om[0] * om[0] + om[1] * om[1] + om[2] * om[2];
  double ar = 0;
  for (int e = 0; e < 9; ++e) ar += ab[e] * r[e];
  const double kx = ab[5] - ab[7], ky = ab[6] - ab[2], kz = ab[1] - ab[3];
  const double kk[3] = {kx, ky, kz};
  for (int c = 0; c < 3; ++c) {
    double sym = 0;
    for (int e = 0; e < 3; ++e) sym += (ab[3 * c + e] + ab[3 * e + c]) * om[e];
    out[c] = (sym + kk[c]) / D - 2 * om[c] * ar / D;
  }
}

template <int P>
long adjoint_mover_scatter(const Layout& L, const Grid& g, double qom, double dt, double c, const void* rx,
                           const void* ry, const void* rz, const void* u, const void* v, const void* w,
                           const int32_t* key, const uint64_t* id, long count, long nid, const double* xbar,
                           const double* vbar, const double* theta, const void* bnode, double* scatter) {
  using Fld = typename Prec<P>::Fld;
  const double beta = qom * dt / 2, boc = beta / c;
  const double inv[3] = {1.0 / g.dx, 1.0 / g.dy, 1.0 / g.dz};
  long invalid = 0;
  for (long n = 0; n < count; ++n) {
    AdjointParticle a;
    if (!adjoint_load<P>(L, rx, ry, rz, u, v, w, key, n, a) || id[n] >= uint64_t(nid)) { ++invalid; continue; }
    const long pid = long(id[n]);
    double bp[3];
    adjoint_gather(L, (const Fld*)bnode, a, bp);
    const Response<double> r(bp[0], bp[1], bp[2], boc);
    double gv[3], eb[3];
    for (int cc = 0; cc < 3; ++cc) gv[cc] = 2 * (vbar[cc * nid + pid] + dt * inv[cc] * xbar[cc * nid + pid]);
    transpose_apply(r.a, gv, eb);
    for (int cc = 0; cc < 3; ++cc) eb[cc] *= beta;
    adjoint_scatter(L, scatter, a, eb);
  }
  return invalid;
}

template <int P>
long adjoint_particles(const Layout& L, const Grid& g, double qom, double dt, double theta_, double c,
                       const void* rx, const void* ry, const void* rz, const void* u, const void* v, const void* w,
                       const double* q, const int32_t* key, const uint64_t* id, long count, long nid, double* xbar,
                       double* vbar, double* qbar, const double* theta, const void* bnode, const double* lambda,
                       double* bscatter) {
  using Fld = typename Prec<P>::Fld;
  const double beta = qom * dt / 2, boc = beta / c;
  const double inv[3] = {1.0 / g.dx, 1.0 / g.dy, 1.0 / g.dz};
  const double volume = (g.dx * g.dy) * g.dz, iv = 1.0 / volume;
  const double kfac = 4 * kPi * (theta_ * dt);
  long invalid = 0;
  for (long n = 0; n < count; ++n) {
    AdjointParticle a;
    if (!adjoint_load<P>(L, rx, ry, rz, u, v, w, key, n, a) || id[n] >= uint64_t(nid)) { ++invalid; continue; }
    const long pid = long(id[n]);
    double bp[3], ep[3], lp[3];
    adjoint_gather(L, (const Fld*)bnode, a, bp);
    adjoint_gather(L, theta, a, ep);
    adjoint_gather(L, lambda, a, lp);
    const Response<double> r(bp[0], bp[1], bp[2], boc);
    const double om[3] = {boc * bp[0], boc * bp[1], boc * bp[2]};
    double xb[3], vt[3], gv[3];
    for (int cc = 0; cc < 3; ++cc) {
      xb[cc] = xbar[cc * nid + pid];
      vt[cc] = vbar[cc * nid + pid] + dt * inv[cc] * xb[cc];
      gv[cc] = 2 * vt[cc];
    }
    double ab[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    double vn[3], t[3];
    // Mover: v' = 2 R (v + beta E_theta) - v, x' = x + dt v' / dx.
    transpose_apply(r.a, gv, t);
    double eb[3];
    for (int cc = 0; cc < 3; ++cc) {
      vn[cc] = -vt[cc] + t[cc];
      eb[cc] = beta * t[cc];
    }
    const double uu[3] = {a.v[0] + beta * ep[0], a.v[1] + beta * ep[1], a.v[2] + beta * ep[2]};
    for (int r0 = 0; r0 < 3; ++r0)
      for (int c0 = 0; c0 < 3; ++c0) ab[3 * r0 + c0] += gv[r0] * uu[c0];
    adjoint_position_term(L, theta, a, eb, xb);
    // Current: J = sum (q/V) W (R v); its gradient is -k lambda (the RHS).
    double h[3];
    r.apply(a.v[0], a.v[1], a.v[2], h[0], h[1], h[2]);
    const double jb[3] = {-kfac * lp[0], -kfac * lp[1], -kfac * lp[2]};
    const double qv = q[n] * iv;
    transpose_apply(r.a, jb, t);
    for (int cc = 0; cc < 3; ++cc) vn[cc] += qv * t[cc];
    for (int r0 = 0; r0 < 3; ++r0)
      for (int c0 = 0; c0 < 3; ++c0) ab[3 * r0 + c0] += qv * jb[r0] * a.v[c0];
    double qb = iv * (jb[0] * h[0] + jb[1] * h[1] + jb[2] * h[2]);
    {
      const double hq[3] = {-kfac * qv * h[0], -kfac * qv * h[1], -kfac * qv * h[2]};
      adjoint_position_term(L, lambda, a, hq, xb);
    }
    // Mass: -(k/V) lambda^T M E_theta = -(k/V) sum_p s lambda_p^T R e_p, s = (beta/c) q.
    const double cm = -kfac * iv, sq = boc * q[n];
    double re[3];
    r.apply(ep[0], ep[1], ep[2], re[0], re[1], re[2]);
    qb += cm * boc * (lp[0] * re[0] + lp[1] * re[1] + lp[2] * re[2]);
    for (int r0 = 0; r0 < 3; ++r0)
      for (int c0 = 0; c0 < 3; ++c0) ab[3 * r0 + c0] += cm * sq * lp[r0] * ep[c0];
    {
      const double g1[3] = {cm * sq * re[0], cm * sq * re[1], cm * sq * re[2]};
      adjoint_position_term(L, lambda, a, g1, xb);
      double rl[3];
      transpose_apply(r.a, lp, rl);
      const double g2[3] = {cm * sq * rl[0], cm * sq * rl[1], cm * sq * rl[2]};
      adjoint_position_term(L, theta, a, g2, xb);
    }
    // The response's dependence on B at the particle.
    double ob[3];
    response_omega_gradient(om, r.a, ab, ob);
    const double bb[3] = {boc * ob[0], boc * ob[1], boc * ob[2]};
    adjoint_scatter(L, bscatter, a, bb);
    adjoint_position_term(L, (const Fld*)bnode, a, bb, xb);
    for (int cc = 0; cc < 3; ++cc) {
      xbar[cc * nid + pid] = xb[cc];
      vbar[cc * nid + pid] = vn[cc];
    }
    qbar[pid] += qb;
  }
  return invalid;
}

}  // namespace

extern "C" {

// Adjoint of the field advance: e_theta_bar = e_bar'/theta - c dt C2N(b_bar')
// (e_bar' when theta is 1), e_bar = -(1-theta)/theta e_bar' (0 when theta is
// 1), b_bar = b_bar'. b_bar_next needs filled ghosts; outputs are consistent
// node fields / a cell field with ghosts.
void oracle_adjoint_advance(const oracle_grid* gp, double dt, double th, double c, const double* e_bar_next,
                            const double* b_bar_next, double* e_theta_bar, double* e_bar, double* b_bar) {
  const Grid g = to_grid(gp);
  const Layout L(g);
  const double inv[3] = {1.0 / g.dx, 1.0 / g.dy, 1.0 / g.dz};
  std::vector<double> curl_node(3 * L.nodes, 0.0);
  curl_c2n(L, b_bar_next, curl_node.data(), inv);
  const bool one = std::fabs(th - 1.0) < 1e-10;
  for (int cc = 0; cc < 3; ++cc)
    for (int k = 0; k <= L.nz; ++k)
      for (int j = 0; j <= L.ny; ++j)
        for (int i = 0; i <= L.nx; ++i) {
          const long at = cc * L.nodes + L.node(i, j, k);
          e_theta_bar[at] = (one ? e_bar_next[at] : e_bar_next[at] / th) + (-c * dt) * curl_node[at];
          e_bar[at] = one ? 0.0 : (-(1.0 - th) / th) * e_bar_next[at];
        }
  for (int cc = 0; cc < 3; ++cc) {
    node_ghosts(L, e_theta_bar + cc * L.nodes, 1, 1);
    node_ghosts(L, e_bar + cc * L.nodes, 1, 1);
  }
  std::copy(b_bar_next, b_bar_next + 3 * L.cells, b_bar);
  cell_ghosts(L, b_bar);
}

// Scatter of the mover's E_theta gradient (raw node field, add): per record,
// W_a(x) beta R^T (2 (v_bar' + dt x_bar' / dx)). Returns the invalid records.
long oracle_adjoint_mover_scatter(int precision, const oracle_grid* gp, double qom, double dt, double c,
                                  const void* rx, const void* ry, const void* rz, const void* u, const void* v,
                                  const void* w, const int32_t* key, const uint64_t* id, long count, long nid,
                                  const double* xbar, const double* vbar, const double* theta, const void* bnode,
                                  double* scatter) {
  const Grid g = to_grid(gp);
  const Layout L(g);
  return precision == 0
             ? adjoint_mover_scatter<0>(L, g, qom, dt, c, rx, ry, rz, u, v, w, key, id, count, nid, xbar, vbar,
                                        theta, bnode, scatter)
             : adjoint_mover_scatter<1>(L, g, qom, dt, c, rx, ry, rz, u, v, w, key, id, count, nid, xbar, vbar,
                                        theta, bnode, scatter);
}

// Per record: the adjoints of the mover and of its current and mass
// deposition at the cycle start, x_bar and v_bar replaced (by id), q_bar
// accumulated, the B gradient scattered into bscatter (raw node field, add).
long oracle_adjoint_particles(int precision, const oracle_grid* gp, double qom, double dt, double th, double c,
                              const void* rx, const void* ry, const void* rz, const void* u, const void* v,
                              const void* w, const double* q, const int32_t* key, const uint64_t* id, long count,
                              long nid, double* xbar, double* vbar, double* qbar, const double* theta,
                              const void* bnode, const double* lambda, double* bscatter) {
  const Grid g = to_grid(gp);
  const Layout L(g);
  return precision == 0
             ? adjoint_particles<0>(L, g, qom, dt, th, c, rx, ry, rz, u, v, w, q, key, id, count, nid, xbar, vbar,
                                    qbar, theta, bnode, lambda, bscatter)
             : adjoint_particles<1>(L, g, qom, dt, th, c, rx, ry, rz, u, v, w, q, key, id, count, nid, xbar, vbar,
                                    qbar, theta, bnode, lambda, bscatter);
}

// The adjoint solve A^T lambda = rhs (rhs a consistent node field) by the
// GMRES above from a zero guess; lambda gets its ghosts.
int oracle_adjoint_solve(const oracle_grid* gp, double dt, double th, double c, const double* M, const double* rhs,
                         double* lambda, int restart, int max_iterations, double tol, oracle_gmres_result* out) {
  const Grid g = to_grid(gp);
  const Layout L(g);
  const Physics ph(g, dt, th, c);
  const long N = 3 * L.interior;
  std::vector<double> curl_node(3 * L.nodes, 0.0), curl_cell(3 * L.cells, 0.0), input(3 * L.nodes, 0.0),
      image(3 * L.nodes, 0.0);
  std::vector<double> x(N, 0.0), b(N);
  pack(L, rhs, b.data());
  auto apply = [&](const double* vec, double* result) {
    unpack(L, vec, input.data());
    maxwell_apply(L, ph, M, input.data(), image.data(), curl_cell.data(), curl_node.data(), Smoothing{}, true);
    pack(L, image.data(), result);
  };
  oracle_gmres_result res{};
  if (gmres(apply, b.data(), x.data(), N, restart, max_iterations, tol, res) < 0) return -1;
  std::fill(lambda, lambda + 3 * L.nodes, 0.0);
  unpack(L, x.data(), lambda);
  for (int cc = 0; cc < 3; ++cc) node_ghosts(L, lambda + cc * L.nodes, 1, 1);
  if (out) *out = res;
  return res.converged ? 0 : 1;
}

// The field part after the solve: e_bar += lambda (the RHS's E term);
// b_bar += delta N2C(lambda) (C2N^T) + cell_to_node^T(bnode_bar), with
// bnode_bar a consistent node field; b_bar's ghosts refilled.
void oracle_adjoint_fields(const oracle_grid* gp, double dt, double th, double c, const double* lambda,
                           const double* bnode_bar, double* e_bar, double* b_bar) {
  const Grid g = to_grid(gp);
  const Layout L(g);
  const Physics ph(g, dt, th, c);
  for (int cc = 0; cc < 3; ++cc) {
    for (int k = 0; k <= L.nz; ++k)
      for (int j = 0; j <= L.ny; ++j)
        for (int i = 0; i <= L.nx; ++i) {
          const long at = cc * L.nodes + L.node(i, j, k);
          e_bar[at] += lambda[at];
        }
    node_ghosts(L, e_bar + cc * L.nodes, 1, 1);
  }
  std::vector<double> curl_cell(3 * L.cells, 0.0);
  curl_n2c(L, lambda, curl_cell.data(), ph.inv);
  for (int cc = 0; cc < 3; ++cc)
    for (int k = 0; k < L.nz; ++k)
      for (int j = 0; j < L.ny; ++j)
        for (int i = 0; i < L.nx; ++i) {
          const long cl = cc * L.cells + L.cell(i, j, k);
          double sum = 0;
          // cell_to_node^T: the cell receives 1/8 of each unique node whose
          // average reads it (nodes i..i+1 per axis, folded periodically).
          for (int b = 0; b < 8; ++b) {
            int ni = i + (b & 1), nj = j + ((b >> 1) & 1), nk = k + ((b >> 2) & 1);
            if (ni == L.nx) ni = 0;
            if (nj == L.ny) nj = 0;
            if (nk == L.nz) nk = 0;
            sum += bnode_bar[cc * L.nodes + L.node(ni, nj, nk)];
          }
          b_bar[cl] += ph.delta * curl_cell[cl] + 0.125 * sum;
        }
  cell_ghosts(L, b_bar);
}

// Gradient of we * W_E + wb * W_B (the energies of oracle_field_energy) with
// respect to E at the unique nodes and B at the cells: e_bar = we V/(4 pi) E,
// b_bar = wb V/(4 pi) B, stored as consistent fields.
void oracle_energy_gradient(const oracle_grid* gp, double we, double wb, const double* E, const double* B,
                            double* e_bar, double* b_bar) {
  const Grid g = to_grid(gp);
  const Layout L(g);
  const double norm = ((g.dx * g.dy) * g.dz) / (4 * kPi);
  std::fill(e_bar, e_bar + 3 * L.nodes, 0.0);
  std::fill(b_bar, b_bar + 3 * L.cells, 0.0);
  for (int cc = 0; cc < 3; ++cc) {
    for (int k = 0; k < L.nz; ++k)
      for (int j = 0; j < L.ny; ++j)
        for (int i = 0; i < L.nx; ++i) {
          const long n = cc * L.nodes + L.node(i, j, k), cl = cc * L.cells + L.cell(i, j, k);
          e_bar[n] = we * norm * E[n];
          b_bar[cl] = wb * norm * B[cl];
        }
    // Duplicate endpoint nodes take their unique node's value, then ghosts.
    double* f = e_bar + cc * L.nodes;
    for (int k = 0; k <= L.nz; ++k)
      for (int j = 0; j <= L.ny; ++j)
        for (int i = 0; i <= L.nx; ++i)
          f[L.node(i, j, k)] = f[L.node(i == L.nx ? 0 : i, j == L.ny ? 0 : j, k == L.nz ? 0 : k)];
    node_ghosts(L, f, 1, 1);
  }
  cell_ghosts(L, b_bar);
}

}  // extern "C"
