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
template <class M>
void mass_apply_node(const Layout& L, const M* mass, const double* in, int i, int j, int k,
                     double row_inverse_volume, double out[3]) {
  const long nn = L.nodes;
  auto block = [&](long vertex, int s, long at, double& x, double& y, double& z) {
    const M* b = mass + vertex * 126 + s * 9;
    const double vx = in[at], vy = in[nn + at], vz = in[2 * nn + at];
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
                   double* curl_cell, double* curl_node, const Smoothing& sm = Smoothing{}) {
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
          mass_apply_node(L, mass, in, i, j, k, ph.inv_volume, m);
        for (int c = 0; c < 3; ++c) {
          const long at = c * L.nodes + g;
          image[at] = (1.0 * in[at] + d2 * curl_node[at]) + ph.kfac * m[c];
        }
      }
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

struct oracle_gmres_result {
  int converged, iterations;
  double initial_residual, residual, rhs_norm, relative_residual;
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
  std::vector<double> x(N), b(N), r(N), Ax(N), w(N);
  std::vector<double> V((size_t)(restart + 1) * N);
  std::vector<double> H((size_t)restart * (restart + 1)), cs(restart), sn(restart), s(restart + 1),
      y(restart);
  pack(L, E, x.data());
  pack(L, rhs.data(), b.data());
  auto apply = [&](const double* vec, double* result) {
    unpack(L, vec, input.data());
    maxwell_apply(L, ph, M, input.data(), image.data(), curl_cell.data(), curl_node.data(), sm);
    pack(L, image.data(), result);
  };
  auto dot = [&](const double* a, const double* bb) {
    double sum = 0;
    for (long n = 0; n < N; ++n) sum += a[n] * bb[n];
    return sum;
  };
  apply(x.data(), Ax.data());
  for (long n = 0; n < N; ++n) r[n] = b[n] - Ax[n];
  oracle_gmres_result res{};
  res.residual = res.initial_residual = std::sqrt(dot(r.data(), r.data()));
  res.rhs_norm = std::sqrt(dot(b.data(), b.data()));
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
    apply(x.data(), Ax.data());
    for (long n = 0; n < N; ++n) r[n] = b[n] - Ax[n];
    res.residual = std::sqrt(dot(r.data(), r.data()));
    res.relative_residual = res.residual / scale;
    res.converged = res.residual <= atol;
    if (breakdown && !res.converged) break;
  }
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
