// Pin harness: exports the reference's own header-only numerics, compiled by
// g++ from the TPIC source tree, so that the tests can check the oracle's
// restatement against them. TEST INFRASTRUCTURE ONLY; built into oracle/_ref/
// by oracle/Makefile when the reference tree is present. Nothing here is
// copied from the reference: the functions below only call its headers.
//
// Wrapped reference entry points:
//   make_cic_weights               ecsim/particles/cic.hpp:24-36
//   ParticleResponse               ecsim/particles/particle_response.hpp:16-42
//   mass_pair_stencil              ecsim/mass_matrix/mass_matrix_stencil.hpp:37-40
//   apply_mass_matrix_node         ecsim/mass_matrix/mass_matrix_stencil.hpp:119-149
//   node_cell_curl                 ecsim/fields/node_cell_curl.hpp:116-126
//   cell_to_node_average           ecsim/fields/cell_to_node.hpp:19-32
//   ParticleCellMap encode/decode  data/particles/particle_cell.hpp:34-46
//   node_smoothing_value           ecsim/fields/node_smoothing.hpp:24-52
//   PreparedSerialParticleSort     lpfx/algorithm/particle/host/sort.hpp:180-290
#include <tpic/data/mass_matrix/mass_matrix_layout.hpp>
#include <tpic/data/particles/particle_cell.hpp>
#include <tpic/ecsim/fields/cell_to_node.hpp>
#include <tpic/ecsim/fields/node_cell_curl.hpp>
#include <tpic/ecsim/fields/node_smoothing.hpp>
#include <tpic/ecsim/mass_matrix/mass_matrix_stencil.hpp>
#include <tpic/ecsim/particles/cic.hpp>
#include <tpic/ecsim/particles/particle_response.hpp>
#include <lpfx/algorithm/particle/host/sort.hpp>
#include <lpfx/api/particle/host_particles.hpp>

#include <cstdint>
#include <cstring>

namespace {

// A component view in the layout of include/tpicb200.h (one-node or one-cell
// halo, x fastest), with the location tag the reference's stencils require.
template <class Location> struct Component {
  using location_type = Location;
  using value_type = double;
  const double* values;
  long ex, ey;
  double operator()(int i, int j, int k) const {
    return values[(i + 1) + ex * ((j + 1) + ey * long(k + 1))];
  }
};

template <class Location> struct Vector {
  static constexpr std::size_t component_count = 3;
  Component<Location> c[3];
  template <std::size_t I> Component<Location> component() const { return c[I]; }
};

// A two-attribute host schema for the stable serial sort: the int32 cell key
// and the record's input index, whose sorted order is the permutation.
using SortKeyAttribute = lpfx::particle::attribute<"cell", std::int32_t>;
using SortIndexAttribute = lpfx::particle::attribute<"source", std::uint32_t>;
using SortSchema = lpfx::particle::schema<SortKeyAttribute, SortIndexAttribute>;
using SortPolicy = lpfx::BasicParticleSortIndexPolicy<std::uint32_t, std::uint32_t, std::uint32_t, std::uint32_t>;
using SortKeyAccessor = lpfx::ParticleAttributeKey<SortKeyAttribute::name_type>;

}  // namespace

extern "C" {

// The reference's PreparedSerialParticleSort::run on `count` keys over
// `bins` direct-cell bins: perm[dest] = source, counts and offsets of the
// published bins. Returns the lpfx::ErrorCode value (0 = success), or -1
// when the owners could not be built.
int ref_serial_sort(const int32_t* keys, long count, long bins, uint32_t* perm, uint32_t* counts,
                    uint32_t* offsets) {
  auto made = lpfx::particle::make<SortSchema>({std::size_t(count), std::size_t(count)});
  if (!made.has_value()) return -1;
  auto particles = std::move(made).value();
  {
    auto view = particles.view();
    auto key = view.template get<0>();
    auto source = view.template get<1>();
    for (long n = 0; n < count; ++n) {
      key[n] = keys[n];
      source[n] = std::uint32_t(n);
    }
  }
  lpfx::HostMemoryBudget budget;
  if (!budget.try_set_limit(std::size_t(1) << 40) || !budget.seal()) return -1;
  lpfx::PreparedCellBins<std::uint32_t, std::uint32_t> prepared_bins{};
  if (lpfx::try_prepare_cell_bins(bins, prepared_bins) != lpfx::ErrorCode::success) return -1;
  auto made_bins = lpfx::make_host_cell_bins(budget, prepared_bins);
  if (!made_bins.has_value()) return -1;
  auto cell_bins = std::move(made_bins).value();
  lpfx::PreparedSerialParticleSortWorkspace<SortPolicy> prepared_workspace{};
  if (lpfx::try_prepare_serial_particle_sort_workspace<SortPolicy>(bins, particles.capacity(), prepared_workspace) !=
      lpfx::ErrorCode::success)
    return -1;
  auto made_workspace = lpfx::make_host_serial_particle_sort_workspace(budget, prepared_workspace);
  if (!made_workspace.has_value()) return -1;
  auto workspace = std::move(made_workspace).value();
  lpfx::DirectCellBinLayout<std::int32_t> layout{};
  if (!lpfx::try_make_direct_cell_bin_layout<std::int32_t>(bins, layout)) return -1;
  lpfx::PreparedSerialParticleSort<SortSchema, SortKeyAccessor, SortPolicy> sort{};
  if (lpfx::try_prepare_serial_particle_sort(particles, cell_bins, workspace, layout, sort) != lpfx::ErrorCode::success)
    return -1;
  const lpfx::ErrorCode status = sort.run();
  if (status != lpfx::ErrorCode::success) return int(status);
  const auto view = std::as_const(particles).view();
  const auto source = view.template get<1>();
  for (long n = 0; n < count; ++n) perm[n] = source[n];
  lpfx::CellBinsView<std::uint32_t, std::uint32_t> published{};
  if (!cell_bins.try_completed_view(published)) return -1;
  for (long b = 0; b < bins; ++b) counts[b] = published.counts()[b];
  for (long b = 0; b <= bins; ++b) offsets[b] = published.offsets()[b];
  return 0;
}

void ref_cic_weights_f64(double x, double y, double z, double* w) {
  const auto r = tpic::ecsim::make_cic_weights<double>(x, y, z);
  std::memcpy(w, r.value, sizeof(r.value));
}
void ref_cic_weights_f32(float x, float y, float z, float* w) {
  const auto r = tpic::ecsim::make_cic_weights<float>(x, y, z);
  std::memcpy(w, r.value, sizeof(r.value));
}
void ref_response_f64(double bx, double by, double bz, double boc, double* a) {
  const tpic::ecsim::ParticleResponse<double> r(bx, by, bz, boc);
  std::memcpy(a, r.a, sizeof(r.a));
}
void ref_response_f32(float bx, float by, float bz, float boc, float* a) {
  const tpic::ecsim::ParticleResponse<float> r(bx, by, bz, boc);
  std::memcpy(a, r.a, sizeof(r.a));
}
int ref_pair_stencil(int a, int b) { return tpic::ecsim::mass_pair_stencil(a, b); }
void ref_stencil_offset(int s, int* out) {
  const auto o = tpic::data::mass_stencil_offset(s);
  out[0] = o.i; out[1] = o.j; out[2] = o.k;
}

int ref_encode_key(int nx, int ny, int nz, int i, int j, int k) {
  const tpic::data::ParticleCellMap map{nx, ny, nz, nx + 4, ny + 4, (nx + 4) * (ny + 4) * (nz + 4)};
  return map.encode(i, j, k);
}
void ref_decode_key(int nx, int ny, int nz, int key, int* out) {
  const tpic::data::ParticleCellMap map{nx, ny, nz, nx + 4, ny + 4, (nx + 4) * (ny + 4) * (nz + 4)};
  const auto c = map.decode(key);
  out[0] = c.i; out[1] = c.j; out[2] = c.k;
}

// Curl of a node field at cell (i,j,k) (N2C) or of a cell field at node
// (i,j,k) (C2N). Fields are 3 x count component-major arrays.
void ref_curl_n2c(int nx, int ny, int nz, const double* node, double ix, double iy, double iz,
                  int i, int j, int k, double* out) {
  const long ex = nx + 3, ey = ny + 3, count = ex * ey * (nz + 3L);
  const Vector<lpfx::Node> v{{{node, ex, ey}, {node + count, ex, ey}, {node + 2 * count, ex, ey}}};
  const auto c = tpic::ecsim::node_cell_curl(v, i, j, k, tpic::ecsim::NodeCellSpacing<double>{ix, iy, iz});
  out[0] = c.x; out[1] = c.y; out[2] = c.z;
}
void ref_curl_c2n(int nx, int ny, int nz, const double* cell, double ix, double iy, double iz,
                  int i, int j, int k, double* out) {
  const long ex = nx + 2, ey = ny + 2, count = ex * ey * (nz + 2L);
  const Vector<lpfx::Cell> v{{{cell, ex, ey}, {cell + count, ex, ey}, {cell + 2 * count, ex, ey}}};
  const auto c = tpic::ecsim::node_cell_curl(v, i, j, k, tpic::ecsim::NodeCellSpacing<double>{ix, iy, iz});
  out[0] = c.x; out[1] = c.y; out[2] = c.z;
}
double ref_cell_to_node(int nx, int ny, const double* cell, int i, int j, int k) {
  const Component<lpfx::Cell> c{cell, nx + 2L, ny + 2L};
  return tpic::ecsim::cell_to_node_average<double>(c, i, j, k);
}

// One smoothing pass at node (i,j,k) of a node component with its one-node
// halo: op 0 Face7 (centre weight alpha, faces (1 - alpha)/6), 1 Binomial27.
double ref_smooth_node(int nx, int ny, int op, double alpha, const double* node, int i, int j, int k) {
  using Op = tpic::config::EcsimSmoothingOperator;
  const Component<lpfx::Node> c{node, nx + 3L, ny + 3L};
  if (op == 0)
    return tpic::ecsim::node_smoothing_value<Op::Face7, double>(
        c, i, j, k, tpic::ecsim::SmoothingWeights<Op::Face7, double>{alpha, (1.0 - alpha) / 6.0});
  return tpic::ecsim::node_smoothing_value<Op::Binomial27, double>(
      c, i, j, k, tpic::ecsim::SmoothingWeights<Op::Binomial27, double>{});
}

// (M v) at node (i,j,k) with the reference's compact layout and apply order.
void ref_mass_apply_node(int nx, int ny, int nz, const double* mass, const double* in,
                         double row_inverse_volume, int i, int j, int k, double* out) {
  const int ex = nx + 3, ey = ny + 3, ez = nz + 3;
  const tpic::data::MassMatrixLayout layout{nx + 1, ny + 1, nz + 1, ex, ey, ez, ex, ex * ey,
                                            (nx + 1) * (ny + 1) * (nz + 1), ex * ey * ez};
  const long count = long(ex) * ey * ez;
  const Component<lpfx::Node> vx{in, ex, ey}, vy{in + count, ex, ey}, vz{in + 2 * count, ex, ey};
  double x, y, z;
  tpic::ecsim::apply_mass_matrix_node(mass, layout, vx, vy, vz, i, j, k, row_inverse_volume, x, y, z);
  out[0] = x; out[1] = y; out[2] = z;
}

}  // extern "C"
