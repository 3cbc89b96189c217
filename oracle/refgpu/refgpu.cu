// GPU comparator harness (test infrastructure): launches the reference's own
// device kernels, compiled from its headers for sm_100a, on caller-owned
// device buffers in the layouts of include/tpicb200.h, so that the tests can
// check the library against the reference's kernels on the same inputs and
// time both on the same GPU. Nothing in the library links or calls this.
//
// Kernels (the reference's launch shapes: 128 threads, one warp per bin or
// interior cell, at most 65535 blocks; lpfx/backend/launch.hpp:27-53):
//   sorted_current_kernel          ecsim/deposition/current_deposition_device.hpp:168
//   sorted_mass_matrix_scalar_kernel ecsim/mass_matrix/mass_matrix_scalar_device.hpp:122
//   sorted_mass_matrix_mma_kernel  ecsim/mass_matrix/mass_matrix_mma_device.hpp:58 (FP64 mma.sync)
//   sorted_particle_mover_kernel   ecsim/particles/particle_mover_device.hpp:157
// Precision levels: 0 = double storage and compute; 1 = single particles,
// moments and fields (config/precision.hpp); 2 = level 1 with double mass
// (the float level that admits the FP64 matrix-core mass kernel).
#include <tpic/config/precision.hpp>
#include <tpic/communication/particles/local_particle_destination_sink_device.hpp>
#include <tpic/communication/particles/particle_geometry.hpp>
#include <tpic/ecsim/deposition/current_deposition_device.hpp>
#include <tpic/ecsim/mass_matrix/mass_matrix_deposition_device.hpp>
#include <tpic/ecsim/particles/particle_mover_device.hpp>

#include <cstdint>
#include <type_traits>

namespace {

namespace cfg = tpic::config;
using Level0 = cfg::Precision<cfg::StorageDouble, cfg::ComputeDouble>;
using Level1 = cfg::Precision<cfg::StorageSingleParticlesMomentsFields, cfg::ComputeSingleParticlesMomentsFields>;
using Level2 = cfg::Precision<cfg::StorageSingleParticlesMomentsFieldsDoubleMass,
                              cfg::ComputeSingleParticlesMomentsFieldsDoubleMass>;

constexpr unsigned kThreads = 128;       // tpic::device::particle_block_threads
constexpr unsigned kWarpsPerBlock = 4;   // sorted_cell_max_warps
constexpr unsigned kBlockLimit = 65535;  // lpfx::device::kernel_grid_block_limit

unsigned blocks_for(unsigned long long work) {
  const unsigned long long wanted = (work + kWarpsPerBlock - 1) / kWarpsPerBlock;
  return unsigned(wanted < kBlockLimit ? (wanted ? wanted : 1) : kBlockLimit);
}

// One species' records (SoA) as the reference's particle views expose them.
template <class Precision> struct Records {
  using S = tpic::data::ParticleSchema<Precision>;
  using Pos = typename Precision::Storage::Position;
  using Vel = typename Precision::Storage::Velocity;
  using Wt = typename Precision::Storage::Weight;
  Pos *rx, *ry, *rz;
  Vel *u, *v, *w;
  Wt* q;
  std::int32_t* cell;
  std::uint64_t* id;
  template <class Tag> __host__ __device__ auto get() const {
    if constexpr (std::is_same_v<Tag, typename S::Rx>) return rx;
    else if constexpr (std::is_same_v<Tag, typename S::Ry>) return ry;
    else if constexpr (std::is_same_v<Tag, typename S::Rz>) return rz;
    else if constexpr (std::is_same_v<Tag, typename S::U>) return u;
    else if constexpr (std::is_same_v<Tag, typename S::V>) return v;
    else if constexpr (std::is_same_v<Tag, typename S::W>) return w;
    else if constexpr (std::is_same_v<Tag, typename S::Charge>) return q;
    else if constexpr (std::is_same_v<Tag, typename S::Cell>) return cell;
    else return id;
  }
};

// A node-field component: node (i, j, k), i = -1 .. n+1, of a field stored
// with a one-node halo, (i+1) + NX((j+1) + NY(k+1)).
template <class T> struct NodeComponent {
  using location_type = lpfx::Node;
  using value_type = T;
  T* origin;  // node (0, 0, 0)
  int sy, sz;
  __host__ __device__ T& operator()(int i, int j, int k) const { return origin[i + sy * j + sz * k]; }
};

template <class T, class X, class Y, class Z> struct NodeField {
  T* base;            // component 0, halo included
  long long stride;   // elements per component
  int nx, ny;         // cells
  template <std::size_t Axis> __host__ __device__ NodeComponent<T> component() const {
    const int sy = nx + 3, sz = (nx + 3) * (ny + 3);
    return {base + Axis * stride + 1 + sy + sz, sy, sz};
  }
  template <class Tag> __host__ __device__ NodeComponent<T> get() const {
    static_assert(std::is_same_v<Tag, X> || std::is_same_v<Tag, Y> || std::is_same_v<Tag, Z>);
    return component<std::is_same_v<Tag, X> ? 0 : std::is_same_v<Tag, Y> ? 1 : 2>();
  }
};

}  // namespace

extern "C" {

typedef struct {
  int nx, ny, nz;
  double dx, dy, dz;
} refgpu_grid;

typedef struct {
  void *rx, *ry, *rz, *u, *v, *w;
  double* q;
  std::int32_t* cell;
  std::uint64_t* id;
  unsigned count;
} refgpu_records;

}  // extern "C"

namespace {

tpic::data::ParticleCellMap cell_map(const refgpu_grid& g) {
  return tpic::data::ParticleCellMap{g.nx, g.ny, g.nz, g.nx + 4, g.ny + 4, (g.nx + 4) * (g.ny + 4) * (g.nz + 4)};
}

tpic::data::MassMatrixLayout mass_layout(const refgpu_grid& g) {
  const int ex = g.nx + 3, ey = g.ny + 3, ez = g.nz + 3;
  return tpic::data::MassMatrixLayout{g.nx + 1, g.ny + 1, g.nz + 1, ex, ey, ez, ex, ex * ey,
                                      (g.nx + 1) * (g.ny + 1) * (g.nz + 1), ex * ey * ez};
}

template <class Precision> Records<Precision> records(const refgpu_records& r) {
  using R = Records<Precision>;
  return R{(typename R::Pos*)r.rx, (typename R::Pos*)r.ry, (typename R::Pos*)r.rz, (typename R::Vel*)r.u,
           (typename R::Vel*)r.v,  (typename R::Vel*)r.w,  r.q, r.cell, r.id};
}

template <class Precision>
int deposit(int kind, const refgpu_grid& g, const refgpu_records& r, const unsigned* counts, const unsigned* offsets,
            const void* b_node, void* out, double qom, double dt, double c, unsigned* failure, unsigned* invalid,
            cudaStream_t s) {
  using F = tpic::data::FieldSchema<Precision>;
  using BT = typename Precision::Storage::Magnetic;
  using JT = typename Precision::Storage::Current;
  using MT = typename Precision::Storage::Mass;
  using B = NodeField<const BT, typename F::Bnx, typename F::Bny, typename F::Bnz>;
  using J = NodeField<JT, typename F::Jx, typename F::Jy, typename F::Jz>;
  using P = Records<Precision>;
  const auto cells = cell_map(g);
  const long long nodes = (long long)(g.nx + 3) * (g.ny + 3) * (g.nz + 3);
  const B magnetic{(const BT*)b_node, nodes, g.nx, g.ny};
  const tpic::ecsim::ParticleBins bins{{counts, offsets, unsigned(cells.count)}, failure, r.count};
  const unsigned grid = blocks_for(unsigned(cells.count));
  const double beta_over_c = (qom * dt / 2) / c;
  const double volume = (g.dx * g.dy) * g.dz;
  if (kind == 0) {
    using C = typename Precision::Compute::Current;
    tpic::ecsim::kernels::sorted_current_kernel<Precision, P, B, J><<<grid, kThreads, 0, s>>>(
        records<Precision>(r), magnetic, J{(JT*)out, nodes, g.nx, g.ny}, cells, cfg::convert<C>(1.0 / volume),
        cfg::convert<C>(beta_over_c), bins, invalid);
  } else {
    using C = typename Precision::Compute::Mass;
    if (kind == 1) {
      tpic::ecsim::kernels::sorted_mass_matrix_scalar_kernel<Precision, P, B><<<grid, kThreads, 0, s>>>(
          records<Precision>(r), magnetic, (MT*)out, mass_layout(g), cells, cfg::convert<C>(beta_over_c), bins,
          invalid);
    } else if constexpr (std::is_same_v<C, double>) {
      tpic::ecsim::kernels::sorted_mass_matrix_mma_kernel<Precision, P, B><<<grid, kThreads, 0, s>>>(
          records<Precision>(r), magnetic, (MT*)out, mass_layout(g), cells, cfg::convert<C>(beta_over_c), bins,
          invalid);
    } else {
      return 1;
    }
  }
  return cudaGetLastError() == cudaSuccess ? 0 : 4;
}

template <class Precision>
int move(const refgpu_grid& g, const refgpu_records& r, const unsigned* counts, const unsigned* offsets,
         const void* b_node, const void* e_theta, double qom, double dt, double c, unsigned* failure,
         unsigned* invalid, cudaStream_t s) {
  using F = tpic::data::FieldSchema<Precision>;
  using BT = typename Precision::Storage::Magnetic;
  using ET = typename Precision::Storage::Electric;
  using B = NodeField<const BT, typename F::Bnx, typename F::Bny, typename F::Bnz>;
  using E = NodeField<const ET, typename F::Ex, typename F::Ey, typename F::Ez>;
  using P = Records<Precision>;
  using Sink = tpic::communication::LocalParticleDestinationSink;
  const auto cells = cell_map(g);
  const long long nodes = (long long)(g.nx + 3) * (g.ny + 3) * (g.nz + 3);
  tpic::communication::ParticleMigrationGeometry geometry{};
  geometry.cells = cells;
  const int extents[3] = {g.nx, g.ny, g.nz};
  for (int a = 0; a < 3; ++a) {
    geometry.global_cells[a] = extents[a];
    geometry.partition_base[a] = extents[a];
    geometry.periodic[a] = true;
  }
  // prepare_particle_mover_parameters (ecsim/particles/particle_mover_parameters.hpp:23-45).
  using VC = typename Precision::Compute::Velocity;
  using PC = typename Precision::Compute::Position;
  const double beta = qom * dt / 2;
  tpic::ecsim::ParticleMoverParameters<Precision> parameters{
      cfg::convert<VC>(beta), cfg::convert<VC>(beta / c), cfg::convert<PC>(dt),
      {cfg::convert<PC>(1.0 / g.dx), cfg::convert<PC>(1.0 / g.dy), cfg::convert<PC>(1.0 / g.dz)}};
  const tpic::ecsim::ParticleBins bins{{counts, offsets, unsigned(cells.count)}, failure, r.count};
  const unsigned grid = blocks_for((unsigned long long)g.nx * g.ny * g.nz);
  tpic::ecsim::kernels::sorted_particle_mover_kernel<Precision, P, B, E, Sink><<<grid, kThreads, 0, s>>>(
      B{(const BT*)b_node, nodes, g.nx, g.ny}, E{(const ET*)e_theta, nodes, g.nx, g.ny}, records<Precision>(r),
      Sink{invalid, r.count}, geometry, parameters, bins, invalid);
  return cudaGetLastError() == cudaSuccess ? 0 : 4;
}

}  // namespace

extern "C" {

// kind: 0 current (J node field), 1 scalar mass, 2 matrix-core mass (records
// layout, 126 scalars per node-field vertex). Adds into `out`. failure: one
// zero device word (the producer's failure flag of the bins).
int refgpu_deposit(int level, int kind, const refgpu_grid* g, const refgpu_records* r, const unsigned* counts,
                   const unsigned* offsets, const void* b_node, void* out, double qom, double dt, double c,
                   unsigned* failure, unsigned* invalid, cudaStream_t s) {
  if (!g || !r || kind < 0 || kind > 2) return 1;
  switch (level) {
    case 0: return deposit<Level0>(kind, *g, *r, counts, offsets, b_node, out, qom, dt, c, failure, invalid, s);
    case 1: return deposit<Level1>(kind, *g, *r, counts, offsets, b_node, out, qom, dt, c, failure, invalid, s);
    case 2: return deposit<Level2>(kind, *g, *r, counts, offsets, b_node, out, qom, dt, c, failure, invalid, s);
    default: return 1;
  }
}

// The sorted mover of one species in place (periodic, one rank).
int refgpu_move(int level, const refgpu_grid* g, const refgpu_records* r, const unsigned* counts,
                const unsigned* offsets, const void* b_node, const void* e_theta, double qom, double dt, double c,
                unsigned* failure, unsigned* invalid, cudaStream_t s) {
  if (!g || !r) return 1;
  switch (level) {
    case 0: return move<Level0>(*g, *r, counts, offsets, b_node, e_theta, qom, dt, c, failure, invalid, s);
    case 1: return move<Level1>(*g, *r, counts, offsets, b_node, e_theta, qom, dt, c, failure, invalid, s);
    default: return 1;
  }
}

}  // extern "C"
