// The C ABI (include/tpicb200.h): context, argument checks, stage entry
// points and the cycle driver. Every entry point validates its arguments,
// enqueues on the caller's stream and maps CUDA failures to status codes.
#include "kernels.cuh"

#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <atomic>
#include <utility>

using namespace tpicb200;

struct tpicb200_context {
  int device = 0;
  Geom g{};
  tpicb200_grid grid{};
  tpicb200_options opt{};
  SolverWorkspace* solver = nullptr;
  uint32_t* cursor = nullptr;
  uint32_t* perm = nullptr;
  uint32_t* perm2 = nullptr;     // ranks of the second species of a pair (the cycle)
  uint32_t* scan = nullptr;
  uint32_t* binned = nullptr;    // binned-sort state, old bins and transfer counts
  uint16_t* codes = nullptr;     // binned-sort run code per record
  uint32_t* invalid = nullptr;   // context's own invalid counter
  double* partials = nullptr;    // energy reduction partials
  double* mover_partials = nullptr;  // species scalars of the cycle's movers (5 rows per species)
  int mover_written[TPICB200_MAX_SPECIES]{};
  double* reduced = nullptr;     // energy reduction results
  double* center = nullptr;      // velocity-centring partials (4 rows of energy_blocks) and 4 sums
  double* particle_theta = nullptr;  // S^n(E_theta), the movers' field when smoothing is on
  double* pinned = nullptr;      // host mirror of `reduced` + invalid
  int energy_blocks = 0;
  cudaEvent_t events[6 + 3 * TPICB200_MAX_SPECIES]{};
  void* moments = nullptr;       // per-cell moments of the moment forms (float: tensor core; double: FP64)
  bool moments_pending = false;  // moments hold deposits not yet assembled
  // J and mass buffers zeroed by the last tpicb200_clear_moments that nothing
  // else has deposited into since: the assembly may store instead of add.
  const void* cleared_j = nullptr;
  const void* cleared_mass = nullptr;
  uint32_t wait_polls = 0;  // device wait bound of the stream kernel and the TMA apply (0: the default)
  int stall_site = TPICB200_STALL_NONE;  // tpicb200_inject_stall
  uint32_t stall_index = 0;
};

namespace {

thread_local std::string last_error;

int fail(int status, const std::string& message) {
  last_error = message;
  return status;
}

int cuda_status(cudaError_t e, const char* what) {
  if (e == cudaSuccess) return TPICB200_SUCCESS;
  return fail(TPICB200_BACKEND_FAILURE, std::string(what) + ": " + cudaGetErrorString(e));
}

int check_ctx(const tpicb200_context* ctx) {
  if (!ctx) return fail(TPICB200_INVALID_ARGUMENT, "null context");
  return TPICB200_SUCCESS;
}

int check_particles(const tpicb200_context* ctx, const tpicb200_particles* p) {
  if (!p) return fail(TPICB200_INVALID_ARGUMENT, "null particle set");
  if (p->count > ctx->opt.max_particles)
    return fail(TPICB200_CAPACITY_EXCEEDED, "particle count above the context capacity");
  if (p->count && (!p->rx || !p->ry || !p->rz || !p->u || !p->v || !p->w || !p->q || !p->cell))
    return fail(TPICB200_INVALID_ARGUMENT, "null particle attribute");
  return TPICB200_SUCCESS;
}

uint32_t* invalid_or_own(tpicb200_context* ctx, uint32_t* invalid) {
  return invalid ? invalid : ctx->invalid;
}

// Forms that deposit per-cell moments, assembled into J and the mass records
// by the fold: the tensor-core forms (mixed precision) and the FP64 moments.
bool moment_form(int kind) {
  return kind == TPICB200_MASS_TF32 || kind == TPICB200_MASS_BF16X3 || kind == TPICB200_MASS_MOMENTS_F64;
}

// The mass form is admitted by the precision mode.
int check_mass_kind(const tpicb200_context* ctx, int kind) {
  if (kind < TPICB200_MASS_SCALAR || kind > TPICB200_MASS_MOMENTS_F64)
    return fail(TPICB200_INVALID_ARGUMENT, "unknown mass kind");
  const bool dbl = ctx->opt.precision == TPICB200_PRECISION_DOUBLE;
  if (dbl && (kind == TPICB200_MASS_TF32 || kind == TPICB200_MASS_BF16X3))
    return fail(TPICB200_INVALID_ARGUMENT, "tensor-core mass forms need the mixed precision mode");
  if (!dbl && kind == TPICB200_MASS_MOMENTS_F64)
    return fail(TPICB200_INVALID_ARGUMENT, "the FP64 moment form needs the double precision mode");
  return TPICB200_SUCCESS;
}

cudaError_t launch_moments(tpicb200_context* ctx, int kind, int ns, const double* qom,
                           const tpicb200_particles* const* parts, const uint32_t* const* counts,
                           const uint32_t* const* offsets, const void* b_node, int accumulate, uint32_t* invalid,
                           const SortedCopy* const* copies, cudaStream_t s) {
  if (kind == TPICB200_MASS_MOMENTS_F64)
    return launch_deposit_moments_f64(ctx->g, ns, qom, ctx->opt.dt, ctx->opt.c, parts, counts, offsets, b_node,
                                      (double*)ctx->moments, accumulate, invalid, copies, s);
  return launch_deposit_tc(kind, ctx->g, ns, qom, ctx->opt.dt, ctx->opt.c, parts, counts, offsets, b_node,
                           (float*)ctx->moments, accumulate, invalid, copies, s, ctx->wait_polls,
                           ctx->stall_site == TPICB200_STALL_DEPOSIT ? ctx->stall_index : 0u);
}

}  // namespace

namespace tpicb200 {
static std::atomic<unsigned long long> g_launches{0};
void count_launches(unsigned n) { g_launches.fetch_add(n, std::memory_order_relaxed); }
unsigned long long launches_so_far() { return g_launches.load(std::memory_order_relaxed); }
void uncount_launches(unsigned long long n) { g_launches.fetch_sub(n, std::memory_order_relaxed); }
int report_error(int status, const std::string& message) { return fail(status, message); }

Geom make_geom(const tpicb200_grid& grid) {
  Geom g{};
  g.nx = grid.nx; g.ny = grid.ny; g.nz = grid.nz;
  g.NX = grid.nx + 3; g.NY = grid.ny + 3; g.NZ = grid.nz + 3;
  g.CX = grid.nx + 2; g.CY = grid.ny + 2; g.CZ = grid.nz + 2;
  g.ex = grid.nx + 4; g.ey = grid.ny + 4; g.ez = grid.nz + 4;
  g.nodes = (long long)g.NX * g.NY * g.NZ;
  g.cells = (long long)g.CX * g.CY * g.CZ;
  g.bins = (long long)g.ex * g.ey * g.ez;
  g.inx = grid.nx + 1; g.iny = grid.ny + 1; g.inz = grid.nz + 1;
  g.interior = (long long)g.inx * g.iny * g.inz;
  g.dx = grid.lx / grid.nx; g.dy = grid.ly / grid.ny; g.dz = grid.lz / grid.nz;
  g.inv[0] = 1.0 / g.dx; g.inv[1] = 1.0 / g.dy; g.inv[2] = 1.0 / g.dz;
  g.volume = (g.dx * g.dy) * g.dz;
  g.inv_volume = 1.0 / g.volume;
  g.mvs = 126;
  g.mes = 1;
  g.MX = g.NX;
  g.mnodes = g.nodes;
  g.run_len = kRunCells;
  while (g.run_len > 1 && (long long)((g.nx + g.run_len - 1) / g.run_len) * g.ny * g.nz < kRunTarget) g.run_len >>= 1;
  return g;
}
}  // namespace tpicb200

extern "C" {

const char* tpicb200_version(void) { return "tpicb200 0.1 (sm_100a)"; }
const char* tpicb200_last_error(void) { return last_error.c_str(); }
unsigned long long tpicb200_launch_count(void) { return tpicb200::g_launches.load(); }

int tpicb200_create(const tpicb200_grid* grid, const tpicb200_options* options, tpicb200_context** out) {
  if (!grid || !options || !out) return fail(TPICB200_INVALID_ARGUMENT, "null create argument");
  *out = nullptr;
  if (grid->nx <= 0 || grid->ny <= 0 || grid->nz <= 0 || !(grid->lx > 0) || !(grid->ly > 0) ||
      !(grid->lz > 0) || !std::isfinite(grid->lx) || !std::isfinite(grid->ly) || !std::isfinite(grid->lz))
    return fail(TPICB200_INVALID_ARGUMENT, "grid extents must be positive and finite");
  const long long bins = (grid->nx + 4LL) * (grid->ny + 4LL) * (grid->nz + 4LL);
  const long long nodes = (grid->nx + 3LL) * (grid->ny + 3LL) * (grid->nz + 3LL);
  if (bins > 0x7fffffffLL || nodes * 126 > (1LL << 40))
    return fail(TPICB200_OVERFLOW, "grid too large for int32 cell keys");
  if (!(options->dt > 0) || !std::isfinite(options->dt) || !(options->theta > 0) || options->theta > 1 ||
      !(options->c > 0) || !std::isfinite(options->c) || !(options->gmres_tol >= 0) ||
      options->gmres_restart <= 0 || options->gmres_restart > 1024 || options->gmres_max_iterations <= 0)
    return fail(TPICB200_INVALID_ARGUMENT, "invalid time step, theta, c or GMRES parameters");
  if (options->precision != TPICB200_PRECISION_DOUBLE && options->precision != TPICB200_PRECISION_MIXED)
    return fail(TPICB200_INVALID_ARGUMENT, "unknown precision mode");
  if (options->mass_layout != TPICB200_MASS_LAYOUT_RECORDS &&
      options->mass_layout != TPICB200_MASS_LAYOUT_STENCIL_MAJOR &&
      options->mass_layout != TPICB200_MASS_LAYOUT_TILED)
    return fail(TPICB200_INVALID_ARGUMENT, "unknown mass layout");
  // config/physics.cpp:65-70: 0 <= Smooth <= 1, SmoothNiter >= 0.
  if (options->smooth_iterations < 0 || !std::isfinite(options->smooth_alpha) ||
      (options->smooth_iterations > 0 && (options->smooth_alpha < 0 || options->smooth_alpha > 1)) ||
      (options->smooth_operator != TPICB200_SMOOTH_FACE7 && options->smooth_operator != TPICB200_SMOOTH_BINOMIAL27))
    return fail(TPICB200_INVALID_ARGUMENT,
                "energy-conserving smoothing requires SmoothNiter >= 0, 0 <= Smooth <= 1 and a known operator");
  int device = 0, count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0)
    return fail(TPICB200_BACKEND_FAILURE, "no CUDA device: the ECSIM cycle has no CPU fallback");
  cudaGetDevice(&device);
  int major = 0;
  cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, device);
  if (major != 10) return fail(TPICB200_BACKEND_FAILURE, "this build targets sm_100a (B200) only");
  auto* ctx = new tpicb200_context();
  ctx->device = device;
  ctx->g = make_geom(*grid);
  ctx->grid = *grid;
  if (options->mass_layout == TPICB200_MASS_LAYOUT_STENCIL_MAJOR) {
    ctx->g.mvs = 1;
    ctx->g.mes = ctx->g.nodes;
  } else if (options->mass_layout == TPICB200_MASS_LAYOUT_TILED) {
    ctx->g.MX = (ctx->g.NX + 3) & ~3;
    ctx->g.mnodes = (long long)ctx->g.MX * ctx->g.NY * ctx->g.NZ;
    ctx->g.mvs = 1;
    ctx->g.mes = ctx->g.mnodes;
  }
  ctx->opt = *options;
  cudaError_t e = cudaSuccess;
  SmoothingPlan smoothing;
  if (options->smooth_iterations > 0 && options->smooth_alpha < 1)
    smoothing = SmoothingPlan{options->smooth_iterations, options->smooth_alpha, options->smooth_operator};
  ctx->solver = solver_create(options->precision, ctx->g, options->gmres_restart, options->dt,
                              options->theta, options->c, smoothing, &e);
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  ctx->energy_blocks = 4 * sms;
  auto alloc = [&](void** p, size_t bytes) {
    if (e == cudaSuccess) e = cudaMalloc(p, bytes ? bytes : 4);
  };
  alloc((void**)&ctx->cursor, size_t(ctx->g.bins) * 4);
  alloc((void**)&ctx->perm, size_t(options->max_particles) * 4);
  alloc((void**)&ctx->perm2, size_t(options->max_particles) * 4);
  alloc((void**)&ctx->scan, sort_scan_words(ctx->g.bins) * 4);
  alloc((void**)&ctx->binned, binned_scratch_words(ctx->g) * 4);
  alloc((void**)&ctx->codes, size_t(options->max_particles) * 2);
  alloc((void**)&ctx->invalid, 4);
  alloc((void**)&ctx->partials, size_t(ctx->energy_blocks) * (2 + 5 * TPICB200_MAX_SPECIES) * 8);
  alloc((void**)&ctx->mover_partials, size_t(kMoverPartials) * 5 * TPICB200_MAX_SPECIES * 8);
  alloc((void**)&ctx->reduced, (2 + 5 * TPICB200_MAX_SPECIES + 2) * 8);
  alloc((void**)&ctx->center, (size_t(4) * ctx->energy_blocks + 4) * 8);
  if (smoothing.iterations > 0) alloc((void**)&ctx->particle_theta, size_t(3) * ctx->g.nodes * 8);
  alloc((void**)&ctx->moments, moment_floats(ctx->g) * (options->precision == TPICB200_PRECISION_MIXED ? 4 : 8));
  if (e == cudaSuccess) e = cudaMallocHost((void**)&ctx->pinned, (2 + 5 * TPICB200_MAX_SPECIES + 2) * 8);
  if (e == cudaSuccess) e = cudaMemset(ctx->invalid, 0, 4);
  if (e == cudaSuccess && ctx->solver) solver_set_invalid(ctx->solver, ctx->invalid);
  for (auto& ev : ctx->events)
    if (e == cudaSuccess) e = cudaEventCreate(&ev);
  if (e != cudaSuccess) {
    tpicb200_destroy(ctx);
    return cuda_status(e, "context allocation failed");
  }
  *out = ctx;
  return TPICB200_SUCCESS;
}

int tpicb200_destroy(tpicb200_context* ctx) {
  if (!ctx) return TPICB200_SUCCESS;
  cudaDeviceSynchronize();
  solver_destroy(ctx->solver);
  cudaFree(ctx->cursor); cudaFree(ctx->perm); cudaFree(ctx->perm2); cudaFree(ctx->scan); cudaFree(ctx->binned); cudaFree(ctx->codes);
  cudaFree(ctx->invalid);
  cudaFree(ctx->partials); cudaFree(ctx->mover_partials); cudaFree(ctx->reduced); cudaFree(ctx->moments);
  cudaFree(ctx->center);
  cudaFree(ctx->particle_theta);
  if (ctx->pinned) cudaFreeHost(ctx->pinned);
  for (auto& ev : ctx->events)
    if (ev) cudaEventDestroy(ev);
  delete ctx;
  return TPICB200_SUCCESS;
}

int tpicb200_get_layout(const tpicb200_context* ctx, tpicb200_layout* out) {
  if (check_ctx(ctx) || !out) return fail(TPICB200_INVALID_ARGUMENT, "null layout argument");
  out->node_count = ctx->g.nodes;
  out->cell_count = ctx->g.cells;
  out->bin_count = ctx->g.bins;
  out->interior_nodes = ctx->g.interior;
  const bool dbl = ctx->opt.precision == TPICB200_PRECISION_DOUBLE;
  out->field_scalar_bytes = dbl ? 8 : 4;
  out->mass_scalar_bytes = dbl ? 8 : 4;
  out->velocity_scalar_bytes = dbl ? 8 : 4;
  out->mass_count = 126 * ctx->g.mnodes;
  return TPICB200_SUCCESS;
}

int tpicb200_mover(tpicb200_context* ctx, double qom, tpicb200_particles* p, const double* e_theta,
                   const void* b_node, uint32_t* invalid, tpicb200_stream stream) {
  if (int s = check_ctx(ctx)) return s;
  if (int s = check_particles(ctx, p)) return s;
  if (!e_theta || !b_node || !std::isfinite(qom))
    return fail(TPICB200_INVALID_ARGUMENT, "mover needs E_theta, B nodes and a finite q/m");
  const double beta = qom * ctx->opt.dt / 2;
  if (!std::isfinite(beta)) return fail(TPICB200_OVERFLOW, "q/m*dt/2 is not finite");
  return cuda_status(launch_mover(ctx->opt.precision, ctx->g, qom, ctx->opt.dt, ctx->opt.c, p, nullptr, nullptr,
                                  e_theta, b_node, invalid_or_own(ctx, invalid), nullptr, nullptr,
                                  (cudaStream_t)stream),
                     "mover launch failed");
}

int tpicb200_sort(tpicb200_context* ctx, const tpicb200_particles* in, tpicb200_particles* out,
                  uint32_t* counts, uint32_t* offsets, uint32_t* invalid, tpicb200_stream stream) {
  if (int s = check_ctx(ctx)) return s;
  if (int s = check_particles(ctx, in)) return s;
  if (!out || !counts || !offsets) return fail(TPICB200_INVALID_ARGUMENT, "sort needs output records and bins");
  if (in->count && (!out->rx || !out->ry || !out->rz || !out->u || !out->v || !out->w || !out->q ||
                    !out->cell || (in->id && !out->id)))
    return fail(TPICB200_INVALID_ARGUMENT, "null output attribute");
  if (in->count && (in->rx == out->rx || in->cell == out->cell))
    return fail(TPICB200_INVALID_ARGUMENT, "sort input and output alias");
  return cuda_status(launch_sort(ctx->opt.precision, ctx->g, in, out, counts, offsets, ctx->cursor, ctx->perm,
                                 ctx->scan, invalid_or_own(ctx, invalid), (cudaStream_t)stream),
                     "sort launch failed");
}

int tpicb200_sort_binned(tpicb200_context* ctx, const tpicb200_particles* in, const uint32_t* in_counts,
                         const uint32_t* in_offsets, tpicb200_particles* out, uint32_t* counts,
                         uint32_t* offsets, uint32_t* invalid, tpicb200_stream stream) {
  if (int s = check_ctx(ctx)) return s;
  if (!in_counts || !in_offsets) return fail(TPICB200_INVALID_ARGUMENT, "binned sort needs the input's bins");
  if (!binned_sort_applies(ctx->g))
    return tpicb200_sort(ctx, in, out, counts, offsets, invalid, stream);
  if (int s = check_particles(ctx, in)) return s;
  if (!out || !counts || !offsets) return fail(TPICB200_INVALID_ARGUMENT, "sort needs output records and bins");
  if (in->count && (!out->rx || !out->ry || !out->rz || !out->u || !out->v || !out->w || !out->q ||
                    !out->cell || (in->id && !out->id)))
    return fail(TPICB200_INVALID_ARGUMENT, "null output attribute");
  if (in->count && (in->rx == out->rx || in->cell == out->cell))
    return fail(TPICB200_INVALID_ARGUMENT, "sort input and output alias");
  return cuda_status(launch_sort_binned(ctx->opt.precision, ctx->g, in, in_counts, in_offsets, out, counts, offsets,
                                        ctx->cursor, ctx->perm, ctx->scan, ctx->binned, ctx->codes,
                                        invalid_or_own(ctx, invalid),
                                        (cudaStream_t)stream),
                     "binned sort launch failed");
}

int tpicb200_sort_static(const tpicb200_grid* grid, int precision, const tpicb200_particles* in,
                         tpicb200_particles* out, uint32_t* counts, uint32_t* offsets, uint32_t* invalid,
                         tpicb200_stream stream) {
  if (!grid || !in || !out || !counts || !offsets)
    return fail(TPICB200_INVALID_ARGUMENT, "static sort needs a grid, records and bins");
  if (grid->nx < 1 || grid->ny < 1 || grid->nz < 1 || !(grid->lx > 0) || !(grid->ly > 0) || !(grid->lz > 0))
    return fail(TPICB200_INVALID_ARGUMENT, "invalid grid");
  if (precision != TPICB200_PRECISION_DOUBLE && precision != TPICB200_PRECISION_MIXED)
    return fail(TPICB200_INVALID_ARGUMENT, "unknown precision");
  const Geom g = make_geom(*grid);
  if (in->count > TPICB200_SORT_STATIC_MAX_RECORDS)
    return fail(TPICB200_CAPACITY_EXCEEDED, "static sort: more than TPICB200_SORT_STATIC_MAX_RECORDS (1048576) records");
  if (g.bins > TPICB200_SORT_STATIC_MAX_BINS)
    return fail(TPICB200_CAPACITY_EXCEEDED, "static sort: grid has more than TPICB200_SORT_STATIC_MAX_BINS (1048576) bins");
  if (in->count && (!in->rx || !in->ry || !in->rz || !in->u || !in->v || !in->w || !in->q || !in->cell))
    return fail(TPICB200_INVALID_ARGUMENT, "null particle attribute");
  if (in->count && (!out->rx || !out->ry || !out->rz || !out->u || !out->v || !out->w || !out->q ||
                    !out->cell || (in->id && !out->id)))
    return fail(TPICB200_INVALID_ARGUMENT, "null output attribute");
  if (in->count && (in->rx == out->rx || in->cell == out->cell))
    return fail(TPICB200_INVALID_ARGUMENT, "sort input and output alias");
  uint32_t* scratch = nullptr;
  if (int r = cuda_status(sort_static_setup(&scratch), "static sort set-up (device symbol address) failed")) return r;
  return cuda_status(launch_sort_static(precision, g, in, out, counts, offsets, invalid, scratch, (cudaStream_t)stream),
                     "static sort launch failed");
}

int tpicb200_clear_moments(tpicb200_context* ctx, void* j, void* mass, tpicb200_stream stream) {
  if (int s = check_ctx(ctx)) return s;
  const size_t fb = ctx->opt.precision == TPICB200_PRECISION_DOUBLE ? 8 : 4;
  cudaError_t e = cudaSuccess;
  ctx->moments_pending = false;
  ctx->cleared_j = j && mass ? j : nullptr;
  ctx->cleared_mass = j && mass ? mass : nullptr;
  if (j) e = cudaMemsetAsync(j, 0, 3 * size_t(ctx->g.nodes) * fb, (cudaStream_t)stream);
  if (mass && e == cudaSuccess) e = cudaMemsetAsync(mass, 0, 126 * size_t(ctx->g.mnodes) * fb, (cudaStream_t)stream);
  return cuda_status(e, "moment clear failed");
}

int tpicb200_deposit(tpicb200_context* ctx, double qom, const tpicb200_particles* p, const uint32_t* counts,
                     const uint32_t* offsets, const void* b_node, void* j, void* mass, int mass_kind,
                     uint32_t* invalid, tpicb200_stream stream) {
  if (int s = check_ctx(ctx)) return s;
  if (int s = check_particles(ctx, p)) return s;
  if (!b_node || !std::isfinite(qom)) return fail(TPICB200_INVALID_ARGUMENT, "deposit needs B nodes and finite q/m");
  if ((counts == nullptr) != (offsets == nullptr))
    return fail(TPICB200_INVALID_ARGUMENT, "counts and offsets go together");
  if (int r = check_mass_kind(ctx, mass_kind)) return r;
  const double boc = qom * ctx->opt.dt / 2 / ctx->opt.c;
  if (!std::isfinite(boc)) return fail(TPICB200_OVERFLOW, "beta/c is not finite");
  uint32_t* inv = invalid_or_own(ctx, invalid);
  cudaStream_t s = (cudaStream_t)stream;
  if (moment_form(mass_kind)) {
    if (!counts) return fail(TPICB200_INVALID_ARGUMENT, "moment mass forms need sorted bins");
    if (!j || !mass) return fail(TPICB200_INVALID_ARGUMENT, "moment mass forms deposit J-hat and mass together");
    const int accumulate = ctx->moments_pending ? 1 : 0;
    const int r = cuda_status(launch_moments(ctx, mass_kind, 1, &qom, &p, &counts, &offsets, b_node, accumulate, inv,
                                             nullptr, s),
                              "moment deposition launch failed");
    if (r == TPICB200_SUCCESS) ctx->moments_pending = true;
    return r;
  }
  ctx->cleared_j = ctx->cleared_mass = nullptr;
  return cuda_status(launch_deposit(ctx->opt.precision, mass_kind, ctx->g, qom, ctx->opt.dt, ctx->opt.c, p,
                                    counts, offsets, b_node, j, mass, inv, nullptr, s),
                     "deposition launch failed");
}

int tpicb200_fold_periodic(tpicb200_context* ctx, void* j, void* mass, tpicb200_stream stream) {
  if (int s = check_ctx(ctx)) return s;
  if (ctx->moments_pending) {
    // Cell moments of the moment forms are added into the unique nodes first.
    if (!j || !mass) return fail(TPICB200_INVALID_ARGUMENT, "pending cell moments need J-hat and mass");
    const int overwrite = j == ctx->cleared_j && mass == ctx->cleared_mass ? 1 : 0;
    if (int r = cuda_status(launch_assemble_moments(ctx->opt.precision, ctx->g, ctx->moments, j, mass, overwrite,
                                                    (cudaStream_t)stream),
                            "moment assembly failed"))
      return r;
    ctx->moments_pending = false;
    ctx->cleared_j = ctx->cleared_mass = nullptr;
  }
  return cuda_status(launch_fold(ctx->opt.precision, ctx->g, j, mass, (cudaStream_t)stream), "fold launch failed");
}

int tpicb200_smooth(tpicb200_context* ctx, const double* in, double* out, tpicb200_stream stream) {
  if (int s = check_ctx(ctx)) return s;
  if (!in || !out || in == out) return fail(TPICB200_INVALID_ARGUMENT, "smoothing needs distinct in and out fields");
  if (!ctx->particle_theta) return fail(TPICB200_INVALID_STATE, "the context has no energy-conserving smoothing");
  return cuda_status(solver_smooth(ctx->solver, in, out, (cudaStream_t)stream), "smoothing launch failed");
}

int tpicb200_mass_apply(tpicb200_context* ctx, const void* mass, const double* in, double* out,
                        tpicb200_stream stream) {
  if (int s = check_ctx(ctx)) return s;
  if (!mass || !in || !out || in == out) return fail(TPICB200_INVALID_ARGUMENT, "mass apply needs distinct fields");
  return cuda_status(solver_mass_apply(ctx->solver, mass, in, out, (cudaStream_t)stream), "mass apply failed");
}

int tpicb200_field_solve(tpicb200_context* ctx, const void* e, const void* b_cell, const void* j,
                         const void* mass, double* e_theta, tpicb200_gmres_result* result,
                         tpicb200_stream stream) {
  if (int s = check_ctx(ctx)) return s;
  if (!e || !b_cell || !j || !mass || !e_theta) return fail(TPICB200_INVALID_ARGUMENT, "null field-solve argument");
  cudaError_t err = cudaSuccess;
  const int status = solver_solve(ctx->solver, e, b_cell, j, mass, e_theta, result, ctx->opt.gmres_max_iterations,
                                  ctx->opt.gmres_tol, (cudaStream_t)stream, &err);
  if (err != cudaSuccess) return cuda_status(err, "field solve failed");
  if (status == TPICB200_NOT_CONVERGED) return fail(status, "GMRES did not converge");
  if (status != TPICB200_SUCCESS) return fail(status, "field solve failed (non-finite residual)");
  return status;
}

int tpicb200_field_advance(tpicb200_context* ctx, void* e, const void* b_cell, const double* e_theta,
                           void* b_cell_next, void* b_node_next, tpicb200_stream stream) {
  if (int s = check_ctx(ctx)) return s;
  if (!e || !b_cell || !e_theta || !b_cell_next || !b_node_next || b_cell == b_cell_next)
    return fail(TPICB200_INVALID_ARGUMENT, "null or aliased field-advance argument");
  cudaStream_t s = (cudaStream_t)stream;
  const int p = ctx->opt.precision;
  cudaError_t err = launch_field_advance(p, ctx->g, ctx->opt.theta, -ctx->opt.c * ctx->opt.dt, e, b_cell, e_theta,
                                         b_cell_next, ctx->invalid, s);
  if (err == cudaSuccess) err = launch_cell_ghosts(p, ctx->g, b_cell_next, s);
  if (err == cudaSuccess) err = launch_cell_to_node(p, ctx->g, b_cell_next, b_node_next, s);
  return cuda_status(err, "field advance failed");
}

int tpicb200_magnetic_to_nodes(tpicb200_context* ctx, void* b_cell, void* b_node, tpicb200_stream stream) {
  if (int s = check_ctx(ctx)) return s;
  if (!b_cell || !b_node) return fail(TPICB200_INVALID_ARGUMENT, "null magnetic field");
  cudaError_t err = launch_cell_ghosts(ctx->opt.precision, ctx->g, b_cell, (cudaStream_t)stream);
  if (err == cudaSuccess) err = launch_cell_to_node(ctx->opt.precision, ctx->g, b_cell, b_node, (cudaStream_t)stream);
  return cuda_status(err, "cell-to-node failed");
}

namespace {
int check_deck_grid(const tpicb200_context* ctx, const tpicb200_deck* deck, int s) {
  if (!deck || s < 0 || s >= deck->ns || s >= TPICB200_MAX_SPECIES)
    return fail(TPICB200_INVALID_ARGUMENT, "invalid deck or species index");
  const Geom dg = make_geom(deck->grid);
  if (dg.nx != ctx->g.nx || dg.ny != ctx->g.ny || dg.nz != ctx->g.nz || dg.dx != ctx->g.dx || dg.dy != ctx->g.dy ||
      dg.dz != ctx->g.dz)
    return fail(TPICB200_INVALID_ARGUMENT, "the deck's grid is not the context's");
  return TPICB200_SUCCESS;
}
}  // namespace

int tpicb200_load_species(tpicb200_context* ctx, const tpicb200_deck* deck, int s, uint64_t seed, uint64_t first,
                          tpicb200_particles* p, uint32_t* invalid, tpicb200_stream stream) {
  if (int st = check_ctx(ctx)) return st;
  if (int st = check_deck_grid(ctx, deck, s)) return st;
  if (int st = check_particles(ctx, p)) return st;
  const tpicb200_deck_species& sp = deck->species[s];
  if (sp.npcel[0] < 1 || sp.npcel[1] < 1 || sp.npcel[2] < 1)
    return fail(TPICB200_INVALID_ARGUMENT, "npcel must be positive");
  const unsigned long long ppc = (unsigned long long)sp.npcel[0] * sp.npcel[1] * sp.npcel[2];
  const unsigned long long total = ppc * (unsigned long long)ctx->g.nx * ctx->g.ny * ctx->g.nz;
  if (ppc > 0xffffffffULL || first > total || p->count > total - first)
    return fail(TPICB200_INVALID_ARGUMENT, "records beyond the species' cells x particles per cell");
  CaseProfile prof{};
  if (int st = case_profile_of(deck, s, &prof)) return st;
  LoadPlan plan{};
  plan.first = first;
  plan.ppc = uint32_t(ppc);
  for (int a = 0; a < 3; ++a) {
    plan.npc[a] = sp.npcel[a];
    plan.inverse_npc[a] = 1.0 / sp.npcel[a];
    plan.vth[a] = sp.vth[a];
  }
  plan.q_factor = (sp.qom > 0 ? 1.0 : -1.0) * ctx->g.volume / double(ppc);
  plan.key0 = uint32_t(seed);
  plan.key1 = uint32_t(seed >> 32);
  plan.species = uint32_t(s);
  plan.quiet = deck->quiet_start ? 1 : 0;
  return cuda_status(launch_load_species(ctx->opt.precision, ctx->g, plan, prof, p, invalid_or_own(ctx, invalid),
                                         (cudaStream_t)stream),
                     "particle loading launch failed");
}

int tpicb200_center_velocities(tpicb200_context* ctx, const tpicb200_deck* deck, int s, tpicb200_particles* p,
                               uint32_t* invalid, tpicb200_stream stream) {
  if (int st = check_ctx(ctx)) return st;
  if (int st = check_deck_grid(ctx, deck, s)) return st;
  if (int st = check_particles(ctx, p)) return st;
  CaseProfile prof{};
  if (int st = case_profile_of(deck, s, &prof)) return st;
  const int blocks = ctx->energy_blocks;
  return cuda_status(launch_center_velocities(ctx->opt.precision, ctx->g, prof, p, ctx->center, blocks,
                                              ctx->center + 4 * blocks, invalid_or_own(ctx, invalid),
                                              (cudaStream_t)stream),
                     "velocity centring launch failed");
}

int tpicb200_energy(tpicb200_context* ctx, const void* e, const void* b_cell, const tpicb200_particles* species,
                    const double* qom, int ns, double* out, tpicb200_stream stream) {
  if (int s = check_ctx(ctx)) return s;
  if (!e || !b_cell || !out || ns < 0 || ns > TPICB200_MAX_SPECIES || (ns > 0 && (!species || !qom)))
    return fail(TPICB200_INVALID_ARGUMENT, "invalid energy arguments");
  cudaStream_t s = (cudaStream_t)stream;
  const int blocks = ctx->energy_blocks;
  cudaError_t err = launch_field_energy(ctx->opt.precision, ctx->g, e, b_cell, ctx->partials, blocks, s);
  for (int sp = 0; sp < ns && err == cudaSuccess; ++sp)
    err = launch_species_scalars(ctx->opt.precision, &species[sp], qom[sp],
                                 ctx->partials + size_t(blocks) * (2 + 5 * sp), blocks, s);
  const int rows = 2 + 5 * ns;
  if (err == cudaSuccess) err = launch_reduce_rows(ctx->partials, ctx->reduced, rows, blocks, blocks, rows, s);
  if (err == cudaSuccess) err = cudaMemcpyAsync(ctx->pinned, ctx->reduced, rows * 8, cudaMemcpyDeviceToHost, s);
  if (err == cudaSuccess) err = cudaStreamSynchronize(s);
  if (err != cudaSuccess) return cuda_status(err, "energy reduction failed");
  const double norm = ctx->g.volume / (8 * 3.14159265358979323846);
  out[0] = norm * ctx->pinned[0];
  out[1] = norm * ctx->pinned[1];
  for (int r = 2; r < rows; ++r) out[r] = ctx->pinned[r];
  return TPICB200_SUCCESS;
}

int tpicb200_deposit_species(tpicb200_context* ctx, int ns, const double* qom, const tpicb200_particles* species,
                             const uint32_t* const* counts, const uint32_t* const* offsets, const void* b_node,
                             void* j, void* mass, int mass_kind, uint32_t* invalid, tpicb200_stream stream) {
  if (int s = check_ctx(ctx)) return s;
  if (ns < 0 || ns > TPICB200_MAX_SPECIES || (ns > 0 && (!qom || !species || !counts || !offsets)))
    return fail(TPICB200_INVALID_ARGUMENT, "invalid species arrays");
  if (!moment_form(mass_kind)) {
    for (int sp = 0; sp < ns; ++sp)
      if (int r = tpicb200_deposit(ctx, qom[sp], &species[sp], counts[sp], offsets[sp], b_node, j, mass, mass_kind,
                                   invalid, stream))
        return r;
    return TPICB200_SUCCESS;
  }
  // Moment forms: the per-species checks of tpicb200_deposit, then one
  // fused pass per species pair.
  if (int r = check_mass_kind(ctx, mass_kind)) return r;
  if (!b_node) return fail(TPICB200_INVALID_ARGUMENT, "deposit needs B nodes");
  if (!j || !mass) return fail(TPICB200_INVALID_ARGUMENT, "moment mass forms deposit J-hat and mass together");
  if (ns == 0) return TPICB200_SUCCESS;
  const tpicb200_particles* parts[TPICB200_MAX_SPECIES];
  for (int sp = 0; sp < ns; ++sp) {
    parts[sp] = &species[sp];
    if (int r = check_particles(ctx, parts[sp])) return r;
    if (!counts[sp] || !offsets[sp]) return fail(TPICB200_INVALID_ARGUMENT, "moment mass forms need sorted bins");
    if (!std::isfinite(qom[sp])) return fail(TPICB200_INVALID_ARGUMENT, "deposit needs finite q/m");
    if (!std::isfinite(qom[sp] * ctx->opt.dt / 2 / ctx->opt.c)) return fail(TPICB200_OVERFLOW, "beta/c is not finite");
  }
  const int r = cuda_status(launch_moments(ctx, mass_kind, ns, qom, parts, counts, offsets, b_node,
                                           ctx->moments_pending ? 1 : 0, invalid_or_own(ctx, invalid), nullptr,
                                           (cudaStream_t)stream),
                            "moment deposition launch failed");
  if (r == TPICB200_SUCCESS) ctx->moments_pending = true;
  return r;
}

static int deposit_all(tpicb200_context* ctx, tpicb200_state* st, const void* b_node, cudaStream_t s) {
  if (int r = tpicb200_clear_moments(ctx, st->j, st->mass, (tpicb200_stream)s)) return r;
  tpicb200_particles live[TPICB200_MAX_SPECIES];
  const uint32_t* counts[TPICB200_MAX_SPECIES];
  const uint32_t* offsets[TPICB200_MAX_SPECIES];
  for (int sp = 0; sp < st->ns; ++sp) {
    live[sp] = st->slot[sp][st->current[sp]];
    counts[sp] = st->counts[sp];
    offsets[sp] = st->offsets[sp];
  }
  if (int r = tpicb200_deposit_species(ctx, st->ns, st->qom, live, counts, offsets, b_node, st->j, st->mass,
                                       st->mass_kind, nullptr, (tpicb200_stream)s))
    return r;
  return tpicb200_fold_periodic(ctx, st->j, st->mass, (tpicb200_stream)s);
}

// Startup sort of every species' live slot into its idle slot.
static int sort_all(tpicb200_context* ctx, tpicb200_state* st, cudaStream_t s) {
  for (int sp = 0; sp < st->ns; ++sp) {
    const int cur = st->current[sp];
    tpicb200_particles* in = &st->slot[sp][cur];
    tpicb200_particles* out = &st->slot[sp][1 - cur];
    if (int r = tpicb200_sort(ctx, in, out, st->counts[sp], st->offsets[sp], nullptr, (tpicb200_stream)s)) return r;
    st->current[sp] = 1 - cur;
  }
  return TPICB200_SUCCESS;
}

static int check_state(tpicb200_context* ctx, tpicb200_state* st) {
  if (!st || st->ns <= 0 || st->ns > TPICB200_MAX_SPECIES)
    return fail(TPICB200_INVALID_ARGUMENT, "invalid state or species count");
  if (!st->e || !st->b_cell || !st->b_node || !st->b_cell_next || !st->b_node_next || !st->j || !st->mass ||
      !st->e_theta)
    return fail(TPICB200_INVALID_ARGUMENT, "null state field");
  for (int sp = 0; sp < st->ns; ++sp) {
    if (!st->counts[sp] || !st->offsets[sp] || (st->current[sp] != 0 && st->current[sp] != 1))
      return fail(TPICB200_INVALID_ARGUMENT, "invalid species bins or slot");
    if (int r = check_particles(ctx, &st->slot[sp][st->current[sp]])) return r;
    st->slot[sp][1 - st->current[sp]].count = st->slot[sp][st->current[sp]].count;
    if (int r = check_particles(ctx, &st->slot[sp][1 - st->current[sp]])) return r;
  }
  return TPICB200_SUCCESS;
}

// How the deposition reads a species after move_and_sort, and whether the
// live slot flips after it.
// The field the cycle's movers gather: S^n(E_theta) with smoothing, else E_theta.
static const double* particle_field(const tpicb200_context* ctx, const tpicb200_state* st) {
  return ctx->particle_theta ? ctx->particle_theta : st->e_theta;
}

struct DepositPlan {
  const tpicb200_particles* read;  // records the deposition reads
  SortedCopy copy;                 // through which ranks, and where to write them sorted
  bool flip;                       // the idle slot becomes live after the deposition
};

// The mover of species sp, then the sort of the moved records;
// `moved` and `sorted` are recorded after each. On grids whose extents are
// all at least 3 the mover emits direction codes and transfer counts and the
// binned sort ranks the records by them:
//  - a species with a rank buffer (state.ranks) is moved out of place: the
//    mover reads the live records through the previous ranks (when ranked)
//    and writes the moved records in the previous sorted order into the idle
//    slot, which becomes live; the new ranks go to the rank buffer and the
//    species stays ranked (the deposition reads through the ranks);
//  - otherwise the mover moves in place, the ranks go to `perm`, and the
//    deposition reads through them and writes the sorted records into the
//    idle slot.
// On smaller grids the mover moves in place and the general sort writes the
// sorted records.
static int move_and_sort(tpicb200_context* ctx, tpicb200_state* st, int sp, uint32_t* perm, cudaEvent_t moved,
                         cudaEvent_t sorted, DepositPlan* plan, const SpeciesScalars* scalars, cudaStream_t s) {
  const int cur = st->current[sp];
  tpicb200_particles* in = &st->slot[sp][cur];
  tpicb200_particles* out = &st->slot[sp][1 - cur];
  const double qom = st->qom[sp];
  if (int r = check_particles(ctx, in)) return r;
  if (!std::isfinite(qom) || !std::isfinite(qom * ctx->opt.dt / 2)) return fail(TPICB200_OVERFLOW, "q/m*dt/2 is not finite");
  if (in->count && (!out->rx || !out->ry || !out->rz || !out->u || !out->v || !out->w || !out->q || !out->cell ||
                    (in->id && !out->id)))
    return fail(TPICB200_INVALID_ARGUMENT, "null attribute in the idle slot");
  if (in->count && (in->rx == out->rx || in->cell == out->cell))
    return fail(TPICB200_INVALID_ARGUMENT, "live and idle slots alias");
  out->count = in->count;
  const int p = ctx->opt.precision;
  const tpicb200_particles none{};
  if (!binned_sort_applies(ctx->g)) {
    if (st->ranked[sp]) return fail(TPICB200_INVALID_STATE, "ranked species on a grid without the binned sort");
    cudaError_t e = launch_mover(p, ctx->g, qom, ctx->opt.dt, ctx->opt.c, in, nullptr, nullptr, particle_field(ctx, st),
                                 st->b_node, ctx->invalid, nullptr, scalars, s);
    if (e == cudaSuccess) e = cudaEventRecord(moved, s);
    if (e == cudaSuccess)
      e = launch_sort(p, ctx->g, in, out, st->counts[sp], st->offsets[sp], ctx->cursor, perm, ctx->scan,
                      ctx->invalid, s);
    if (e == cudaSuccess) e = cudaEventRecord(sorted, s);
    if (e != cudaSuccess) return cuda_status(e, "mover or sort launch failed");
    *plan = DepositPlan{out, SortedCopy{nullptr, none}, true};
    return TPICB200_SUCCESS;
  }
  const BinnedScratch b = binned_scratch(ctx->g, ctx->binned, ctx->codes);
  cudaError_t e = binned_begin(ctx->g, b, st->counts[sp], st->offsets[sp], true, s);
  if (e == cudaSuccess) e = binned_validate(ctx->g, b, in->count, s);
  const bool ranks = st->ranks[sp] != nullptr;
  if (ranks) {
    // Out of place: the moved records, in the previous sorted order, go live.
    if (e == cudaSuccess)
      e = launch_mover(p, ctx->g, qom, ctx->opt.dt, ctx->opt.c, in, out, st->ranked[sp] ? st->ranks[sp] : nullptr,
                       particle_field(ctx, st), st->b_node, ctx->invalid, &b, scalars, s);
    if (e == cudaSuccess) e = cudaEventRecord(moved, s);
    if (e == cudaSuccess)
      e = binned_finish(p, ctx->g, b, false, false, out, in, st->counts[sp], st->offsets[sp], ctx->cursor,
                        st->ranks[sp], ctx->scan, ctx->invalid, s);
    if (e == cudaSuccess) e = cudaEventRecord(sorted, s);
    if (e != cudaSuccess) return cuda_status(e, "mover or binned sort launch failed");
    st->current[sp] = 1 - cur;
    st->ranked[sp] = 1;
    *plan = DepositPlan{out, SortedCopy{st->ranks[sp], none}, false};
    return TPICB200_SUCCESS;
  }
  if (st->ranked[sp]) return fail(TPICB200_INVALID_STATE, "ranked species without a rank buffer");
  if (e == cudaSuccess)
    e = launch_mover(p, ctx->g, qom, ctx->opt.dt, ctx->opt.c, in, nullptr, nullptr, particle_field(ctx, st), st->b_node,
                     ctx->invalid, &b, scalars, s);
  if (e == cudaSuccess) e = cudaEventRecord(moved, s);
  if (e == cudaSuccess)
    e = binned_finish(p, ctx->g, b, false, false, in, out, st->counts[sp], st->offsets[sp], ctx->cursor, perm,
                      ctx->scan, ctx->invalid, s);
  if (e == cudaSuccess) e = cudaEventRecord(sorted, s);
  if (e != cudaSuccess) return cuda_status(e, "mover or binned sort launch failed");
  *plan = DepositPlan{in, SortedCopy{perm, *out}, true};
  return TPICB200_SUCCESS;
}

// Deposition of species [first, first + count) (at most two) after
// move_and_sort, as their plans say; then the planned slot flips.
static int deposit_pair(tpicb200_context* ctx, tpicb200_state* st, int first, int count, const DepositPlan* plan,
                        bool accumulate, cudaStream_t s) {
  const tpicb200_particles* parts[2];
  const uint32_t* counts[2];
  const uint32_t* offsets[2];
  const SortedCopy* copies[2];
  double qom[2];
  for (int i = 0; i < count; ++i) {
    const int sp = first + i;
    parts[i] = plan[i].read;
    copies[i] = &plan[i].copy;
    counts[i] = st->counts[sp];
    offsets[i] = st->offsets[sp];
    qom[i] = st->qom[sp];
  }
  const int kind = st->mass_kind;
  const int p = ctx->opt.precision;
  cudaError_t e = cudaSuccess;
  if (moment_form(kind)) {
    if (int r = check_mass_kind(ctx, kind)) return r;
    e = launch_moments(ctx, kind, count, qom, parts, counts, offsets, st->b_node_next, accumulate ? 1 : 0,
                       ctx->invalid, copies, s);
    if (e == cudaSuccess) ctx->moments_pending = true;
  } else {
    ctx->cleared_j = ctx->cleared_mass = nullptr;
    for (int i = 0; i < count && e == cudaSuccess; ++i)
      e = launch_deposit(p, kind, ctx->g, qom[i], ctx->opt.dt, ctx->opt.c, parts[i], counts[i], offsets[i],
                         st->b_node_next, st->j, st->mass, ctx->invalid, copies[i], s);
  }
  for (int i = 0; i < count && e == cudaSuccess; ++i) e = launch_copy_ids(parts[i], copies[i], s);
  if (e != cudaSuccess) return cuda_status(e, "deposition launch failed");
  for (int i = 0; i < count; ++i)
    if (plan[i].flip) st->current[first + i] = 1 - st->current[first + i];
  return TPICB200_SUCCESS;
}

}  // extern "C"

namespace tpicb200 {
const Geom& context_geom(const tpicb200_context* ctx) { return ctx->g; }
const tpicb200_options& context_options(const tpicb200_context* ctx) { return ctx->opt; }
const tpicb200_grid& context_grid(const tpicb200_context* ctx) { return ctx->grid; }
uint32_t* context_invalid(tpicb200_context* ctx) { return ctx->invalid; }
int context_check_state(tpicb200_context* ctx, tpicb200_state* st) {
  if (int s = check_ctx(ctx)) return s;
  return check_state(ctx, st);
}
}  // namespace tpicb200

extern "C" {

int tpicb200_materialize(tpicb200_context* ctx, tpicb200_state* st, tpicb200_stream stream) {
  if (int s = check_ctx(ctx)) return s;
  if (int r = check_state(ctx, st)) return r;
  for (int sp = 0; sp < st->ns; ++sp) {
    if (!st->ranked[sp]) continue;
    if (!st->ranks[sp]) return fail(TPICB200_INVALID_STATE, "ranked species without a rank buffer");
    const int cur = st->current[sp];
    tpicb200_particles* in = &st->slot[sp][cur];
    tpicb200_particles* out = &st->slot[sp][1 - cur];
    if (int r = check_particles(ctx, in)) return r;
    if (int r = cuda_status(launch_sorted_gather(ctx->opt.precision, st->ranks[sp], in, out, (cudaStream_t)stream),
                            "materialize gather failed"))
      return r;
    st->current[sp] = 1 - cur;
    st->ranked[sp] = 0;
  }
  return TPICB200_SUCCESS;
}

int tpicb200_prepare(tpicb200_context* ctx, tpicb200_state* st, tpicb200_stream stream) {
  if (int s = check_ctx(ctx)) return s;
  if (int r = check_state(ctx, st)) return r;
  cudaStream_t s = (cudaStream_t)stream;
  if (int r = tpicb200_magnetic_to_nodes(ctx, st->b_cell, st->b_node, stream)) return r;
  if (int r = sort_all(ctx, st, s)) return r;
  for (int sp = 0; sp < st->ns; ++sp) st->ranked[sp] = 0;
  return deposit_all(ctx, st, st->b_node, s);
}

static int read_invalid(tpicb200_context* ctx, cudaStream_t s, uint32_t* value) {
  cudaError_t err = cudaMemcpyAsync(ctx->pinned, ctx->invalid, 4, cudaMemcpyDeviceToHost, s);
  if (err == cudaSuccess) err = cudaStreamSynchronize(s);
  if (err != cudaSuccess) return cuda_status(err, "invalid-flag readback failed");
  std::memcpy(value, ctx->pinned, 4);
  return TPICB200_SUCCESS;
}

int tpicb200_set_wait_limit(tpicb200_context* ctx, uint32_t polls) {
  if (int s = check_ctx(ctx)) return s;
  ctx->wait_polls = polls;
  if (ctx->solver)
    solver_set_waits(ctx->solver, polls, ctx->stall_site == TPICB200_STALL_APPLY ? int(ctx->stall_index) : -1);
  return TPICB200_SUCCESS;
}

int tpicb200_inject_stall(tpicb200_context* ctx, int site, uint32_t index) {
  if (int s = check_ctx(ctx)) return s;
  if (site == TPICB200_STALL_NONE) {
    index = 0;
  } else if (site == TPICB200_STALL_DEPOSIT) {
    if (index < 1) return fail(TPICB200_INVALID_ARGUMENT, "the deposition stall index is a chunk >= 1");
  } else if (site == TPICB200_STALL_APPLY) {
    if (index > 13) return fail(TPICB200_INVALID_ARGUMENT, "the apply stall index is a stencil 0..13");
  } else {
    return fail(TPICB200_INVALID_ARGUMENT, "unknown stall site");
  }
  ctx->stall_site = site;
  ctx->stall_index = index;
  if (ctx->solver) solver_set_waits(ctx->solver, ctx->wait_polls, site == TPICB200_STALL_APPLY ? int(index) : -1);
  return TPICB200_SUCCESS;
}

int tpicb200_read_invalid(tpicb200_context* ctx, uint32_t* count, int clear, tpicb200_stream stream) {
  if (int s = check_ctx(ctx)) return s;
  if (!count) return fail(TPICB200_INVALID_ARGUMENT, "read_invalid needs an output");
  cudaStream_t s = (cudaStream_t)stream;
  if (int r = read_invalid(ctx, s, count)) return r;
  if (clear) return cuda_status(cudaMemsetAsync(ctx->invalid, 0, 4, s), "invalid-counter clear failed");
  return TPICB200_SUCCESS;
}

// The cycle's energy report: the field energies of the committed fields and
// the species scalars the movers accumulated (the values tpicb200_energy
// computes from the live slots, summed in the movers' block order).
static int cycle_energy(tpicb200_context* ctx, const tpicb200_state* st, double* out, cudaStream_t s) {
  const int blocks = ctx->energy_blocks;
  cudaError_t err = launch_field_energy(ctx->opt.precision, ctx->g, st->e, st->b_cell, ctx->partials, blocks, s);
  if (err == cudaSuccess) err = launch_reduce_rows(ctx->partials, ctx->reduced, 2, blocks, blocks, 2, s);
  for (int sp = 0; sp < st->ns && err == cudaSuccess; ++sp)
    err = launch_reduce_rows(ctx->mover_partials + size_t(kMoverPartials) * 5 * sp, ctx->reduced + 2 + 5 * sp, 5,
                             kMoverPartials, ctx->mover_written[sp], ctx->mover_written[sp] > 0 ? 5 : 0, s);
  const int rows = 2 + 5 * st->ns;
  if (err == cudaSuccess) err = cudaMemcpyAsync(ctx->pinned, ctx->reduced, rows * 8, cudaMemcpyDeviceToHost, s);
  if (err == cudaSuccess) err = cudaStreamSynchronize(s);
  if (err != cudaSuccess) return cuda_status(err, "energy reduction failed");
  const double norm = ctx->g.volume / (8 * 3.14159265358979323846);
  out[0] = norm * ctx->pinned[0];
  out[1] = norm * ctx->pinned[1];
  for (int r = 2; r < rows; ++r) out[r] = ctx->pinned[r];
  return TPICB200_SUCCESS;
}

int tpicb200_cycle(tpicb200_context* ctx, tpicb200_state* st, int ncycles, tpicb200_cycle_report* reports,
                   tpicb200_stream stream) {
  if (int s = check_ctx(ctx)) return s;
  if (int r = check_state(ctx, st)) return r;
  if (ncycles < 0) return fail(TPICB200_INVALID_ARGUMENT, "negative cycle count");
  const int kind = st->mass_kind;
  if (int r = check_mass_kind(ctx, kind)) return r;
  cudaStream_t s = (cudaStream_t)stream;
  cudaEvent_t* ev = ctx->events;
  cudaEvent_t* sev = ctx->events + 6;  // per species: after its mover, after its sort, after its pair's deposition
  uint32_t* perms[2] = {ctx->perm, ctx->perm2};
  for (int cycle = 0; cycle < ncycles; ++cycle) {
    tpicb200_cycle_report report{};
    cudaEventRecord(ev[0], s);
    // Field solve (reads the committed E^n, B^n and the assembled J-hat, M).
    if (int r = tpicb200_field_solve(ctx, st->e, st->b_cell, st->j, st->mass, st->e_theta, &report.gmres, stream))
      return r;
    cudaEventRecord(ev[1], s);
    // Field advance: E^{n+1} and the next B from E_theta (the movers read
    // E_theta and the old B nodes, which the advance does not touch).
    if (ctx->particle_theta) {
      // The movers gather S^n(E_theta); the field advance uses E_theta.
      const cudaError_t e = solver_smooth(ctx->solver, st->e_theta, ctx->particle_theta, s);
      if (e != cudaSuccess) return cuda_status(e, "particle-field smoothing failed");
    }
    if (int r = tpicb200_field_advance(ctx, st->e, st->b_cell, st->e_theta, st->b_cell_next, st->b_node_next, stream))
      return r;
    cudaEventRecord(ev[2], s);
    // Per pair of species: the mover and the sort of each, then one
    // deposition of both with the next B that also writes the sorted records.
    // The moment forms need no cleared J and mass: the assembly stores
    // every entry of the unique nodes and the fold copies every other vertex.
    if (moment_form(kind) && st->ns > 0) {
      ctx->moments_pending = false;
      ctx->cleared_j = st->j;
      ctx->cleared_mass = st->mass;
    } else if (int r = tpicb200_clear_moments(ctx, st->j, st->mass, stream)) {
      return r;
    }
    for (int first = 0; first < st->ns; first += 2) {
      const int count = st->ns - first < 2 ? st->ns - first : 2;
      DepositPlan plan[2];
      for (int i = 0; i < count; ++i) {
        const int sp = first + i;
        const SpeciesScalars scalars{ctx->mover_partials + size_t(kMoverPartials) * 5 * sp, kMoverPartials,
                                     &ctx->mover_written[sp]};
        if (int r = move_and_sort(ctx, st, sp, perms[i], sev[3 * sp], sev[3 * sp + 1], &plan[i],
                                  reports ? &scalars : nullptr, s))
          return r;
      }
      if (int r = deposit_pair(ctx, st, first, count, plan, first > 0, s)) return r;
      cudaEventRecord(sev[3 * first + 2], s);
    }
    if (int r = tpicb200_fold_periodic(ctx, st->j, st->mass, stream)) return r;
    cudaEventRecord(ev[3], s);
    std::swap(st->b_cell, st->b_cell_next);
    std::swap(st->b_node, st->b_node_next);
    if (reports) {
      double out[2 + 5 * TPICB200_MAX_SPECIES];
      if (int r = cycle_energy(ctx, st, out, s)) return r;
      report.field_energy[0] = out[0];
      report.field_energy[1] = out[1];
      report.total_energy = out[0] + out[1];
      for (int sp = 0; sp < st->ns; ++sp) {
        for (int q = 0; q < 5; ++q) report.species[sp][q] = out[2 + 5 * sp + q];
        report.total_energy += out[2 + 5 * sp];
      }
    }
    cudaEventRecord(ev[4], s);
    uint32_t bad = 0;
    if (int r = read_invalid(ctx, s, &bad)) return r;
    if (bad) return fail(TPICB200_INVALID_DATA, "the cycle raised the invalid-data flag");
    // Stage times: solve, move, advance, sort, deposit, fold + diagnostics.
    float t = 0.0f;
    cudaEventElapsedTime(&report.stage_ms[0], ev[0], ev[1]);
    cudaEventElapsedTime(&report.stage_ms[2], ev[1], ev[2]);
    for (int first = 0; first < st->ns; first += 2) {
      const int count = st->ns - first < 2 ? st->ns - first : 2;
      for (int i = 0; i < count; ++i) {
        const int sp = first + i;
        cudaEventElapsedTime(&t, sp == 0 ? ev[2] : (i == 0 ? sev[3 * (sp - 2) + 2] : sev[3 * (sp - 1) + 1]),
                             sev[3 * sp]);
        report.stage_ms[1] += t;
        cudaEventElapsedTime(&t, sev[3 * sp], sev[3 * sp + 1]);
        report.stage_ms[3] += t;
      }
      cudaEventElapsedTime(&t, sev[3 * (first + count - 1) + 1], sev[3 * first + 2]);
      report.stage_ms[4] += t;
    }
    const int last_pair = (st->ns - 1) / 2 * 2;
    cudaEventElapsedTime(&report.stage_ms[5], sev[3 * last_pair + 2], ev[4]);
    if (reports) reports[cycle] = report;
  }
  return TPICB200_SUCCESS;
}

}  // extern "C"

// ---- Adjoint ----------------------------------------------------------------

namespace {

int check_adjoint_context(tpicb200_context* ctx) {
  if (int s = check_ctx(ctx)) return s;
  if (ctx->particle_theta)
    return fail(TPICB200_INVALID_STATE, "the adjoint does not differentiate energy-conserving smoothing");
  return TPICB200_SUCCESS;
}

int check_gradient_records(tpicb200_context* ctx, const tpicb200_particles* p, uint32_t nid, const double* x_bar,
                           const double* v_bar) {
  if (int r = check_particles(ctx, p)) return r;
  if (p->count && !p->id) return fail(TPICB200_INVALID_ARGUMENT, "the adjoint needs record ids");
  if (p->count && (!x_bar || !v_bar || nid == 0)) return fail(TPICB200_INVALID_ARGUMENT, "null record gradients");
  return TPICB200_SUCCESS;
}

size_t field_bytes(const tpicb200_context* ctx) {
  return ctx->opt.precision == TPICB200_PRECISION_DOUBLE ? 8 : 4;
}

cudaError_t copy_records(const tpicb200_context* ctx, const tpicb200_particles* in, tpicb200_particles* out,
                         cudaStream_t s) {
  const size_t n = in->count, vb = field_bytes(ctx);
  cudaError_t e = cudaSuccess;
  auto copy = [&](void* dst, const void* src, size_t bytes) {
    if (e == cudaSuccess && bytes) e = cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToDevice, s);
  };
  copy(out->rx, in->rx, 8 * n);
  copy(out->ry, in->ry, 8 * n);
  copy(out->rz, in->rz, 8 * n);
  copy(out->u, in->u, vb * n);
  copy(out->v, in->v, vb * n);
  copy(out->w, in->w, vb * n);
  copy(out->q, in->q, 8 * n);
  copy(out->cell, in->cell, 4 * n);
  copy(out->id, in->id, 8 * n);
  out->count = in->count;
  return e;
}

}  // namespace

extern "C" {

int tpicb200_cycle_forward(tpicb200_context* ctx, tpicb200_state* st, tpicb200_tape* tape,
                           tpicb200_cycle_report* report, tpicb200_stream stream) {
  if (int s = check_adjoint_context(ctx)) return s;
  if (int r = check_state(ctx, st)) return r;
  if (!tape || tape->ns != st->ns || !tape->e || !tape->b_cell || !tape->e_theta)
    return fail(TPICB200_INVALID_ARGUMENT, "invalid tape");
  cudaStream_t s = (cudaStream_t)stream;
  if (int r = tpicb200_materialize(ctx, st, stream)) return r;
  const size_t fb = field_bytes(ctx);
  cudaError_t e = cudaSuccess;
  for (int sp = 0; sp < st->ns; ++sp) {
    const tpicb200_particles* live = &st->slot[sp][st->current[sp]];
    tpicb200_particles* out = &tape->species[sp];
    if (live->count && (!live->id || !out->id || !out->rx || !out->ry || !out->rz || !out->u || !out->v || !out->w ||
                        !out->q || !out->cell))
      return fail(TPICB200_INVALID_ARGUMENT, "the tape needs every record attribute, ids included");
    if (!tape->counts[sp] || !tape->offsets[sp]) return fail(TPICB200_INVALID_ARGUMENT, "null tape bins");
    if (e == cudaSuccess) e = copy_records(ctx, live, out, s);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(tape->counts[sp], st->counts[sp], size_t(ctx->g.bins) * 4, cudaMemcpyDeviceToDevice, s);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(tape->offsets[sp], st->offsets[sp], size_t(ctx->g.bins + 1) * 4, cudaMemcpyDeviceToDevice,
                          s);
    tape->qom[sp] = st->qom[sp];
  }
  if (e == cudaSuccess) e = cudaMemcpyAsync(tape->e, st->e, 3 * size_t(ctx->g.nodes) * fb, cudaMemcpyDeviceToDevice, s);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(tape->b_cell, st->b_cell, 3 * size_t(ctx->g.cells) * fb, cudaMemcpyDeviceToDevice, s);
  if (e != cudaSuccess) return cuda_status(e, "tape copy failed");
  tape->mass_kind = st->mass_kind;
  if (int r = tpicb200_cycle(ctx, st, 1, report, stream)) return r;
  return cuda_status(cudaMemcpyAsync(tape->e_theta, st->e_theta, 3 * size_t(ctx->g.nodes) * 8,
                                     cudaMemcpyDeviceToDevice, s),
                     "tape E_theta copy failed");
}

int tpicb200_adjoint_energy(tpicb200_context* ctx, const void* e, const void* b_cell, double we, double wb,
                            tpicb200_adjoint* adj, tpicb200_stream stream) {
  if (int s = check_ctx(ctx)) return s;
  if (!e || !b_cell || !adj || !adj->e_bar || !adj->b_bar || adj->ns < 0 || adj->ns > TPICB200_MAX_SPECIES)
    return fail(TPICB200_INVALID_ARGUMENT, "invalid adjoint energy arguments");
  cudaStream_t s = (cudaStream_t)stream;
  cudaError_t err = launch_energy_gradient(ctx->opt.precision, ctx->g, we, wb, e, b_cell, adj->e_bar, adj->b_bar, s);
  for (int sp = 0; sp < adj->ns && err == cudaSuccess; ++sp) {
    const size_t n = adj->count[sp];
    if (!n) continue;
    if (!adj->x_bar[sp] || !adj->v_bar[sp] || !adj->q_bar[sp])
      return fail(TPICB200_INVALID_ARGUMENT, "null record gradients");
    err = cudaMemsetAsync(adj->x_bar[sp], 0, 3 * n * 8, s);
    if (err == cudaSuccess) err = cudaMemsetAsync(adj->v_bar[sp], 0, 3 * n * 8, s);
    if (err == cudaSuccess) err = cudaMemsetAsync(adj->q_bar[sp], 0, n * 8, s);
  }
  return cuda_status(err, "adjoint start failed");
}

int tpicb200_field_advance_backward(tpicb200_context* ctx, double* e_bar, const double* b_bar, double* e_theta_bar,
                                    tpicb200_stream stream) {
  if (int s = check_ctx(ctx)) return s;
  if (!e_bar || !b_bar || !e_theta_bar || e_bar == e_theta_bar)
    return fail(TPICB200_INVALID_ARGUMENT, "advance backward needs distinct gradient fields");
  return cuda_status(launch_adjoint_advance(ctx->g, ctx->opt.theta, ctx->opt.c, ctx->opt.dt, e_bar, b_bar,
                                            e_theta_bar, (cudaStream_t)stream),
                     "advance backward failed");
}

int tpicb200_mover_backward(tpicb200_context* ctx, double qom, const tpicb200_particles* p, const double* e_theta,
                            const void* b_node, uint32_t nid, double* x_bar, double* v_bar, double* e_theta_bar,
                            double* b_node_bar, uint32_t* invalid, tpicb200_stream stream) {
  if (int s = check_ctx(ctx)) return s;
  if (int r = check_gradient_records(ctx, p, nid, x_bar, v_bar)) return r;
  if (!e_theta || !b_node || !e_theta_bar || !b_node_bar)
    return fail(TPICB200_INVALID_ARGUMENT, "mover backward needs its fields");
  cudaStream_t s = (cudaStream_t)stream;
  cudaError_t err = launch_adjoint_records(ctx->opt.precision, kAdjointMover, ctx->g, qom, ctx->opt.dt, ctx->opt.c, p,
                                           nid, x_bar, v_bar, nullptr, e_theta, b_node, nullptr, 0.0, nullptr,
                                           nullptr, 0.0, b_node_bar, e_theta_bar, invalid_or_own(ctx, invalid), s);
  if (err == cudaSuccess) err = launch_node_ghosts(ctx->g, e_theta_bar, 3, s);
  if (err == cudaSuccess) err = launch_node_ghosts(ctx->g, b_node_bar, 3, s);
  return cuda_status(err, "mover backward failed");
}

int tpicb200_deposit_backward(tpicb200_context* ctx, double qom, const tpicb200_particles* p, const void* b_node,
                              const double* j_bar, double j_scale, const double* mass_left,
                              const double* mass_right, double mass_scale, uint32_t nid, double* x_bar,
                              double* v_bar, double* q_bar, double* b_node_bar, uint32_t* invalid,
                              tpicb200_stream stream) {
  if (int s = check_ctx(ctx)) return s;
  if (int r = check_gradient_records(ctx, p, nid, x_bar, v_bar)) return r;
  if (!b_node || !b_node_bar || (p->count && !q_bar) || (mass_left && !mass_right))
    return fail(TPICB200_INVALID_ARGUMENT, "deposit backward needs its fields");
  cudaStream_t s = (cudaStream_t)stream;
  cudaError_t err = launch_adjoint_records(ctx->opt.precision, kAdjointDeposit, ctx->g, qom, ctx->opt.dt, ctx->opt.c,
                                           p, nid, x_bar, v_bar, q_bar, nullptr, b_node, j_bar, j_scale, mass_left,
                                           mass_right, mass_scale, b_node_bar, nullptr, invalid_or_own(ctx, invalid),
                                           s);
  if (err == cudaSuccess) err = launch_node_ghosts(ctx->g, b_node_bar, 3, s);
  return cuda_status(err, "deposit backward failed");
}

int tpicb200_field_solve_backward(tpicb200_context* ctx, const void* mass, const double* e_theta_bar, double* lambda,
                                  double* e_bar, double* b_bar, tpicb200_gmres_result* result,
                                  tpicb200_stream stream) {
  if (int s = check_adjoint_context(ctx)) return s;
  if (!mass || !e_theta_bar || !lambda || !e_bar || !b_bar || lambda == e_theta_bar)
    return fail(TPICB200_INVALID_ARGUMENT, "solve backward needs distinct fields");
  cudaStream_t s = (cudaStream_t)stream;
  cudaError_t err = cudaSuccess;
  tpicb200_gmres_result res{};
  const int status = solver_solve_adjoint(ctx->solver, e_theta_bar, mass, lambda, &res,
                                          ctx->opt.gmres_max_iterations, ctx->opt.gmres_tol, s, &err);
  if (result) *result = res;
  if (err != cudaSuccess) return cuda_status(err, "adjoint solve failed");
  if (status == TPICB200_NOT_CONVERGED) return fail(status, "the adjoint GMRES did not converge");
  if (status != TPICB200_SUCCESS) return fail(status, "the adjoint solve failed");
  err = launch_adjoint_add_nodes(ctx->g, lambda, e_bar, s);
  const double delta = ctx->opt.c * ctx->opt.theta * ctx->opt.dt;
  if (err == cudaSuccess) err = launch_adjoint_cells(ctx->g, delta, lambda, nullptr, b_bar, s);
  return cuda_status(err, "solve backward failed");
}

int tpicb200_magnetic_to_nodes_backward(tpicb200_context* ctx, const double* b_node_bar, double* b_bar,
                                        tpicb200_stream stream) {
  if (int s = check_ctx(ctx)) return s;
  if (!b_node_bar || !b_bar) return fail(TPICB200_INVALID_ARGUMENT, "null gradient field");
  return cuda_status(launch_adjoint_cells(ctx->g, 0.0, nullptr, b_node_bar, b_bar, (cudaStream_t)stream),
                     "magnetic-to-nodes backward failed");
}

int tpicb200_cycle_backward(tpicb200_context* ctx, tpicb200_tape* tape, tpicb200_adjoint* adj,
                            tpicb200_gmres_result* result, tpicb200_stream stream) {
  if (int s = check_adjoint_context(ctx)) return s;
  if (!tape || !adj || tape->ns != adj->ns || tape->ns <= 0 || tape->ns > TPICB200_MAX_SPECIES)
    return fail(TPICB200_INVALID_ARGUMENT, "invalid tape or adjoint");
  if (!adj->e_bar || !adj->b_bar || !adj->e_theta_bar || !adj->lambda || !adj->b_node_bar || !adj->b_node ||
      !adj->j || !adj->mass || !tape->e || !tape->b_cell || !tape->e_theta)
    return fail(TPICB200_INVALID_ARGUMENT, "null adjoint or tape field");
  if (int r = check_mass_kind(ctx, tape->mass_kind)) return r;
  for (int sp = 0; sp < tape->ns; ++sp) {
    if (int r = check_gradient_records(ctx, &tape->species[sp], adj->count[sp], adj->x_bar[sp], adj->v_bar[sp]))
      return r;
    if (tape->species[sp].count && !adj->q_bar[sp]) return fail(TPICB200_INVALID_ARGUMENT, "null charge gradients");
  }
  cudaStream_t s = (cudaStream_t)stream;
  const Geom& g = ctx->g;
  const int prec = ctx->opt.precision;
  const double dt = ctx->opt.dt, c = ctx->opt.c, kfac = 4 * 3.14159265358979323846 * (ctx->opt.theta * dt);
  // The cycle's B at the nodes, J and M, deposited again from the tape.
  if (int r = tpicb200_magnetic_to_nodes(ctx, tape->b_cell, adj->b_node, stream)) return r;
  if (int r = tpicb200_clear_moments(ctx, adj->j, adj->mass, stream)) return r;
  const tpicb200_particles* parts = tape->species;
  const uint32_t* const* counts = tape->counts;
  const uint32_t* const* offsets = tape->offsets;
  if (int r = tpicb200_deposit_species(ctx, tape->ns, tape->qom, parts, counts, offsets, adj->b_node, adj->j,
                                       adj->mass, tape->mass_kind, nullptr, stream))
    return r;
  if (int r = tpicb200_fold_periodic(ctx, adj->j, adj->mass, stream)) return r;
  // Advance backward, then the movers' E_theta gradient.
  cudaError_t err = launch_adjoint_advance(g, ctx->opt.theta, c, dt, adj->e_bar, adj->b_bar, adj->e_theta_bar, s);
  for (int sp = 0; sp < tape->ns && err == cudaSuccess; ++sp)
    err = launch_adjoint_theta_scatter(prec, g, tape->qom[sp], dt, c, &tape->species[sp], adj->count[sp],
                                       adj->x_bar[sp], adj->v_bar[sp], adj->b_node, adj->e_theta_bar, ctx->invalid,
                                       s);
  if (err == cudaSuccess) err = launch_node_ghosts(g, adj->e_theta_bar, 3, s);
  if (err != cudaSuccess) return cuda_status(err, "cycle backward (advance, movers) failed");
  // The solve's backward: lambda, and its E and B terms.
  if (int r = tpicb200_field_solve_backward(ctx, adj->mass, adj->e_theta_bar, adj->lambda, adj->e_bar, adj->b_bar,
                                            result, stream))
    return r;
  // The records: mover, current and mass, with the B gradient.
  err = cudaMemsetAsync(adj->b_node_bar, 0, 3 * size_t(g.nodes) * 8, s);
  for (int sp = 0; sp < tape->ns && err == cudaSuccess; ++sp)
    err = launch_adjoint_records(prec, kAdjointCycle, g, tape->qom[sp], dt, c, &tape->species[sp], adj->count[sp],
                                 adj->x_bar[sp], adj->v_bar[sp], adj->q_bar[sp], tape->e_theta, adj->b_node,
                                 adj->lambda, -kfac, adj->lambda, tape->e_theta, -kfac * g.inv_volume,
                                 adj->b_node_bar, nullptr, ctx->invalid, s);
  if (err == cudaSuccess) err = launch_node_ghosts(g, adj->b_node_bar, 3, s);
  if (err == cudaSuccess) err = launch_adjoint_cells(g, 0.0, nullptr, adj->b_node_bar, adj->b_bar, s);
  if (err != cudaSuccess) return cuda_status(err, "cycle backward (records) failed");
  uint32_t bad = 0;
  if (int r = read_invalid(ctx, s, &bad)) return r;
  if (bad) return fail(TPICB200_INVALID_DATA, "the backward met invalid records");
  return TPICB200_SUCCESS;
}

}  // extern "C"
