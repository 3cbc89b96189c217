/*
 * tpicb200.h - C ABI of the B200-native single-GPU ECSIM particle cycle.
 *
 * TPIC exposes its hot path as stream-ordered C++ template "enqueue"
 * functions that take LPFx owners, an executor (CUDA stream) and an
 * `unsigned* invalid` device flag, return an lpfx::ErrorCode, allocate
 * nothing and never synchronise (e.g.
 * include/tpic/ecsim/deposition/current_deposition_device.hpp:285-313).
 * The reference promises no binary ABI (docs/developer/architecture.md:459-460),
 * so this header is the plain-C form of those entry points: caller-owned
 * device buffers in the layouts below, a cudaStream_t, an optional device
 * `uint32_t* invalid` counter and an int status that mirrors lpfx::ErrorCode.
 *
 * Layouts (all device memory, all fully periodic grids of nx*ny*nz cells):
 *   node field  : 3 components, component-major; each component has extent
 *                 (nx+3)(ny+3)(nz+3): interior nodes 0..n plus a one-node
 *                 halo, index (i+1) + (nx+3)*((j+1) + (ny+3)*(k+1)).
 *                 Node n is the periodic duplicate of node 0 (TPIC keeps
 *                 cells+1 nodes per axis, data/fields/grid_shape.hpp:25-50).
 *   cell field  : 3 components, extent (nx+2)(ny+2)(nz+2) with a one-cell
 *                 halo, index (i+1) + (nx+2)*((j+1) + (ny+2)*(k+1)).
 *   mass records: 126 scalars per node-field vertex (same vertex index as a
 *                 node field): 14 canonical stencils x 9 row-major tensor
 *                 entries, TPIC's compact layout
 *                 (data/mass_matrix/mass_matrix_layout.hpp:11-68), or the
 *                 same entries stencil-major (tpicb200_options.mass_layout).
 *   particles   : SoA records of one species (data/particles/particle_schema.hpp:20-36):
 *                 rx, ry, rz cell-relative fractions in [0,1), u, v, w,
 *                 signed macro-charge q (double), int32 cell key
 *                 (i+2) + (nx+4)*((j+2) + (ny+4)*(k+2))
 *                 (data/particles/particle_cell.hpp:34-46), optional uint64 id.
 *   bins        : counts[(nx+4)(ny+4)(nz+4)] and offsets[bins+1] (uint32),
 *                 one bin per halo-2 cell key, as LPFx's direct-cell sort.
 *   solver field: E_theta and the other solver vectors are node fields of
 *                 double (TPIC's SolverStorage, ecsim/gmres/gmres.hpp:44-52).
 *
 * Precision modes (types of the stored quantities):
 *   TPICB200_PRECISION_DOUBLE : everything double (TPIC's "double" level).
 *   TPICB200_PRECISION_MIXED  : positions and charges double, velocities,
 *                               E, B, J and mass float; mover, current and
 *                               scalar mass arithmetic float; positions
 *                               accumulated in double; GMRES Krylov basis
 *                               float with double dots, Givens rotations,
 *                               residuals and solution (refined cycles).
 *
 * Threading: a context is used by one host thread at a time; calls are
 * stream-ordered and not re-entrant. No entry point allocates device memory
 * except tpicb200_create (the checkpoint calls stage through host memory).
 * The product fails loudly (TPICB200_BACKEND_FAILURE) without a usable
 * sm_100 device; there is no CPU fallback.
 */
#ifndef TPICB200_H
#define TPICB200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* cudaStream_t-compatible handle (0 = legacy default stream). */
typedef struct CUstream_st* tpicb200_stream;
typedef struct tpicb200_context tpicb200_context;

/* Status codes: 0-4 mirror lpfx::ErrorCode (success, invalid_argument,
 * invalid_state, overflow, backend_failure); include/lpfx/core/error.hpp. */
enum {
  TPICB200_SUCCESS = 0,
  TPICB200_INVALID_ARGUMENT = 1,
  TPICB200_INVALID_STATE = 2,
  TPICB200_OVERFLOW = 3,
  TPICB200_BACKEND_FAILURE = 4,
  TPICB200_NOT_CONVERGED = 5,     /* GMRES did not reach its tolerance */
  TPICB200_CAPACITY_EXCEEDED = 6, /* a particle count above the context's capacity */
  TPICB200_INVALID_DATA = 7       /* a cycle raised the device invalid flag */
};

enum { TPICB200_PRECISION_DOUBLE = 0, TPICB200_PRECISION_MIXED = 1 };

/* Storage order of the mass coefficients (every call of a context uses its
 * option). RECORDS is TPIC's compact layout: 126 consecutive scalars per
 * vertex (data/mass_matrix/mass_matrix_layout.hpp:30-46). STENCIL_MAJOR keeps
 * the same 126 entries as 126 arrays of node_count scalars, entry
 * k = 9*stencil + component of vertex v at k*node_count + v, so a warp
 * applying the matrix to 32 consecutive nodes reads each entry with one
 * coalesced 128-byte request. */
enum { TPICB200_MASS_LAYOUT_RECORDS = 0, TPICB200_MASS_LAYOUT_STENCIL_MAJOR = 1, TPICB200_MASS_LAYOUT_TILED = 2 };
/* TILED is STENCIL_MAJOR with each x row of a plane padded from nx+3 to a
 * multiple of 4 vertices: entry k of vertex (i, j, k3) at
 * k*plane + (i+1) + mx*((j+1) + (ny+3)*(k3+1)), mx = (nx+3) rounded up to a
 * multiple of 4, plane = mx*(ny+3)*(nz+3). Every row then starts on a 16-byte
 * boundary, so the field solve reads the mass with tensor-memory-access box
 * copies. The padding is never read or written. A mass buffer holds
 * tpicb200_layout.mass_count scalars in every layout. */

/* Mass-matrix assembly forms, the extended `--mass-matrix` selection
 * (TPIC: scalar | matrix-core, config/numerics_options.hpp:31-47). */
enum {
  TPICB200_MASS_SCALAR = 0,     /* CUDA cores, the precision mode's compute type */
  TPICB200_MASS_SCALAR_F64 = 1, /* CUDA cores, FP64 cell sums, narrowed once at the flush */
  TPICB200_MASS_TF32 = 2,       /* tcgen05 tensor cores, TF32 operands, FP32 accumulation */
  TPICB200_MASS_BF16X3 = 3,     /* tcgen05, BF16 hi/lo split products, FP32 accumulation */
  TPICB200_MASS_MOMENTS_F64 = 4 /* CUDA cores, FP64 per-cell moments (27 pair-weight classes x
                                   (9 response + 3 current) entries), then a per-node assembly;
                                   DOUBLE precision only */
};

typedef struct {
  int nx, ny, nz;       /* cells per axis (fully periodic) */
  double lx, ly, lz;    /* box lengths */
} tpicb200_grid;

typedef struct {
  double dt, theta, c;      /* time step, implicitness, light speed (TPIC admits c = 1) */
  double gmres_tol;         /* relative tolerance of the true residual */
  int gmres_restart;        /* 30 in TPIC (config/physics.hpp:20) */
  int gmres_max_iterations; /* 100 in TPIC (config/physics.hpp:21) */
  int precision;            /* TPICB200_PRECISION_* */
  uint32_t max_particles;   /* capacity of the sort scratch (largest species) */
  int mass_layout;          /* TPICB200_MASS_LAYOUT_* (0: TPIC records) */
  /* Energy-conserving smoothing (TPIC ECSimSmoothing = energy_conserving,
   * config/physics.cpp:65-70): on when smooth_iterations > 0 and
   * smooth_alpha < 1. Zero-initialized options leave it off. */
  int smooth_iterations;    /* SmoothNiter: passes of S, >= 0 */
  double smooth_alpha;      /* Smooth: Face7 centre weight in [0, 1] */
  int smooth_operator;      /* TPICB200_SMOOTH_FACE7 or TPICB200_SMOOTH_BINOMIAL27 */
} tpicb200_options;
enum { TPICB200_SMOOTH_FACE7 = 0, TPICB200_SMOOTH_BINOMIAL27 = 1 };

typedef struct {
  void* rx; void* ry; void* rz; /* double */
  void* u; void* v; void* w;    /* double (DOUBLE) or float (MIXED) */
  double* q;
  int32_t* cell;
  uint64_t* id;                 /* may be NULL */
  uint32_t count;
} tpicb200_particles;

typedef struct {
  int64_t node_count;     /* elements per node-field component */
  int64_t cell_count;     /* elements per cell-field component */
  int64_t bin_count;      /* halo-2 particle bins */
  int64_t interior_nodes; /* (nx+1)(ny+1)(nz+1): GMRES vector length / 3 */
  size_t field_scalar_bytes; /* sizeof E/B/J scalars: 8 (DOUBLE) or 4 (MIXED) */
  size_t mass_scalar_bytes;  /* sizeof mass scalars */
  size_t velocity_scalar_bytes;
  int64_t mass_count;        /* scalars of a mass buffer in the context's layout */
} tpicb200_layout;

typedef struct {
  int converged, iterations;
  double initial_residual, residual, rhs_norm, relative_residual;
  int host_waits;  /* times the solve waited for the device (once per restart cycle, plus one) */
} tpicb200_gmres_result;

/* Whole-cycle state: every pointer is a caller-owned device buffer.
 * Particles are double-buffered per species (slot[s][current] is live; the
 * sort writes the other slot and flips current). */
#define TPICB200_MAX_SPECIES 8
typedef struct {
  int ns;
  double qom[TPICB200_MAX_SPECIES];
  tpicb200_particles slot[TPICB200_MAX_SPECIES][2];
  int current[TPICB200_MAX_SPECIES];
  uint32_t* counts[TPICB200_MAX_SPECIES];  /* bins of the live slot */
  uint32_t* offsets[TPICB200_MAX_SPECIES];
  void* e;          /* node field, committed E^n */
  void* b_cell;     /* cell field, committed B^n */
  void* b_node;     /* node field, particle-facing B^n */
  void* b_cell_next;
  void* b_node_next;
  void* j;          /* node field, assembled J-hat */
  void* mass;       /* mass records */
  double* e_theta;  /* solver node field */
  int mass_kind;    /* TPICB200_MASS_* */
  /* Optional rank buffers (uint32, the slots' capacity; NULL: not used).
   * With ranks[s] set, tpicb200_cycle leaves species s ranked (ranked[s]
   * nonzero): the live slot holds the moved records in the order of the
   * previous sort and ranks[s][p] is the live record at sorted position p of
   * the bins counts/offsets; the next cycle's mover reads through the ranks
   * and writes the moved records in that order into the idle slot, the sort
   * only ranks, the deposition reads through the ranks. tpicb200_materialize
   * writes the sorted records into the live slot (ranked[s] = 0). */
  uint32_t* ranks[TPICB200_MAX_SPECIES];
  int ranked[TPICB200_MAX_SPECIES];
} tpicb200_state;

typedef struct {
  tpicb200_gmres_result gmres;
  double field_energy[2];               /* electric, magnetic after the cycle */
  double species[TPICB200_MAX_SPECIES][5]; /* kinetic, charge, momentum x/y/z */
  double total_energy;
  float stage_ms[6]; /* solve, move, advance, sort, deposit, fold+diagnostics */
} tpicb200_cycle_report;

const char* tpicb200_version(void);
/* Message of the last failure on the calling thread. */
const char* tpicb200_last_error(void);
/* Number of kernels this library has launched since it was loaded (a
 * host-side count kept by every launch site; for benchmarks and tests). */
unsigned long long tpicb200_launch_count(void);

/* Set up a context: geometry, constants and the solver/sort workspace.
 * Replaces the owner construction of MaxwellOperator, Gmres and the sort
 * workspace (ecsim/maxwell/maxwell_device.hpp:60-95,
 * ecsim/gmres/gmres_device.hpp:316-336). The calling thread's current CUDA
 * device is used. */
int tpicb200_create(const tpicb200_grid* grid, const tpicb200_options* options,
                    tpicb200_context** out);
int tpicb200_destroy(tpicb200_context* ctx);
int tpicb200_get_layout(const tpicb200_context* ctx, tpicb200_layout* out);

/* Implicit theta-scheme mover of one species over `p->count` records:
 * v_new = 2*(alpha v + beta alpha E_theta) - v, x += dt v_new, periodic wrap.
 * Replaces enqueue_local_particle_mover (ecsim/particles/particle_mover_device.hpp:310-328).
 * e_theta: solver node field; b_node: the old particle-facing B (node field).
 * An invalid record keeps its attributes and increments *invalid. */
int tpicb200_mover(tpicb200_context* ctx, double qom, tpicb200_particles* p,
                   const double* e_theta, const void* b_node, uint32_t* invalid,
                   tpicb200_stream stream);

/* Stable counting sort by cell key: out receives the records of `in` in key
 * order (equal keys keep their input order), counts/offsets the bins.
 * Replaces FullParticleSort::enqueue (ecsim/particles/particle_sort_device.hpp:132-145)
 * whose device sort is unstable within a bin; this one is bit-exact against
 * the stable host sort (lpfx/algorithm/particle/host/sort.hpp:205-290).
 * in and out must not alias; an out-of-range key stops the sort on the
 * device (no record is written) and increments *invalid. */
int tpicb200_sort(tpicb200_context* ctx, const tpicb200_particles* in, tpicb200_particles* out,
                  uint32_t* counts, uint32_t* offsets, uint32_t* invalid,
                  tpicb200_stream stream);

/* Stable sort of records that are grouped by the bins (in_counts,
 * in_offsets) of an earlier tpicb200_sort and whose keys changed since (the
 * mover updates keys in place): the same output, counts and offsets as
 * tpicb200_sort of the same input. When every record moved to one of the 27
 * cells around its bin (periodic) and the old bins tile the records in key
 * order, the records go straight to their output positions through per-cell
 * transfer counts; any other input takes the general path, which the device
 * selects without a host round trip. in_counts/in_offsets may alias
 * counts/offsets (they are read before the new bins are written). No single
 * reference counterpart: it replaces FullParticleSort::enqueue
 * (simulation/actions/local_species_actions_device.hpp:202-216 ->
 * lpfx/algorithm/particle/device/cuda_hip/sort.hpp:64-260) on the cycle's
 * post-mover sort. */
int tpicb200_sort_binned(tpicb200_context* ctx, const tpicb200_particles* in, const uint32_t* in_counts,
                         const uint32_t* in_offsets, tpicb200_particles* out, uint32_t* counts,
                         uint32_t* offsets, uint32_t* invalid, tpicb200_stream stream);

/* Capacity of tpicb200_sort_static: records per call and halo-2 bins
 * ((nx+4)(ny+4)(nz+4)) of the grid. */
#define TPICB200_SORT_STATIC_MAX_RECORDS 1048576
#define TPICB200_SORT_STATIC_MAX_BINS 1048576

/* The stable counting sort of tpicb200_sort (same output, counts, offsets
 * and invalid-key behaviour) without a context and without allocating
 * anything: its scratch (permutation, cursors, scan sums; 12.6 MB) is one
 * fixed device array of the library. No counterpart in the reference: it
 * serves callers that cannot allocate device memory for a sort (no context,
 * memory held by another allocator's pool, or a loop that must not pay an
 * allocation's implicit device synchronisation). Limits: at most
 * TPICB200_SORT_STATIC_MAX_RECORDS records on grids of at most
 * TPICB200_SORT_STATIC_MAX_BINS bins; larger inputs return
 * TPICB200_CAPACITY_EXCEEDED and enqueue nothing. The calling thread's
 * current CUDA context is used (the current device's primary context when
 * none is current). The first call in each context resolves the array's
 * address in that context; make that call before any stream capture. The
 * address is cached per context id, so a context created later (after
 * cudaDeviceReset, or a driver context made current) resolves its own.
 * Every call shares the one array: calls
 * that overlap in time (on other streams or host threads) race on it and
 * must be ordered on one stream. precision: TPICB200_PRECISION_* (the
 * velocity type of the records). */
int tpicb200_sort_static(const tpicb200_grid* grid, int precision, const tpicb200_particles* in,
                         tpicb200_particles* out, uint32_t* counts, uint32_t* offsets, uint32_t* invalid,
                         tpicb200_stream stream);

/* S^n of a double node field (ghosts of `in` filled) into `out` with its
 * ghosts filled: the context's energy-conserving smoothing, n passes of
 * Face7 (alpha centre, (1-alpha)/6 faces) or Binomial27 ([1,2,1]^3/64) over
 * the interior nodes in the field arithmetic of the precision mode. The
 * particle field of a smoothed run is S^n(E_theta); tpicb200_cycle applies it
 * itself. Replaces MaxwellOperator::complete_smoothing
 * (ecsim/maxwell/maxwell_device.hpp:455-487) with node_smoothing_value
 * (ecsim/fields/node_smoothing.hpp:24-52). Returns TPICB200_INVALID_STATE
 * when the context has no smoothing; in and out must not alias. */
int tpicb200_smooth(tpicb200_context* ctx, const double* in, double* out, tpicb200_stream stream);

/* The context's own invalid counter (the one entry points use when their
 * `invalid` argument is NULL, and the one tpicb200_cycle and the solver's
 * smoothing passes raise): *count receives its value once the work enqueued
 * on `stream` so far has completed; clear != 0 then zeroes it (stream
 * ordered). TPIC's callers read their `unsigned* invalid` flag the same way
 * after the enqueued work (simulation/driver/pipeline.hpp:145-146). Host-blocking. */
int tpicb200_read_invalid(tpicb200_context* ctx, uint32_t* count, int clear, tpicb200_stream stream);

/* Bound of the device-side waits: polls before a wait gives up, 0 restoring
 * the default of 4,194,304.
 * - The BF16X3 tensor-core deposition (the wait for a chunk's MMAs and for
 *   the issuer's published decision): a wait that gives up makes its CTA
 *   leave the chunk loop, wait (with the default bound) for the MMAs it has
 *   in flight and free its tensor memory; the deposition adds 1 << 20 to the
 *   invalid counter.
 * - The operator apply that stages mass boxes by TMA (mass buffers with
 *   16-byte rows: the tiled layout): a wait for a box that gives up makes
 *   its CTA wait (with the default bound) for its copies in flight and
 *   return without writing its rows; the apply adds 1 << 21 to the invalid
 *   counter.
 * tpicb200_cycle then returns TPICB200_INVALID_DATA. */
int tpicb200_set_wait_limit(tpicb200_context* ctx, uint32_t polls);

/* Test of the bounded waits (tpicb200_set_wait_limit) without a fault: with
 * site TPICB200_STALL_DEPOSIT the tensor-core deposition's wait for the MMAs
 * of chunk index - 1 (index >= 1), with TPICB200_STALL_APPLY the TMA apply's
 * wait for the mass box of stencil `index` (0..13) waits instead on an
 * mbarrier that nothing arrives on, so it gives up at its bound and takes
 * the recovery path above. TPICB200_STALL_NONE turns it off. */
enum { TPICB200_STALL_NONE = 0, TPICB200_STALL_DEPOSIT = 1, TPICB200_STALL_APPLY = 2 };
int tpicb200_inject_stall(tpicb200_context* ctx, int site, uint32_t index);

/* Zero J (node field) and the mass records. Replaces enqueue_clear_mass_matrix
 * (ecsim/mass_matrix/mass_matrix_deposition_device.hpp:107-121) and the moment clear. */
int tpicb200_clear_moments(tpicb200_context* ctx, void* j, void* mass, tpicb200_stream stream);

/* Implicit current and mass-matrix deposition of one species, added into j
 * and mass (either may be NULL for the scalar forms) at the periodic unique
 * nodes; call tpicb200_fold_periodic after the last species. The
 * tensor-core forms (TF32, BF16X3; mixed precision, sorted bins) keep the
 * cell moments of every species deposited since tpicb200_clear_moments in
 * the context and tpicb200_fold_periodic adds them into j and mass, with no
 * atomics and a fixed summation order. With counts/offsets (the
 * bins of p, from tpicb200_sort) the sorted cell-tile kernels run; with NULL
 * bins the per-particle kernels run (scalar forms only). Replaces
 * enqueue_sorted_current / enqueue_unsorted_current
 * (ecsim/deposition/current_deposition_device.hpp:340-421) and
 * enqueue_sorted_mass_matrix<Kernel> / enqueue_unsorted_mass_matrix
 * (ecsim/mass_matrix/mass_matrix_deposition_device.hpp:124-182). */
int tpicb200_deposit(tpicb200_context* ctx, double qom, const tpicb200_particles* p,
                     const uint32_t* counts, const uint32_t* offsets, const void* b_node,
                     void* j, void* mass, int mass_kind, uint32_t* invalid,
                     tpicb200_stream stream);

/* Deposition of ns species (arrays of ns entries: q/m, records and their
 * bins) with the semantics of ns calls of tpicb200_deposit. The tensor-core
 * forms read the records of both species of a pair in one pass over the
 * cells (one record stream per cell, species in array order), so a cell's
 * chunk padding and its moment store are paid once per pair. No single
 * reference counterpart: the reference enqueues one species at a time
 * (enqueue_sorted_mass_matrix, ecsim/mass_matrix/mass_matrix_deposition_device.hpp:124-182,
 * from the species loop of simulation/actions/local_species_actions_device.hpp). */
int tpicb200_deposit_species(tpicb200_context* ctx, int ns, const double* qom,
                             const tpicb200_particles* species, const uint32_t* const* counts,
                             const uint32_t* const* offsets, const void* b_node, void* j, void* mass,
                             int mass_kind, uint32_t* invalid, tpicb200_stream stream);

/* Periodic fold: pending tensor-core cell moments are assembled into the
 * unique nodes, then the duplicate endpoint nodes and the one-node ghosts
 * of j and of the mass records take the values of their periodic unique node.
 * Replaces the self-periodic J.add/ghost exchange and the compact mass halo
 * (ecsim/deposition/current_assembly_device.hpp:26-53,
 * communication/mass_halo/mass_halo_device.hpp:91-160,350-364). */
int tpicb200_fold_periodic(tpicb200_context* ctx, void* j, void* mass, tpicb200_stream stream);

/* out = M * in / V at the interior nodes (double node fields, in with
 * ghosts). Replaces enqueue_mass_matrix_apply (ecsim/mass_matrix/mass_matrix_apply_device.hpp:65-96). */
int tpicb200_mass_apply(tpicb200_context* ctx, const void* mass, const double* in, double* out,
                        tpicb200_stream stream);

/* Field solve: rhs = E + delta curl_C2N(B) - k J; GMRES(restart) on
 * A(v) = v + delta^2 curl_C2N curl_N2C v + k M v / V from the guess E; writes
 * E_theta (interior nodes and ghosts) when converged. Host-blocking like
 * Gmres::host_blocking_solve (ecsim/gmres/gmres_device.hpp:353-454), which
 * reads two scalars back per Arnoldi step; here the steps of a restart cycle
 * run as one CUDA graph (a WHILE node) and the host waits once per restart
 * cycle plus once for the initial residual. With the environment variable
 * TPICB200_STEP_GRAPH=0 when the context is created, the host steps the loop
 * (one wait per step). b_cell needs filled ghosts. */
int tpicb200_field_solve(tpicb200_context* ctx, const void* e, const void* b_cell, const void* j,
                         const void* mass, double* e_theta, tpicb200_gmres_result* result,
                         tpicb200_stream stream);

/* Field advance: e <- E_theta/theta - (1-theta)/theta e; b_cell_next <-
 * b_cell - c dt curl_N2C(E_theta) with periodic ghosts; b_node_next <-
 * cell_to_node(b_cell_next). Replaces MaxwellOperator::enqueue_next_e_and_cell
 * and enqueue_next_cell_closure_and_node_interpolation (ecsim/maxwell/maxwell_device.hpp:234-252). */
int tpicb200_field_advance(tpicb200_context* ctx, void* e, const void* b_cell,
                           const double* e_theta, void* b_cell_next, void* b_node_next,
                           tpicb200_stream stream);

/* Particle-facing B: b_node <- cell_to_node(b_cell) (ghosts of b_cell are
 * refreshed first). Startup form of complete_initial_magnetic_field. */
int tpicb200_magnetic_to_nodes(tpicb200_context* ctx, void* b_cell, void* b_node,
                               tpicb200_stream stream);

/* Scalar diagnostics (diagnostics/scalar_diagnostics_device.hpp:49-133):
 * out[0] = V/(8 pi) sum |E|^2 over unique nodes, out[1] = V/(8 pi) sum |B|^2
 * over cells, then per species kinetic energy, charge, momentum x/y/z.
 * Host-blocking (synchronises `stream`). */
int tpicb200_energy(tpicb200_context* ctx, const void* e, const void* b_cell,
                    const tpicb200_particles* species, const double* qom, int ns, double* out,
                    tpicb200_stream stream);

/* Startup: B nodes from cells, the first sort and the bootstrap deposition
 * (docs/developer/architecture.md:161-171). */
int tpicb200_prepare(tpicb200_context* ctx, tpicb200_state* state, tpicb200_stream stream);

/* Sorted records of every ranked species: the live records are gathered
 * through their ranks into the idle slot, which becomes live (ranked[s] = 0).
 * A no-op for species that are not ranked. */
int tpicb200_materialize(tpicb200_context* ctx, tpicb200_state* state, tpicb200_stream stream);

/* ncycles ECSIM cycles: solve; per species the mover (old B) and the sort
 * of the moved records (the mover emits the direction codes the binned sort
 * places records by, see tpicb200_sort_binned); field advance; deposition
 * of every species (next B); fold; commit. reports (may be NULL) receive one
 * entry per cycle with the energies of the committed state. Host-blocking;
 * returns TPICB200_INVALID_DATA when a cycle raised the invalid flag. */
int tpicb200_cycle(tpicb200_context* ctx, tpicb200_state* state, int ncycles,
                   tpicb200_cycle_report* reports, tpicb200_stream stream);

/* ------------------------------------------------------------------------
 * Adjoint: reverse-mode gradients of the cycle.
 *
 * TPIC has no adjoint. These entry points transpose this library's forward
 * stages so that the gradient of an objective of the state after n cycles
 * (e.g. the final field energy) with respect to the state before them is
 * carried back cycle by cycle, shaped like a torch.autograd.Function: a
 * forward call saves what the backward needs (the tape), a backward call
 * takes the gradients of a stage's outputs and returns those of its inputs.
 * The transpose of each scatter is a gather at the particle positions (the
 * current and mass deposition's backward), the transpose of each gather a
 * scatter (the mover's backward), and the solve's backward is a GMRES solve
 * with A^T (every 3x3 mass block transposed; the curl-curl part is symmetric).
 * Gradients are FP64 in both precision modes. Smoothing is not differentiated
 * (TPICB200_INVALID_STATE).
 *
 * Gradient layouts: node and cell fields of double in the field layouts
 * above, holding the gradient with respect to the unique periodic values
 * (duplicate endpoint nodes and ghosts hold copies); per species, indexed by
 * record id (ids 0..count-1, as the loader assigns them): x_bar[3][count]
 * (per axis, with respect to the position in cells), v_bar[3][count],
 * q_bar[count].
 * ------------------------------------------------------------------------ */
typedef struct {
  int ns;
  double* e_bar;                        /* node field: d/dE */
  double* b_bar;                        /* cell field (ghosts filled): d/dB */
  double* x_bar[TPICB200_MAX_SPECIES];  /* [3][count] */
  double* v_bar[TPICB200_MAX_SPECIES];  /* [3][count] */
  double* q_bar[TPICB200_MAX_SPECIES];  /* [count]: summed over every cycle carried back */
  uint32_t count[TPICB200_MAX_SPECIES]; /* records (ids) per species */
  /* Scratch of tpicb200_cycle_backward: double node fields, and B at the
   * nodes, J and the mass records in the storage types of the context. */
  double* e_theta_bar;
  double* lambda;
  double* b_node_bar;
  void* b_node;
  void* j;
  void* mass;
} tpicb200_adjoint;

/* What the backward of one cycle needs: the state at the cycle's start
 * (sorted records with ids, their bins, E at the nodes and B at the cells,
 * in the storage types) and the cycle's E_theta. Caller-owned device
 * buffers; species[s] holds room for the species' records. */
typedef struct {
  int ns;
  double qom[TPICB200_MAX_SPECIES];
  tpicb200_particles species[TPICB200_MAX_SPECIES];
  uint32_t* counts[TPICB200_MAX_SPECIES];
  uint32_t* offsets[TPICB200_MAX_SPECIES];
  void* e;
  void* b_cell;
  double* e_theta;
  int mass_kind;
} tpicb200_tape;

/* One cycle of tpicb200_cycle that first saves its starting state into the
 * tape (ranked species are materialized) and then the cycle's E_theta. The
 * state's records need ids. Host-blocking like tpicb200_cycle. */
int tpicb200_cycle_forward(tpicb200_context* ctx, tpicb200_state* state, tpicb200_tape* tape,
                           tpicb200_cycle_report* report, tpicb200_stream stream);

/* The backward of the cycle recorded in `tape`: on entry adj holds the
 * gradients with respect to the state after the cycle, on return those with
 * respect to the state at its start (q_bar accumulates). Steps: B at the
 * nodes and the deposition of the tape's records (J and M into the adjoint's
 * scratch, the tape's mass form), the advance's backward, the scatter of the
 * movers' E_theta gradient, the solve with A^T (the context's GMRES tolerance
 * and step limit; result may be NULL), the records' backward (mover, current
 * and mass, with the B gradient scattered), and the fields' backward. The
 * host waits for the adjoint solve as for the forward one. */
int tpicb200_cycle_backward(tpicb200_context* ctx, tpicb200_tape* tape, tpicb200_adjoint* adj,
                            tpicb200_gmres_result* result, tpicb200_stream stream);

/* Starts a backward run: adj->e_bar and adj->b_bar receive the gradient of
 * we * W_E + wb * W_B of the fields e (node) and b_cell (cell, storage types),
 * the energies of tpicb200_energy (W_E over the unique nodes, W_B over the
 * cells); the particle gradients of adj's ns species are zeroed. */
int tpicb200_adjoint_energy(tpicb200_context* ctx, const void* e, const void* b_cell, double we, double wb,
                            tpicb200_adjoint* adj, tpicb200_stream stream);

/* Stage backwards (the transposes of the stage entry points above). Each
 * adds into the unique values of its gradient outputs and refills their
 * duplicates and ghosts. */

/* Backward of tpicb200_field_advance: e_bar holds d/dE' on entry and d/dE
 * (from the advance alone) on return; e_theta_bar receives
 * e_bar'/theta - c dt C2N(b_bar'); b_bar (d/dB' = d/dB) is read. */
int tpicb200_field_advance_backward(tpicb200_context* ctx, double* e_bar, const double* b_bar, double* e_theta_bar,
                                    tpicb200_stream stream);

/* Backward of tpicb200_mover for records p (sorted by cell for speed, with
 * ids below nid) as they were before the move: x_bar/v_bar hold the
 * gradients of the moved records on entry and of the records before the
 * move on return; the gradients of E_theta and of B at the nodes are added
 * into e_theta_bar and b_node_bar. */
int tpicb200_mover_backward(tpicb200_context* ctx, double qom, const tpicb200_particles* p, const double* e_theta,
                            const void* b_node, uint32_t nid, double* x_bar, double* v_bar, double* e_theta_bar,
                            double* b_node_bar, uint32_t* invalid, tpicb200_stream stream);

/* Backward of tpicb200_deposit for the objective
 *   j_scale <j_bar, J> + mass_scale <mass_left, M mass_right>
 * (M the mass matrix applied without its 1/V row scale; j_bar, mass_left
 * and mass_right double node fields with ghosts, any may be NULL): the
 * gradients are added into x_bar, v_bar, q_bar and b_node_bar. In a cycle,
 * j_bar = mass_left = lambda, j_scale = -k, mass_right = E_theta,
 * mass_scale = -k/V. */
int tpicb200_deposit_backward(tpicb200_context* ctx, double qom, const tpicb200_particles* p, const void* b_node,
                              const double* j_bar, double j_scale, const double* mass_left,
                              const double* mass_right, double mass_scale, uint32_t nid, double* x_bar,
                              double* v_bar, double* q_bar, double* b_node_bar, uint32_t* invalid,
                              tpicb200_stream stream);

/* Backward of tpicb200_field_solve: lambda = A^-T e_theta_bar (GMRES from a
 * zero guess, the context's tolerance), then e_bar += lambda and
 * b_bar += delta N2C(lambda) (the right-hand side's E and B terms); the
 * gradients of J and M are -k lambda and -(k/V) lambda E_theta^T (pass them
 * to tpicb200_deposit_backward). Host-blocking like the forward solve. */
int tpicb200_field_solve_backward(tpicb200_context* ctx, const void* mass, const double* e_theta_bar, double* lambda,
                                  double* e_bar, double* b_bar, tpicb200_gmres_result* result,
                                  tpicb200_stream stream);

/* Backward of tpicb200_magnetic_to_nodes: b_bar += cell_to_node^T(b_node_bar). */
int tpicb200_magnetic_to_nodes_backward(tpicb200_context* ctx, const double* b_node_bar, double* b_bar,
                                        tpicb200_stream stream);

/* ------------------------------------------------------------------------
 * Input decks and analytic initial cases (host code, no device needed).
 *
 * TPIC reads a run from an input deck of `key = value` lines ('#' starts a
 * comment, a list is whitespace-separated, the last assignment of a key
 * wins; src/config/simulation_parameters.cpp:55-200) and prepares the case
 * the deck's `Case` names (include/tpic/initialization/cases/initial_case.hpp:27-60).
 * These entry points read the keys of the periodic, unsmoothed, one-rank
 * path and the cases built here: Uniform, Weibel, TwoStream and the Harris
 * sheet family (GEMHarris, GEM, GEMnoPert, DoubleGEM, DoubleGEMnoPert,
 * plasmoidChain), with energy-conserving smoothing. Other case names, wall
 * boundaries and Ampere currents are rejected with TPICB200_INVALID_ARGUMENT.
 * ------------------------------------------------------------------------ */
#define TPICB200_CASE_NAME_MAX 32
typedef struct {
  double rho;          /* rhoINIT */
  double qom;          /* qom */
  double vth[3];       /* uth, vth, wth */
  double drift[3];     /* u0, v0, w0 */
  int npcel[3];        /* npcelx, npcely, npcelz */
  int center_velocity; /* CenterInitialVelocity */
} tpicb200_deck_species;

typedef struct {
  char case_name[TPICB200_CASE_NAME_MAX]; /* Case */
  tpicb200_grid grid;                     /* Lx, Ly, Lz, nxc, nyc, nzc */
  double dt, theta, c, gmres_tol;         /* dt, th, c, GMREStol */
  int ncycles;                            /* ncycles */
  int ns;                                 /* ns */
  tpicb200_deck_species species[TPICB200_MAX_SPECIES];
  double b0[3];                           /* B0x, B0y, B0z (uniform background) */
  /* Harris sheet family (harris_sheet.hpp) */
  double delta, harris_b0x;               /* delta, HarrisB0x */
  double pert_gem, pert_hump;             /* pertGEM, pertHump */
  double deltax_hump, deltay_hump;        /* deltaxHump, deltayHump */
  double kx_hump, ky_hump;                /* kxHump, kyHump (negative: box modes) */
  /* Weibel (weibel.hpp) */
  int weibel_mode_x;                      /* WeibelSeedModeX */
  double weibel_amplitude;                /* WeibelSeedAmplitude */
  double weibel_growth_rate;              /* WeibelSeedGrowthRate */
  /* TwoStream (two_stream.hpp) */
  int two_stream_mode_x;                  /* TwoStreamSeedModeX */
  double two_stream_amplitude;            /* TwoStreamSeedDensityAmplitude */
  double two_stream_phase;                /* TwoStreamSeedPhase */
  int quiet_start;                        /* QuietStart: subcell centres */
  int ignored_keys;                       /* deck keys this front end does not read */
  /* ECSimSmoothing = energy_conserving (config/physics.cpp:65-70): SmoothNiter
   * (default 6), Smooth (default 1) and ECSimSmoothingOperator (face7 or
   * binomial27, as TPICB200_SMOOTH_*); smooth_iterations is 0 when off. */
  int smooth_iterations;
  double smooth_alpha;
  int smooth_operator;
} tpicb200_deck;

/* Fills *out from the deck text with TPIC's defaults for absent keys
 * (th = 1, c = 1, GMREStol = 1e-3, delta = 0.5, deltaxHump = 8,
 * deltayHump = 4, kxHump = kyHump = -1). Replaces SimulationParameters'
 * parse_simulation_parameters (src/config/simulation_parameters.cpp:208-396)
 * for these keys; a malformed line, a missing required key (dt, ncycles,
 * ns, Case, per-species lists), too short a list, an unknown case name or
 * an out-of-scope option returns TPICB200_INVALID_ARGUMENT with the line
 * and key in tpicb200_last_error(). */
int tpicb200_deck_parse(const char* text, tpicb200_deck* out);

/* The case's analytic initial fields at n physical points (x, y, z),
 * double precision: e[3n] and b[3n] (component-major: e[c*n + p]); b
 * includes the uniform background B0 once. Replaces initial_electric and
 * initial_magnetic (src/initialization/initial_case.cpp:146-162) with the
 * case coefficients of prepare_initial_case; returns
 * TPICB200_INVALID_ARGUMENT when the case is not admitted and
 * TPICB200_OVERFLOW for a nonfinite coordinate or sample. */
int tpicb200_case_fields(const tpicb200_deck* deck, long long n, const double* x, const double* y,
                         const double* z, double* e, double* b);

/* The loading profile of species s at n particles: physical position
 * (x, y, z) and cell row j (the y cell index of the particle's cell). Writes
 * the density sample (rhoINIT/(4 pi), shaped by the case), the density
 * multiplier and the drift (drift[3n], component-major); the macro-charge
 * is then q = (sign(qom) (dx dy) dz / ppc * density) * multiplier and the
 * velocity drift + thermal * normal. Replaces the case Profile::evaluate of
 * initial_particle_load_kernel (initialization/particles/particle_loading_device.hpp:120-143,
 * cases/case_interface.hpp:60-77): TwoStream's electron density seed, the
 * Harris sheet density of drifting species (the mean of the cell's two
 * y-node values of sech^2) and the double sheet's drift sign. */
int tpicb200_case_profile(const tpicb200_deck* deck, int s, long long n, const double* x, const double* y,
                          const double* z, const int* cell_j, double* density, double* multiplier,
                          double* drift);

/* ------------------------------------------------------------------------
 * Device particle loading.
 * ------------------------------------------------------------------------ */

/* Loads records [first, first + p->count) of species s of the deck into p,
 * in load order, on the stream: TPIC's dense load (initial_particle_load_kernel,
 * initialization/particles/particle_loading_device.hpp:75-160) with this
 * library's random stream in place of cuRAND XORWOW. Record n of species s:
 *   two Philox-4x32-10 blocks (Salmon et al., SC'11) with counter
 *   (n mod 2^32, n / 2^32, s, 0 | 1) and key (seed mod 2^32, seed / 2^32);
 *   uniforms (r + 1/2) 2^-32: block 0 words 0-2 are the subcell offsets
 *   (1/2 with QuietStart), word 3 with block 1 words 0-2 give three normals
 *   by Box-Muller, (sqrt(-2 ln u1) cos(2 pi u2), sqrt(-2 ln u1) sin(2 pi u2),
 *   sqrt(-2 ln u3) cos(2 pi u4));
 *   cell = n / ppc and subcell = n mod ppc (x fastest), fraction
 *   (subcell + offset) / npcel per axis, a fraction of exactly one carrying
 *   into the next (periodic) cell;
 *   the case profile at the stored position and cell gives the density,
 *   multiplier and drift (tpicb200_case_profile); velocity drift + thermal *
 *   normal stored in the context's velocity type, charge (q_factor *
 *   density) * multiplier, id n.
 * The deck's grid must be the context's. A nonfinite velocity or charge
 * counts in *invalid (NULL: the context's counter). */
int tpicb200_load_species(tpicb200_context* ctx, const tpicb200_deck* deck, int s, uint64_t seed,
                          uint64_t first, tpicb200_particles* p, uint32_t* invalid, tpicb200_stream stream);

/* CenterInitialVelocity of species s, p holding the whole species as loaded
 * (before any sort or move): the loaded drift is removed from every
 * velocity, the charge-weighted mean of the rest (FP64 sums in a fixed
 * order) is subtracted and the drift put back, each stored velocity formed
 * in double and narrowed once (initialization/particles/particle_centering_device.hpp:36-100).
 * A zero charge sum leaves the rest unshifted; a nonfinite sum, mean or
 * velocity counts in *invalid. Stream-ordered. */
int tpicb200_center_velocities(tpicb200_context* ctx, const tpicb200_deck* deck, int s, tpicb200_particles* p,
                               uint32_t* invalid, tpicb200_stream stream);

/* ------------------------------------------------------------------------
 * Checkpoints and restart (docs/user/output.md "Checkpoints and restart",
 * src/io/checkpoint.cpp): a checkpoint holds E at the nodes, B at the cells
 * and every particle record in their stored types, with the cycle number;
 * everything else is rebuilt at restart by tpicb200_prepare. One piece file
 * per checkpoint directory `<directory>/checkpoint_tNNNNNN_n000001/
 * checkpoint_tNNNNNN_r000000.tpcb` (this library's binary format: a header
 * and the arrays, with an FNV-1a 64-bit checksum of the payload). A piece is
 * written under a hidden name, flushed and renamed, so a checkpoint is
 * complete when its piece is listed; writing one removes the older complete
 * checkpoints of the directory.
 * ------------------------------------------------------------------------ */
typedef struct {
  int version;                    /* format version (1) */
  int precision;                  /* TPICB200_PRECISION_* of the stored types */
  int cycle;                      /* cycles completed at the checkpoint */
  int ns;
  tpicb200_grid grid;
  double dt, c;
  double qom[TPICB200_MAX_SPECIES];
  uint32_t count[TPICB200_MAX_SPECIES];  /* records per species */
  int has_id[TPICB200_MAX_SPECIES];      /* ids stored */
} tpicb200_checkpoint_info;

/* Writes the state (after tpicb200_prepare or a cycle; ranked species are
 * materialized first) as the checkpoint of `cycle` under `directory`
 * (created if absent). Host-blocking. TPICB200_BACKEND_FAILURE for a file
 * system error, with the path in tpicb200_last_error(). */
int tpicb200_checkpoint_write(tpicb200_context* ctx, tpicb200_state* state, const char* directory, int cycle,
                              tpicb200_stream stream);

/* The newest complete checkpoint piece under `directory` into path[size]:
 * TPICB200_SUCCESS, or TPICB200_INVALID_ARGUMENT when there is none (or the
 * path does not fit). Replaces find_restart_checkpoint (src/io/checkpoint.cpp:362). */
int tpicb200_checkpoint_find(const char* directory, char* path, size_t size);

/* The header of a checkpoint piece (host only): the sizes a caller needs to
 * allocate the state it restores into. TPICB200_INVALID_DATA for a file that
 * is not a complete piece of this format. */
int tpicb200_checkpoint_info_read(const char* path, tpicb200_checkpoint_info* info);

/* Restores E, B (cells) and the particle records of a piece into the state's
 * live slots (counts set from the piece), after checking that the run is
 * the checkpoint's: grid, dt, c, species count, q/m and storage precision
 * (prepare_restart, src/io/checkpoint.cpp:388-470). The checksum is verified
 * before anything is written. Then call tpicb200_prepare. Host-blocking. */
int tpicb200_checkpoint_read(tpicb200_context* ctx, tpicb200_state* state, const char* path,
                             tpicb200_checkpoint_info* info, tpicb200_stream stream);

/* ------------------------------------------------------------------------
 * Snapshot output (TPIC's output channels, docs/user/output.md; the VTK
 * engine of src/io/vtk_field_engine.cpp and src/io/vtk_particle_engine.cpp).
 * ---------------------------------------------------------------------- */

/* Output moments of one species (diagnostics/output_moment_deposition_device.hpp:30-107),
 * FP64, ADDED into the caller's arrays at the nx*ny*nz unique nodes (x fastest, each
 * component a separate array of that size, components outer): rho = 4 pi sum(q W)/V
 * (the snapshot's rho), J = sum(q v W)/V (3 components) and the raw second moment
 * P_ij = sum((q/qom) v_i v_j W)/V (6 components: xx, xy, xz, yy, yz, zz). Any of the
 * three may be NULL. V is the cell volume, the dual volume of every node of a
 * periodic grid. Records with an invalid key, a fraction outside [0, 1) or a
 * nonfinite amount add nothing and raise the context's invalid counter. */
int tpicb200_output_moments(tpicb200_context* ctx, double qom, const tpicb200_particles* p, double* rho, double* j,
                            double* pressure, tpicb200_stream stream);

/* A species' records in output form on the device: position = (cell + fraction)
 * * spacing (3 per record, interleaved), velocity widened to FP64 (3 per record),
 * charge. A record with an invalid key, a fraction outside [0, 1) or a nonfinite
 * velocity or charge raises the context's invalid counter (TPIC refuses to
 * write such a snapshot). */
int tpicb200_output_particles(tpicb200_context* ctx, const tpicb200_particles* p, double* position, double* velocity,
                              double* charge, tpicb200_stream stream);

/* Writes one Float64 field array as VTK XML ImageData (host only): `values` holds
 * the (nx+1)(ny+1)(nz+1) nodes of the grid, end nodes included, x fastest, the
 * `components` values of a node interleaved. FieldData: TimeValue = time, cycle,
 * final_state and the strings state ("final" or "pre_solve"), precision_profile
 * and precision_roles. overwrite = 0 refuses an existing file
 * (TPICB200_BACKEND_FAILURE with the path in tpicb200_last_error()). The file name
 * is the caller's; TPIC names it <array>_tNNNNNN.vti. */
int tpicb200_vtk_write_field(const char* path, const char* name, int components, const tpicb200_grid* grid,
                             const double* values, int cycle, double time, int final_state, const char* profile,
                             const char* roles, int overwrite);

/* Writes one Float64 cell array (nx ny nz values, x fastest) as VTK XML
 * ImageData CellData over the same node extent and FieldData as
 * tpicb200_vtk_write_field (host only): TPIC's Gauss snapshot array. */
int tpicb200_vtk_write_cells(const char* path, const char* name, const tpicb200_grid* grid, const double* values,
                             int cycle, double time, int final_state, const char* profile, const char* roles,
                             int overwrite);

typedef struct {
  uint64_t count;
  const double* position;  /* 3 * count, global coordinates */
  const double* velocity;  /* 3 * count */
  const double* charge;    /* count */
  const uint64_t* id;      /* count */
  uint64_t species;        /* species index written for every record */
} tpicb200_vtk_species;

/* Writes a particle snapshot under `directory` (host only): the PolyData piece
 * particles_tNNNNNN_r000000.vtp (the species one after another: point data
 * velocity, charge, id, species; points = positions; one vertex per point) and
 * its PPolyData manifest particles_tNNNNNN.pvtp. */
int tpicb200_vtk_write_particles(const char* directory, int cycle, double time, int final_state, const char* profile,
                                 const char* roles, int ns, const tpicb200_vtk_species* species, int overwrite);

/* ------------------------------------------------------------------------
 * Gauss-law residual (TPIC's DiagnosticGaussCycle and FieldOutputTag Gauss;
 * diagnostics/gauss_residual_device.hpp, docs/developer/gauss_diagnostic.md).
 *
 * A sample begun at state n holds per cell s = divC(E^n)/2 - c, where divC is
 * the solver's node-to-cell divergence and c is 4 pi times the 8-node mean of
 * the charge density rho = sum(q W)/V of the state's records (the positions
 * x^{n+1/2}), smoothed like the solver's current when the context smooths;
 * finishing it at state n+1 gives r = s + divC(E^{n+1})/2, the residual at
 * time (n + 1/2) dt. Cell arrays (stash, first, residual) are caller-owned
 * FP64 device buffers of nx ny nz cells, x fastest; sums is a device double[4]
 * in gauss.csv's column order: sum of r^2, of (r - r_first)^2, of r^2 over
 * wall cells (0: a periodic grid has none), of c^2. The root mean squares are
 * sqrt(sum / (nx ny nz)). Stream-ordered; the sums of the same inputs are
 * reproducible (fixed-order reductions).
 * ------------------------------------------------------------------------ */

/* The field part of a sample (gauss_field_partials_kernel): with finish,
 * r = stash + divC(E)/2 into residual, sums[0..2], and first = r when
 * set_first (the run's first finished sample; its drift sum is 0); with
 * begin, stash = divC(E)/2, after the finish has read it (one call serves a
 * state that finishes a sample and begins the next). */
int tpicb200_gauss_field(tpicb200_context* ctx, const void* e, double* stash, double* first, double* residual,
                         int begin, int finish, int set_first, double* sums, tpicb200_stream stream);

/* The charge part of a begun sample (gauss_charge_partials_kernel): rho of
 * the ns species' records, the context's smoothing in FP64 arithmetic when it
 * has one, c per cell, stash -= c and sums[3] = sum of c^2. A record with an
 * invalid key, a fraction outside [0, 1) or a nonfinite charge raises the
 * context's invalid counter. */
int tpicb200_gauss_charge(tpicb200_context* ctx, int ns, const tpicb200_particles* species, double* stash,
                          double* sums, tpicb200_stream stream);

#ifdef __cplusplus
}
#endif

#endif /* TPICB200_H */
