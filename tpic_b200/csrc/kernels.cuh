// Host-side launch entry points of the kernel files (internal to the library).
#pragma once

#include "cases.cuh"
#include "common.cuh"

#include <string>

namespace tpicb200 {

// Host-side count of the kernels this library launched (tpicb200_launch_count).
void count_launches(unsigned n);
// The counter's value, and a correction for launches that were captured into
// a graph rather than run (the graph's runs are counted when they happen).
unsigned long long launches_so_far();
void uncount_launches(unsigned long long n);
// Records the message tpicb200_last_error() returns on this thread; returns status.
int report_error(int status, const std::string& message);

// abi.cu: the context's geometry, options and state checks, for the
// host-side entry points of other files.
const Geom& context_geom(const tpicb200_context* ctx);
const tpicb200_options& context_options(const tpicb200_context* ctx);
const tpicb200_grid& context_grid(const tpicb200_context* ctx);
int context_check_state(tpicb200_context* ctx, tpicb200_state* st);
uint32_t* context_invalid(tpicb200_context* ctx);

// mover.cu
struct BinnedScratch;
// Species scalars accumulated by the movers (kinetic energy, charge,
// momentum of the moved records): row r of the partial sums at
// partials + r * stride, `written` partials per row (set by launch_mover;
// at most kMoverPartials).
constexpr int kMoverPartials = 2 * 148 * 8;
struct SpeciesScalars {
  double* partials;
  long long stride;
  int* written;
};
// With `binned`, the mover also writes direction codes and transfer counts
// for binned_finish (after binned_begin with zeroed transfer counts).
// out (null: in place) receives the moved records, read through ranks when
// given (position p of out <- record ranks[p] of p). With `scalars`, the
// species scalars of the moved records.
cudaError_t launch_mover(int precision, const Geom& g, double qom, double dt, double c,
                         tpicb200_particles* p, tpicb200_particles* out, const uint32_t* ranks,
                         const double* theta, const void* bnode, uint32_t* invalid, const BinnedScratch* binned,
                         const SpeciesScalars* scalars, cudaStream_t s);

// sort.cu: scratch needs `bins` cursor words, `capacity` permutation words and
// the scan workspace returned by sort_scan_words().
size_t sort_scan_words(long long bins);
cudaError_t launch_sort(int precision, const Geom& g, const tpicb200_particles* in,
                        tpicb200_particles* out, uint32_t* counts, uint32_t* offsets,
                        uint32_t* cursor, uint32_t* perm, uint32_t* scan_scratch,
                        uint32_t* invalid, cudaStream_t s);
// Sort of records grouped by the bins (in_counts, in_offsets) of an earlier
// sort, keys updated since: neighbour moves go through the transfer-count
// path, anything else through the general sort (same stable order).
struct BinnedState {
  uint32_t fallback;         // nonzero: the general sort produces the output
  uint32_t bins_bad;         // nonzero: the old bins do not tile the records
  unsigned long long total;  // records in the old bins
};
struct BinnedScratch {
  BinnedState* state;
  uint32_t* old_counts;   // copy of the input's bins
  uint32_t* old_offsets;
  uint32_t* transfer;     // [27][interior cells]: counts, then output bases
  uint16_t* code;         // run code per record (direction, cell in run; kNoMove)
};
size_t binned_scratch_words(const Geom& g);
bool binned_sort_applies(const Geom& g);
BinnedScratch binned_scratch(const Geom& g, uint32_t* words, uint16_t* codes);
// Copies the input's bins and clears the state (and the transfer counts when
// the mover will add into them).
cudaError_t binned_begin(const Geom& g, const BinnedScratch& b, const uint32_t* in_counts,
                         const uint32_t* in_offsets, bool zero_transfer, cudaStream_t s);
// Checks that the old bins tile the n records in key order (else raises
// bins_bad and fallback).
cudaError_t binned_validate(const Geom& g, const BinnedScratch& b, uint32_t n, cudaStream_t s);
// (Classification when `classify`), counts, scan, bases, the ranks (perm:
// sorted position -> input record), the gather of the sorted records when
// `materialize`, and the gated general sort (which always writes `out` and
// the same perm); binned_validate must have run.
cudaError_t binned_finish(int precision, const Geom& g, const BinnedScratch& b, bool classify, bool materialize,
                          const tpicb200_particles* in, tpicb200_particles* out, uint32_t* counts,
                          uint32_t* offsets, uint32_t* cursor, uint32_t* perm, uint32_t* scan_scratch,
                          uint32_t* invalid, cudaStream_t s);
cudaError_t launch_sort_binned(int precision, const Geom& g, const tpicb200_particles* in,
                               const uint32_t* in_counts, const uint32_t* in_offsets, tpicb200_particles* out,
                               uint32_t* counts, uint32_t* offsets, uint32_t* cursor, uint32_t* perm,
                               uint32_t* scan_scratch, uint32_t* binned_words, uint16_t* codes,
                               uint32_t* invalid, cudaStream_t s);

// Context-free sort on the file-scope scratch array (no allocation): the
// first call on a device resolves the array's address (sort_static_setup).
long long sort_static_scratch_bytes();
cudaError_t sort_static_setup(uint32_t** scratch);
cudaError_t launch_sort_static(int precision, const Geom& g, const tpicb200_particles* in, tpicb200_particles* out,
                               uint32_t* counts, uint32_t* offsets, uint32_t* invalid, uint32_t* scratch,
                               cudaStream_t s);

// Records read through perm (sorted position -> record of the read slot;
// null: read in place, in sorted order). With out.rx set, each record is
// also written at its sorted position into `out` (the sort's gather fused
// into the deposition).
struct SortedCopy {
  const uint32_t* perm;
  tpicb200_particles out;
};
// Writes out.id[p] = in.id[perm[p]] for the records a fused deposition
// copied (the deposition kernels copy every other attribute).
cudaError_t launch_copy_ids(const tpicb200_particles* in, const SortedCopy* copy, cudaStream_t s);

// Sorted records: out[p] = in[perm[p]] for every attribute (ids included).
cudaError_t launch_sorted_gather(int precision, const uint32_t* perm, const tpicb200_particles* in,
                                 tpicb200_particles* out, cudaStream_t s);

// deposit.cu
cudaError_t launch_deposit(int precision, int mass_kind, const Geom& g, double qom, double dt,
                           double c, const tpicb200_particles* p, const uint32_t* counts,
                           const uint32_t* offsets, const void* bnode, void* j, void* mass,
                           uint32_t* invalid, const SortedCopy* copy, cudaStream_t s);
cudaError_t launch_fold(int precision, const Geom& g, void* j, void* mass, cudaStream_t s);

// mass_tc.cu (tcgen05 forms): per-cell moments, then their assembly into J
// and the mass coefficients.
size_t moment_floats(const Geom& g);
// Tensor-core deposition of `ns` species (fused two per launch) into the
// per-cell moments; `accumulate` adds to moments already present.
// wait_polls bounds the BF16X3 stream kernel's chunk-loop waits (0: the
// default kDefaultWaitPolls); a wait that gives up sets bit 20 of *invalid.
// stall_chunk >= 1 makes the wait for the MMAs of chunk stall_chunk - 1 wait
// on an mbarrier that nothing arrives on instead (a test of the bound).
constexpr uint32_t kDefaultWaitPolls = 1u << 22;
cudaError_t launch_deposit_tc(int mass_kind, const Geom& g, int ns, const double* qom, double dt, double c,
                              const tpicb200_particles* const* p, const uint32_t* const* counts,
                              const uint32_t* const* offsets, const void* bnode, float* moments, int accumulate,
                              uint32_t* invalid, const SortedCopy* const* copies, cudaStream_t s,
                              uint32_t wait_polls = 0, uint32_t stall_chunk = 0);
// FP64 CUDA-core form of the same moments (double precision; double moments).
cudaError_t launch_deposit_moments_f64(const Geom& g, int ns, const double* qom, double dt, double c,
                                       const tpicb200_particles* const* p, const uint32_t* const* counts,
                                       const uint32_t* const* offsets, const void* bnode, double* moments,
                                       int accumulate, uint32_t* invalid, const SortedCopy* const* copies,
                                       cudaStream_t s);
// Moments (float or double, as the precision mode) into J and the mass records.
cudaError_t launch_assemble_moments(int precision, const Geom& g, const void* moments, void* j, void* mass,
                                    int overwrite, cudaStream_t s);

// fields.cu
cudaError_t launch_node_ghosts(const Geom& g, double* f, int components, cudaStream_t s,
                               bool programmatic = false);
// The output moments of one species (output.cu): rho scaled by rho_scale and,
// where their buffers are given, J and the raw second moments, FP64 atomics
// at the unique nodes.
cudaError_t launch_output_moments(int precision, const Geom& g, const tpicb200_particles& p, double qom,
                                  double rho_scale, double* rho, double* j, double* pressure, uint32_t* invalid,
                                  cudaStream_t s);
cudaError_t launch_smooth(bool double_arithmetic, const Geom& g, int niter, int op, double alpha,
                          const double* src, double* out, double* tmp, uint32_t* invalid, cudaStream_t s);
cudaError_t launch_widen(int precision, const Geom& g, const void* in, double* out, cudaStream_t s);
cudaError_t launch_cell_ghosts(int precision, const Geom& g, void* f, cudaStream_t s);
cudaError_t launch_cell_to_node(int precision, const Geom& g, const void* cellf, void* node,
                                cudaStream_t s);
cudaError_t launch_rhs(int precision, const Geom& g, double delta, double kfac, const void* e,
                       const void* bcell, const void* j, double* rhs, cudaStream_t s, bool j_double = false);
cudaError_t launch_field_advance(int precision, const Geom& g, double theta_value, double faraday,
                                 void* e, const void* bcell, const double* etheta, void* bnext,
                                 uint32_t* invalid, cudaStream_t s);
cudaError_t launch_field_energy(int precision, const Geom& g, const void* e, const void* bcell,
                                double* partials, int blocks, cudaStream_t s);
cudaError_t launch_species_scalars(int precision, const tpicb200_particles* p, double qom,
                                   double* partials, int blocks, cudaStream_t s);
// `programmatic`: launched with programmatic stream serialization (the
// kernels wait for their predecessor before reading).
cudaError_t launch_reduce_rows(const double* partials, double* out, int rows, int row_stride,
                               int count, int filled, cudaStream_t s, bool programmatic = false);
cudaError_t launch_copy_node_field(const Geom& g, const void* in, int in_double, double* out,
                                   cudaStream_t s);

// adjoint.cu: the transposes of the cycle's stages (FP64 adjoint arithmetic;
// particle adjoints indexed by record id, [3][nid] and [nid]).
enum { kAdjointMover = 0, kAdjointDeposit = 1, kAdjointCycle = 2 };
// Adds the mover's E_theta gradient of every record into the unique nodes of
// etheta_bar (x_bar, v_bar: the gradients of the moved records).
cudaError_t launch_adjoint_theta_scatter(int precision, const Geom& g, double qom, double dt, double c,
                                         const tpicb200_particles* p, uint32_t nid, const double* xbar,
                                         const double* vbar, const void* bnode, double* etheta_bar,
                                         uint32_t* invalid, cudaStream_t s);
// Record adjoint: kAdjointMover (the mover's backward, both scatters),
// kAdjointDeposit (current and mass backward: jscale*jbar the J gradient,
// mscale*<mleft, M mright> the mass term) or kAdjointCycle (both, the
// E_theta scatter done before by launch_adjoint_theta_scatter). The B
// gradient goes into the unique nodes of bnode_bar.
cudaError_t launch_adjoint_records(int precision, int mode, const Geom& g, double qom, double dt, double c,
                                   const tpicb200_particles* p, uint32_t nid, double* xbar, double* vbar,
                                   double* qbar, const double* theta, const void* bnode, const double* jbar,
                                   double jscale, const double* mleft, const double* mright, double mscale,
                                   double* bnode_bar, double* etheta_bar, uint32_t* invalid, cudaStream_t s);
// ebar (in place: the gradient of E' becomes that of E) and etheta_bar (out)
// of the field advance; bbar (the gradient of B', equal to that of B) is read.
cudaError_t launch_adjoint_advance(const Geom& g, double theta, double c, double dt, double* ebar, const double* bbar,
                                   double* etheta_bar, cudaStream_t s);
cudaError_t launch_adjoint_add_nodes(const Geom& g, const double* lambda, double* ebar, cudaStream_t s);
cudaError_t launch_adjoint_cells(const Geom& g, double delta, const double* lambda, const double* bnode_bar,
                                 double* bbar, cudaStream_t s);
cudaError_t launch_energy_gradient(int precision, const Geom& g, double we, double wb, const void* e,
                                   const void* bcell, double* ebar, double* bbar, cudaStream_t s);

// solver.cu
struct SolverWorkspace;
// Energy-conserving smoothing of the field solve: passes (0: off), Face7
// centre weight, operator (0 Face7, 1 Binomial27).
struct SmoothingPlan {
  int iterations = 0;
  double alpha = 1.0;
  int op = 0;
};
SolverWorkspace* solver_create(int precision, const Geom& g, int restart, double dt,
                               double theta, double c, const SmoothingPlan& smoothing, cudaError_t* err);
// S^n of a double node field (ghosts filled) into out, in the field
// arithmetic of the precision mode, with the solver's scratch.
cudaError_t solver_smooth(SolverWorkspace* w, const double* in, double* out, cudaStream_t s);
void solver_destroy(SolverWorkspace* w);
// The adjoint solve A^T lambda = rhs (rhs a double node field with its
// duplicates and ghosts filled) from a zero guess, by the same restarted
// GMRES; lambda receives the solution with its ghosts. TPICB200_INVALID_STATE
// with smoothing.
int solver_solve_adjoint(SolverWorkspace* w, const double* rhs, const void* mass, double* lambda,
                         tpicb200_gmres_result* result, int max_iterations, double tol, cudaStream_t s,
                         cudaError_t* err);
// The counter the solver's smoothing passes raise on a nonfinite value.
void solver_set_invalid(SolverWorkspace* w, uint32_t* invalid);
// Bound of the TMA apply's copy waits (0: kDefaultWaitPolls); stall_stencil
// in 0..13 makes the wait for that stencil's box wait on an mbarrier that
// nothing arrives on (a test of the bound), -1 none.
void solver_set_waits(SolverWorkspace* w, uint32_t polls, int stall_stencil);
int solver_solve(SolverWorkspace* w, const void* e, const void* bcell, const void* j,
                 const void* mass, double* etheta, tpicb200_gmres_result* result,
                 int max_iterations, double tol, cudaStream_t s, cudaError_t* err);
cudaError_t solver_mass_apply(SolverWorkspace* w, const void* mass, const double* in, double* out,
                              cudaStream_t s);

// cases.cu: the loading profile of species s of an admitted deck.
int case_profile_of(const tpicb200_deck* deck, int s, CaseProfile* out);

// load.cu
struct LoadPlan {
  uint64_t first;          // load index of the first record
  uint32_t ppc;            // particles per cell
  int npc[3];              // npcel per axis
  double inverse_npc[3];   // 1.0 / npcel
  double q_factor;         // sign(qom) * volume / ppc
  double vth[3];
  uint32_t key0, key1;     // Philox key (seed)
  uint32_t species;        // Philox counter word 2
  int quiet;               // subcell centres
};
cudaError_t launch_load_species(int precision, const Geom& g, const LoadPlan& plan, const CaseProfile& prof,
                                tpicb200_particles* p, uint32_t* invalid, cudaStream_t s);
// partials: 4 rows of `blocks` doubles; sums: 4 doubles.
cudaError_t launch_center_velocities(int precision, const Geom& g, const CaseProfile& prof, tpicb200_particles* p,
                                     double* partials, int blocks, double* sums, uint32_t* invalid,
                                     cudaStream_t s);

}  // namespace tpicb200
