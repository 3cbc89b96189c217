// Implicit theta-scheme particle mover.
//
// Restates push_and_classify_particle (ecsim/particles/particle_mover_device.hpp:37-122)
// with the whole-domain periodic wrap of classify_particle_point
// (communication/particles/particle_boundaries.hpp:112-135). This file is
// compiled with -fmad=false: every multiply and add rounds on its own, as the
// reference's expressions evaluate under strict IEEE rules, so new fractions,
// velocities and cell keys are bit-identical to the CPU oracle.
//
// Two kernels share one push. Each moves record n of the read slot into
// position p of the written slot: in place (n = p), or, for a ranked
// species, n = ranks[p] of the previous sort into the other slot, which then
// holds the moved records in the previous sorted order.
//  - mover_kernel, one thread per record, gathers the 48 field values of a
//    record from global memory (they hit L1/L2 because records are sorted);
//  - run_mover_kernel, for records grouped by the bins of the previous sort
//    (the cycle's path): a warp takes a run of up to 32 consecutive cells of
//    one x-row, stages the B and E_theta nodes of the run (33 x 2 x 2 nodes,
//    converted once to the compute type) in shared memory and streams the
//    run's records, gathering from shared memory. A record whose key is not
//    its bin's cell gathers from global memory instead. Both forms evaluate
//    the same products in the same order, so the results are identical.
// Ahead of the binned sort both also emit each record's direction code and
// the per-cell transfer counts (the sort then needs no classification pass).
//
// HBM-bound: per record the push reads key (4 B), charge (8 B), three double
// fractions (24 B) and three velocities, and writes the fractions, the
// velocities and the key.
#include "kernels.cuh"

#include <climits>
#include <type_traits>

namespace tpicb200 {
namespace {

template <class P>
struct MoverParams {
  typename P::VC beta, beta_over_c;
  double dt, inv[3];
  double inverse_qom;
};

// Species scalars of the moved records (the sums of species_kernel:
// kinetic energy, charge, momentum), accumulated by the movers: each block
// writes its five partial sums at partials[r * stride + offset + block].
struct MoverScalars {
  double* partials;  // null: not accumulated
  long long stride;
  int offset;
};

// Per-thread sums of the five scalars: in registers (RegisterSums) or, where
// registers are short, in the thread's column of a shared-memory array
// (SharedSums: entry r at sums[r * 32]).
struct RegisterSums {
  double (&acc)[5];
  __device__ __forceinline__ void add(int r, double v) const { acc[r] += v; }
};
struct SharedSums {
  double* sums;
  __device__ __forceinline__ void add(int r, double v) const { sums[r * 32] += v; }
};
template <class Sums>
__device__ __forceinline__ void add_scalars(const Sums& acc, double charge, double inverse_qom, double vx, double vy,
                                            double vz) {
  const double mass = charge * inverse_qom;
  acc.add(0, 0.5 * mass * (vx * vx + vy * vy + vz * vz));
  acc.add(1, charge);
  acc.add(2, mass * vx);
  acc.add(3, mass * vy);
  acc.add(4, mass * vz);
}

// Block sums of the five scalars into the block's partials (every thread of
// the block calls it; scratch holds Threads / 32 doubles).
template <int Threads>
__device__ __forceinline__ void store_scalars(const MoverScalars& sc, const double (&acc)[5], double* scratch) {
#pragma unroll
  for (int r = 0; r < 5; ++r) {
    const double total = block_sum<Threads>(acc[r], scratch);
    if (threadIdx.x == 0) sc.partials[r * sc.stride + sc.offset + blockIdx.x] = total;
  }
}

// Direction codes and transfer counts of a mover that feeds the binned sort.
struct MoveCodes {
  uint16_t* code;       // per record: run code (direction, cell in run), kNoMove when not a neighbour move
  uint32_t* transfer;   // [27][interior cells], added into
  uint32_t* fallback;   // raised when any record did not move to a neighbour
  const uint32_t* bins_bad;  // the old bins do not tile the records
  long long cells;
};

template <class P>
struct Records {
  typename P::Pos* __restrict__ rx;
  typename P::Pos* __restrict__ ry;
  typename P::Pos* __restrict__ rz;
  typename P::Vel* __restrict__ u;
  typename P::Vel* __restrict__ v;
  typename P::Vel* __restrict__ w;
  double* __restrict__ q;
  int32_t* __restrict__ key;
  uint64_t* __restrict__ id;
};

// Where the movers read and write: record n of `in` (n = ranks[p] when
// ranks are given, else p) is moved into position p of `out`; with out ==
// in and no ranks the move is in place.
template <class P>
struct MoveIo {
  Records<P> in, out;
  const uint32_t* __restrict__ ranks;
  bool copy;  // out is another slot: every attribute is written
};

// A record that is not moved (invalid) is copied unchanged by a copying mover.
template <class P>
__device__ __forceinline__ void copy_record(const MoveIo<P>& io, uint32_t n, uint32_t p) {
  if (!io.copy) return;
  io.out.rx[p] = io.in.rx[n]; io.out.ry[p] = io.in.ry[n]; io.out.rz[p] = io.in.rz[n];
  io.out.u[p] = io.in.u[n]; io.out.v[p] = io.in.v[n]; io.out.w[p] = io.in.w[n];
  io.out.q[p] = io.in.q[n]; io.out.key[p] = io.in.key[n];
  if (io.out.id) io.out.id[p] = io.in.id[n];
}

// Corner values from global memory: node box of cell (ci, cj, ck).
template <class P>
struct GlobalFields {
  const double* __restrict__ theta;
  const typename P::Fld* __restrict__ bnode;
  long long nn, base;
  int off[8];
  // which 0: B, 1: E_theta; component c; corner a.
  __device__ __forceinline__ typename P::VC operator()(int which, int c, int a) const {
    using C = typename P::VC;
    return which ? C(__ldg(theta + c * nn + base + off[a])) : C(__ldg(bnode + c * nn + base + off[a]));
  }
};

// Corner values staged in shared memory for a run: [which][c][z][y][x].
constexpr int kRunNodes = kRunCells + 1;
template <class C>
struct SharedFields {
  const C* s;  // 2 x 3 x 2 x 2 x kRunNodes values
  int x;       // cell offset in the run
  __device__ __forceinline__ C operator()(int which, int c, int a) const {
    return s[(((which * 3 + c) * 2 + ((a >> 2) & 1)) * 2 + ((a >> 1) & 1)) * kRunNodes + x + (a & 1)];
  }
};

// FP32 corner values staged in shared memory as component pairs for a run:
// pair 0 = (Bx, By), 1 = (Bz, Ex), 2 = (Ey, Ez), layout [pair][z][y][x].
struct SharedPairFields {
  const float2* s;  // 3 x 2 x 2 x kRunNodes pairs
  int x;            // cell offset in the run
  __device__ __forceinline__ float2 operator()(int pair, int a) const {
    return s[((pair * 2 + ((a >> 2) & 1)) * 2 + ((a >> 1) & 1)) * kRunNodes + x + (a & 1)];
  }
};

template <class C, class F>
__device__ __forceinline__ C gather8(const F& field, int which, int c, const C w[8]) {
  C value = 0;
#pragma unroll
  for (int a = 0; a < 8; ++a) value += w[a] * field(which, c, a);
  return value;
}

// B and E_theta at the record: sum over corners a = 0..7 of w[a] * corner
// value, each product and sum rounded on its own.
template <class C, class F>
__device__ __forceinline__ void gather_fields(const F& field, const C w[8], C (&b)[3], C (&e)[3]) {
#pragma unroll
  for (int c = 0; c < 3; ++c) b[c] = gather8<C>(field, 0, c, w);
#pragma unroll
  for (int c = 0; c < 3; ++c) e[c] = gather8<C>(field, 1, c, w);
}
// The same sums, two components per packed FP32 multiply and add (each
// element rounded on its own, so the results equal the scalar sums).
__device__ __forceinline__ void gather_fields(const SharedPairFields& field, const float w[8], float (&b)[3],
                                              float (&e)[3]) {
  float2 sum[3] = {make_float2(0.0f, 0.0f), make_float2(0.0f, 0.0f), make_float2(0.0f, 0.0f)};
#pragma unroll
  for (int a = 0; a < 8; ++a) {
    const float2 weight = make_float2(w[a], w[a]);
#pragma unroll
    for (int p = 0; p < 3; ++p) sum[p] = __fadd2_rn(sum[p], __fmul2_rn(weight, field(p, a)));
  }
  b[0] = sum[0].x; b[1] = sum[0].y; b[2] = sum[1].x;
  e[0] = sum[1].y; e[1] = sum[2].x; e[2] = sum[2].y;
}

// The push of record n, whose valid interior cell (ci, cj, ck) was decoded
// from its key. Returns the direction code of the move (-1: invalid, or a
// move beyond the 27 neighbouring cells when Coded).
template <class P, bool Coded, class F, class Sums>
__device__ __forceinline__ int push(const Geom& g, const MoverParams<P>& mp, const MoveIo<P>& io, uint32_t n,
                                    uint32_t p, int ci, int cj, int ck, typename P::Pos fx, typename P::Pos fy,
                                    typename P::Pos fz, double charge, const F& field, uint32_t* invalid,
                                    const Sums* acc) {
  const Records<P>& r = io.in;
  using C = typename P::VC;
  using Pos = typename P::Pos;
  using Vel = typename P::Vel;
  C wt[8];
  cic_weights<C>(C(fx), C(fy), C(fz), wt);
  C bf[3], ef[3];
  gather_fields(field, wt, bf, ef);
  const C bx = bf[0], by = bf[1], bz = bf[2];
  const C ex = ef[0], ey = ef[1], ez = ef[2];
  const Response<C> rs(bx, by, bz, mp.beta_over_c);
  const C uu = C(r.u[n]), vv = C(r.v[n]), ww = C(r.w[n]);
  C hx, hy, hz, ax, ay, az;
  rs.apply(uu, vv, ww, hx, hy, hz);
  rs.apply(ex, ey, ez, ax, ay, az);
  const C px = hx + mp.beta * ax, py = hy + mp.beta * ay, pz = hz + mp.beta * az;
  const Vel vel[3] = {Vel(C(2) * px - uu), Vel(C(2) * py - vv), Vel(C(2) * pz - ww)};
  long long cell[3] = {ci, cj, ck};
  Pos frac[3] = {fx, fy, fz};
  const int ext[3] = {g.nx, g.ny, g.nz};
  bool ok = true;
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
    copy_record(io, n, p);
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
  if (acc) add_scalars(*acc, charge, mp.inverse_qom, double(vel[0]), double(vel[1]), double(vel[2]));
  const Records<P>& o = io.out;
  o.key[p] = g.encode(int(cell[0]), int(cell[1]), int(cell[2]));
  o.rx[p] = frac[0]; o.ry[p] = frac[1]; o.rz[p] = frac[2];
  o.u[p] = vel[0]; o.v[p] = vel[1]; o.w[p] = vel[2];
  if (io.copy) {
    o.q[p] = charge;
    if (o.id) o.id[p] = r.id[n];
  }
  return Coded ? move_code(g, ci, cj, ck, int(cell[0]), int(cell[1]), int(cell[2])) : 0;
}

// Record checks before the push: a valid interior key, a finite charge and
// fractions in [0, 1). record_ok writes the decoded cell; fields_ok checks
// a record whose key is already known to be a given interior cell's.
template <class P>
__device__ __forceinline__ bool fields_ok(double charge, typename P::Pos fx, typename P::Pos fy, typename P::Pos fz) {
  using Pos = typename P::Pos;
  return isfinite(charge) && fx >= Pos(0) && fx < Pos(1) && fy >= Pos(0) && fy < Pos(1) && fz >= Pos(0) &&
         fz < Pos(1);
}
template <class P>
__device__ __forceinline__ bool record_ok(const Geom& g, int32_t k0, double charge, typename P::Pos fx,
                                          typename P::Pos fy, typename P::Pos fz, int& ci, int& cj, int& ck) {
  if (!(k0 >= 0 && (long long)k0 < g.bins)) return false;
  g.decode(k0, ci, cj, ck);
  return g.interior_cell(ci, cj, ck) && fields_ok<P>(charge, fx, fy, fz);
}

template <class P>
__device__ __forceinline__ GlobalFields<P> global_fields(const Geom& g, const double* theta,
                                                         const typename P::Fld* bnode, int ci, int cj, int ck) {
  // Corner offsets of the node box (an x-y plane of nodes is far below 2^31).
  const int plane = g.NX * g.NY;
  return GlobalFields<P>{theta, bnode, g.nodes, g.node(ci, cj, ck),
                         {0, 1, g.NX, g.NX + 1, plane, plane + 1, plane + g.NX, plane + g.NX + 1}};
}

// Run codes and transfer counts of one warp-wide step (every lane of the warp
// calls it): one atomic per run of consecutive lanes with the same
// (old cell, direction); records are sorted by old cell, so a warp holds few.
__device__ __forceinline__ void record_codes(const MoveCodes& mc, bool live, uint32_t n, int d, int run_cell,
                                             long long old_cell) {
  const int lane = threadIdx.x & 31;
  if (live) mc.code[n] = d < 0 ? kNoMove : uint16_t(d | (run_cell << 5));
  const long long slot = d < 0 ? -1 : old_cell * 27 + d;
  const long long left = __shfl_up_sync(0xffffffffu, slot, 1);
  const unsigned heads = __ballot_sync(0xffffffffu, lane == 0 || slot != left);
  if (d >= 0 && ((heads >> lane) & 1u)) {
    const unsigned later = heads & ~((2u << lane) - 1u);
    const int next = later ? __ffs(later) - 1 : 32;
    atomicAdd(mc.transfer + d * mc.cells + old_cell, unsigned(next - lane));
  }
  if (__any_sync(0xffffffffu, live && d < 0) && lane == 0) atomicExch(mc.fallback, 1u);
}

// Resident CTAs per SM the movers are compiled for (register budget).
#ifndef TPICB200_MOVER_MIN_BLOCKS
#define TPICB200_MOVER_MIN_BLOCKS 4
#endif

// One thread per record. With a gate, the kernel runs only when *gate != 0.
template <class P>
__global__ void __launch_bounds__(256, TPICB200_MOVER_MIN_BLOCKS) mover_kernel(Geom g, MoverParams<P> mp,
    MoveIo<P> io, uint32_t count, const double* __restrict__ theta, const typename P::Fld* __restrict__ bnode,
    uint32_t* __restrict__ invalid, const uint32_t* gate, MoverScalars sc) {
  using Pos = typename P::Pos;
  __shared__ double scratch[8];
  double acc[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
  if (gate && *gate == 0) {
    if (sc.partials && threadIdx.x < 5) sc.partials[threadIdx.x * sc.stride + sc.offset + blockIdx.x] = 0.0;
    return;
  }
  const Records<P>& r = io.in;
  for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < count; p += gridDim.x * blockDim.x) {
    const uint32_t n = io.ranks ? io.ranks[p] : p;
    const int32_t k0 = r.key[n];
    const double charge = r.q[n];
    const Pos fx = r.rx[n], fy = r.ry[n], fz = r.rz[n];
    int ci, cj, ck;
    if (record_ok<P>(g, k0, charge, fx, fy, fz, ci, cj, ck)) {
      const RegisterSums sums{acc};
      push<P, false>(g, mp, io, n, p, ci, cj, ck, fx, fy, fz, charge, global_fields<P>(g, theta, bnode, ci, cj, ck),
                     invalid, sc.partials ? &sums : nullptr);
    } else {
      atomicAdd(invalid, 1u);
      copy_record(io, n, p);
    }
  }
  if (sc.partials) store_scalars<256>(sc, acc, scratch);
}

// Runs of up to g.run_len cells of one x-row; records grouped by the bins
// (old_counts, old_offsets), which validate_bins has checked (the kernel
// returns at once when they do not tile the records).
constexpr int kRunWarps = 4;
// Resident blocks of the run mover: eight (64 registers) in the mixed form,
// six (80 registers, no spills) in FP64, which spills at 64. The grid is one
// wave of them. FP64 move stage of the 128^3-cell, 268M-record workload with
// one-wave grids: 11.3 ms at four blocks, 11.3 at five, 10.3 at six, 11.5 at
// seven (16.5 ms at eight blocks with the spills); mixed: 7.53 ms at eight,
// 7.85 at seven, 8.14 at six.
template <class P>
constexpr int run_mover_blocks() {
  return std::is_same_v<P, PDouble> ? 6 : 2 * TPICB200_MOVER_MIN_BLOCKS;
}

template <class P>
__global__ void __launch_bounds__(kRunWarps * 32, run_mover_blocks<P>()) run_mover_kernel(Geom g,
    MoverParams<P> mp, MoveIo<P> io, uint32_t count, const double* __restrict__ theta,
    const typename P::Fld* __restrict__ bnode, const uint32_t* __restrict__ old_counts,
    const uint32_t* __restrict__ old_offsets, uint32_t* __restrict__ invalid, MoveCodes mc, MoverScalars sc) {
  using C = typename P::VC;
  using Pos = typename P::Pos;
  constexpr int kStaged = 2 * 3 * 2 * 2 * kRunNodes;
  __shared__ __align__(8) C fields[kRunWarps][kStaged];
  __shared__ uint32_t starts[kRunWarps][kRunCells];
  __shared__ double scratch[kRunWarps];
  __shared__ double lane_sums[kRunWarps][5][32];
  if (*mc.bins_bad) {
    if (sc.partials && threadIdx.x < 5) sc.partials[threadIdx.x * sc.stride + sc.offset + blockIdx.x] = 0.0;
    return;
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const long long runs = run_count(g);
  const SharedSums sums{&lane_sums[warp][0][lane]};
#pragma unroll
  for (int r = 0; r < 5; ++r) lane_sums[warp][r][lane] = 0.0;
  const SharedSums* acc = sc.partials ? &sums : nullptr;
  C* sf = fields[warp];
  uint32_t* st = starts[warp];
  for (long long run = (long long)blockIdx.x * kRunWarps + warp; run < runs; run += (long long)gridDim.x * kRunWarps) {
    int i0, len, j, k;
    run_cells(g, run, i0, len, j, k);
    // Cells of the run and their record ranges.
    uint32_t off = 0xffffffffu, stop = 0;
    if (lane < len) {
      const int32_t key = g.encode(i0 + lane, j, k);
      off = old_offsets[key];
      stop = off + old_counts[key];
    }
    st[lane] = off;
    const uint32_t begin = __shfl_sync(0xffffffffu, off, 0);
    const uint32_t end = min(__shfl_sync(0xffffffffu, stop, len - 1), count);
    // Stage the run's nodes: x in [i0, i0 + len], y in {j, j+1}, z in {k, k+1};
    // in FP32 as component pairs (SharedPairFields).
    const int nodes_x = len + 1;
    if constexpr (std::is_same_v<C, float>) {
      float2* sp = reinterpret_cast<float2*>(sf);
      for (int t = lane; t < 12 * nodes_x; t += 32) {
        const int x = t % nodes_x, rest = t / nodes_x;  // rest = (pair*2 + z)*2 + y
        const int y = rest & 1, z = (rest >> 1) & 1, pair = rest >> 2;
        const long long at = g.node(i0 + x, j + y, k + z);
        // Component q = 2 pair + h of (Bx, By, Bz, Ex, Ey, Ez).
        float v[2];
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const int q = 2 * pair + h;
          v[h] = q < 3 ? float(__ldg(bnode + q * g.nodes + at)) : float(__ldg(theta + (q - 3) * g.nodes + at));
        }
        sp[rest * kRunNodes + x] = make_float2(v[0], v[1]);
      }
    } else {
      for (int t = lane; t < 24 * nodes_x; t += 32) {
        const int x = t % nodes_x, rest = t / nodes_x;  // rest = ((which*3 + c)*2 + z)*2 + y
        const int y = rest & 1, z = (rest >> 1) & 1, c = (rest >> 2) % 3, which = (rest >> 2) / 3;
        const long long at = c * g.nodes + g.node(i0 + x, j + y, k + z);
        sf[rest * kRunNodes + x] = which ? C(__ldg(theta + at)) : C(__ldg(bnode + at));
      }
    }
    __syncwarp();
    const Records<P>& r = io.in;
    // The ranks of the next chunk are loaded one chunk ahead, so the record
    // loads do not wait for a rank load.
    uint32_t n_next = 0;
    if (io.ranks && begin + lane < end) n_next = io.ranks[begin + lane];
    for (uint32_t p0 = begin; p0 < end; p0 += 32) {
      const uint32_t p = p0 + lane;  // position in the sorted order of the bins
      const bool live = p < end;
      const uint32_t n_rank = n_next;
      if (io.ranks && p + 32 < end) n_next = io.ranks[p + 32];
      long long old_cell = 0;
      int d = -1, c = 0;
      if (live) {
        const uint32_t n = io.ranks ? n_rank : p;
        const int32_t k0 = r.key[n];
        const double charge = r.q[n];
        const Pos fx = r.rx[n], fy = r.ry[n], fz = r.rz[n];
#pragma unroll
        for (int step = 16; step > 0; step >>= 1)
          if (st[c + step] <= p) c += step;
        int ci = i0 + c, cj = j, ck = k;
        // A record in its bin's cell needs no key decode.
        const bool home = k0 == g.encode(ci, cj, ck);
        if (home ? fields_ok<P>(charge, fx, fy, fz) : record_ok<P>(g, k0, charge, fx, fy, fz, ci, cj, ck)) {
          if (home) {
            if constexpr (std::is_same_v<C, float>)
              d = push<P, true>(g, mp, io, n, p, ci, cj, ck, fx, fy, fz, charge,
                                SharedPairFields{reinterpret_cast<const float2*>(sf), c}, invalid, acc);
            else
              d = push<P, true>(g, mp, io, n, p, ci, cj, ck, fx, fy, fz, charge, SharedFields<C>{sf, c}, invalid,
                                acc);
          }
          else
            d = push<P, true>(g, mp, io, n, p, ci, cj, ck, fx, fy, fz, charge,
                              global_fields<P>(g, theta, bnode, ci, cj, ck), invalid, acc);
          old_cell = ci + (long long)g.nx * (cj + (long long)g.ny * ck);
        } else {
          atomicAdd(invalid, 1u);
          copy_record(io, n, p);
        }
      }
      record_codes(mc, live, p, d, c, old_cell);
    }
    __syncwarp();
  }
  if (sc.partials) {
    double own[5];
#pragma unroll
    for (int r = 0; r < 5; ++r) own[r] = lane_sums[warp][r][lane];
    store_scalars<kRunWarps * 32>(sc, own, scratch);
  }
}

template <class P>
MoverParams<P> mover_params(const Geom& g, double qom, double dt, double c) {
  MoverParams<P> mp;
  const double beta = qom * dt / 2;  // prepare_particle_mover_parameters: double, converted once
  mp.beta = typename P::VC(beta);
  mp.beta_over_c = typename P::VC(beta / c);
  mp.dt = dt;
  for (int a = 0; a < 3; ++a) mp.inv[a] = 1.0 / (a == 0 ? g.dx : a == 1 ? g.dy : g.dz);
  mp.inverse_qom = 1.0 / qom;
  return mp;
}

template <class P>
Records<P> records(const tpicb200_particles* p) {
  return Records<P>{(typename P::Pos*)p->rx, (typename P::Pos*)p->ry, (typename P::Pos*)p->rz,
                    (typename P::Vel*)p->u, (typename P::Vel*)p->v, (typename P::Vel*)p->w, p->q, p->cell, p->id};
}

template <class P>
cudaError_t launch(const Geom& g, double qom, double dt, double c, tpicb200_particles* p, tpicb200_particles* out,
                   const uint32_t* ranks, const double* theta, const void* bnode, uint32_t* invalid,
                   const BinnedScratch* binned, const SpeciesScalars* scalars, cudaStream_t s) {
  const MoverParams<P> mp = mover_params<P>(g, qom, dt, c);
  if (scalars) *scalars->written = 0;
  if (p->count == 0) return cudaSuccess;
  const unsigned blocks = grid_for(p->count, 256, 148u * 8u);
  const MoveIo<P> io{records<P>(p), records<P>(out ? out : p), ranks, out != nullptr && out != p};
  const auto* bn = (const typename P::Fld*)bnode;
  MoverScalars sc{scalars ? scalars->partials : nullptr, scalars ? scalars->stride : 0, 0};
  if (!binned) {
    mover_kernel<P><<<blocks, 256, 0, s>>>(g, mp, io, p->count, theta, bn, invalid, nullptr, sc);
    count_launches(1);
    if (scalars) *scalars->written = int(blocks);
    return cudaGetLastError();
  }
  // Bins checked by validate_bins: the run mover; otherwise the per-record
  // mover moves every record. Exactly one of the two works (the choice
  // depends only on the bins, not on flags the movers themselves raise).
  MoveCodes mc{binned->code, binned->transfer, &binned->state->fallback, &binned->state->bins_bad,
               (long long)g.nx * g.ny * g.nz};
  const long long runs = run_count(g);
  // One wave of resident blocks (148 SMs); each warp strides over the runs.
  const unsigned run_blocks = grid_for(runs * 32, kRunWarps * 32, 148u * unsigned(run_mover_blocks<P>()));
  run_mover_kernel<P><<<run_blocks, kRunWarps * 32, 0, s>>>(g, mp, io, p->count, theta, bn, binned->old_counts,
                                                            binned->old_offsets, invalid, mc, sc);
  sc.offset = int(run_blocks);
  mover_kernel<P><<<blocks, 256, 0, s>>>(g, mp, io, p->count, theta, bn, invalid, &binned->state->bins_bad, sc);
  count_launches(2);
  if (scalars) *scalars->written = int(run_blocks + blocks);
  return cudaGetLastError();
}

}  // namespace

cudaError_t launch_mover(int precision, const Geom& g, double qom, double dt, double c,
                         tpicb200_particles* p, tpicb200_particles* out, const uint32_t* ranks,
                         const double* theta, const void* bnode, uint32_t* invalid, const BinnedScratch* binned,
                         const SpeciesScalars* scalars, cudaStream_t s) {
  if (precision == TPICB200_PRECISION_DOUBLE)
    return launch<PDouble>(g, qom, dt, c, p, out, ranks, theta, bnode, invalid, binned, scalars, s);
  return launch<PMixed>(g, qom, dt, c, p, out, ranks, theta, bnode, invalid, binned, scalars, s);
}

}  // namespace tpicb200
