// Stable counting sort of one species' records by cell key.
//
// TPIC sorts with LPFx's direct-cell counting sort: histogram, scan,
// permutation by atomic cursors and one scatter per attribute
// (lpfx/algorithm/particle/device/cuda_hip/sort.hpp:64-260). Its device form
// is unstable within a bin (lpfx/algorithm/particle/device/sort.hpp:372-374);
// its host form (lpfx/algorithm/particle/host/sort.hpp:205-290) is stable.
// This sort produces the stable order, so the permutation, counts and offsets
// are bit-identical to the host sort:
//   1. histogram with warp-aggregated atomics (__match_any_sync),
//   2. exclusive scan of the bins,
//   3. placement by warp-aggregated atomic cursors (stable within a warp),
//   4. per-bin fix-up: each bin's source indices are sorted ascending, which
//      restores the input order among equal keys (warp bitonic sort in shared
//      memory; block merge-path sort for large bins),
//   5. one fused gather of every attribute through the permutation.
// An out-of-range key stops the sort after step 1 (the kernels of steps 2-5
// test the sort's own flag) and is reported through *invalid.
#include "kernels.cuh"

#include <cuda.h>
#include <mutex>

namespace tpicb200 {
namespace {

constexpr int kScanThreads = 256;
constexpr int kScanItems = 16;
constexpr int kScanTile = kScanThreads * kScanItems;
constexpr int kWarpBinCapacity = 256;   // per-warp shared-memory sort
constexpr int kBlockBinCapacity = 8192; // per-block shared-memory sort (32 KB)

// Scratch words after the scan block sums: [0] sort-local invalid flag,
// [1] number of large bins, then the large-bin list.
struct ScanScratch {
  uint32_t* block_sums;
  uint32_t* flag;
  uint32_t* large_count;
  uint32_t* large_bins;
};

__device__ __forceinline__ void aggregated_add(uint32_t* base, int32_t key, bool valid,
                                               uint32_t& position) {
  const unsigned lane = threadIdx.x & 31;
  const unsigned active = __ballot_sync(0xffffffffu, valid);
  const unsigned peers = __match_any_sync(0xffffffffu, valid ? key : -1);
  if (valid) {
    const unsigned group = peers & active;
    const int leader = __ffs(group) - 1;
    const unsigned rank = __popc(group & ((1u << lane) - 1u));
    uint32_t start = 0;
    if ((int)lane == leader) start = atomicAdd(base + key, __popc(group));
    start = __shfl_sync(group, start, leader);
    position = start + rank;
  }
}

// `gate`: the kernels of the general path run only when it is null or holds a
// nonzero word (the binned sort's fallback flag).
__device__ __forceinline__ bool closed(const uint32_t* gate) { return gate && *gate == 0; }

__global__ void __launch_bounds__(256) fill_kernel(uint32_t* out, long long n, uint32_t value,
                                                   const uint32_t* gate) {
  if (closed(gate)) return;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    out[i] = value;
}

__global__ void __launch_bounds__(256) copy_kernel(uint32_t* out, const uint32_t* __restrict__ in, long long n,
                                                   const uint32_t* gate) {
  if (closed(gate)) return;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    out[i] = in[i];
}

__global__ void __launch_bounds__(256) histogram_kernel(Geom g, const int32_t* __restrict__ keys,
                                                        uint32_t count, uint32_t* counts,
                                                        uint32_t* flag, const uint32_t* gate) {
  if (closed(gate)) return;
  const uint32_t stride = gridDim.x * blockDim.x;
  for (uint32_t base = blockIdx.x * blockDim.x + (threadIdx.x & ~31u); base < count; base += stride) {
    const uint32_t i = base + (threadIdx.x & 31);
    const bool in_range = i < count;
    const int32_t key = in_range ? keys[i] : -1;
    const bool ok = key >= 0 && (long long)key < g.bins;
    if (in_range && !ok) atomicExch(flag, 1u);
    uint32_t unused;
    aggregated_add(counts, key, in_range && ok, unused);
  }
}

__global__ void __launch_bounds__(kScanThreads) scan_reduce_kernel(const uint32_t* __restrict__ counts,
                                                                   long long bins, uint32_t* block_sums,
                                                                   const uint32_t* flag, const uint32_t* gate) {
  __shared__ uint32_t scratch[kScanThreads / 32];
  if (closed(gate) || *flag) return;
  const long long base = (long long)blockIdx.x * kScanTile;
  uint32_t sum = 0;
#pragma unroll
  for (int r = 0; r < kScanItems; ++r) {
    const long long i = base + threadIdx.x + (long long)r * kScanThreads;
    if (i < bins) sum += counts[i];
  }
  sum = block_sum<kScanThreads>(sum, scratch);
  if (threadIdx.x == 0) block_sums[blockIdx.x] = sum;
}

// Exclusive scan of the block sums by one block of 1024 threads.
__global__ void __launch_bounds__(1024) scan_block_sums_kernel(uint32_t* block_sums, int nblocks,
                                                               const uint32_t* flag, const uint32_t* gate) {
  __shared__ uint32_t warp_totals[32];
  if (closed(gate) || *flag) return;
  const int per = (nblocks + 1023) / 1024;
  const int first = threadIdx.x * per;
  uint32_t local = 0;
  for (int i = 0; i < per; ++i)
    if (first + i < nblocks) local += block_sums[first + i];
  // Block exclusive scan of `local`.
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t inclusive = local;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t t = __shfl_up_sync(0xffffffffu, inclusive, o);
    if (lane >= o) inclusive += t;
  }
  if (lane == 31) warp_totals[warp] = inclusive;
  __syncthreads();
  if (warp == 0) {
    uint32_t t = warp_totals[lane];
    uint32_t inc = t;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(0xffffffffu, inc, o);
      if (lane >= o) inc += y;
    }
    warp_totals[lane] = inc - t;
  }
  __syncthreads();
  uint32_t running = warp_totals[warp] + inclusive - local;
  for (int i = 0; i < per; ++i)
    if (first + i < nblocks) {
      const uint32_t v = block_sums[first + i];
      block_sums[first + i] = running;
      running += v;
    }
}

__global__ void __launch_bounds__(kScanThreads) scan_down_kernel(const uint32_t* __restrict__ counts,
                                                                 long long bins,
                                                                 const uint32_t* __restrict__ block_sums,
                                                                 uint32_t* offsets, const uint32_t* flag,
                                                                 const uint32_t* gate) {
  __shared__ uint32_t warp_totals[kScanThreads / 32];
  if (closed(gate) || *flag) return;
  const long long base = (long long)blockIdx.x * kScanTile + (long long)threadIdx.x * kScanItems;
  uint32_t items[kScanItems];
  uint32_t local = 0;
#pragma unroll
  for (int r = 0; r < kScanItems; ++r) {
    items[r] = base + r < bins ? counts[base + r] : 0u;
    local += items[r];
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t inclusive = local;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t t = __shfl_up_sync(0xffffffffu, inclusive, o);
    if (lane >= o) inclusive += t;
  }
  if (lane == 31) warp_totals[warp] = inclusive;
  __syncthreads();
  uint32_t warp_prefix = 0;
  for (int w = 0; w < warp; ++w) warp_prefix += warp_totals[w];
  uint32_t running = block_sums[blockIdx.x] + warp_prefix + inclusive - local;
#pragma unroll
  for (int r = 0; r < kScanItems; ++r) {
    if (base + r < bins) offsets[base + r] = running;
    running += items[r];
  }
  if (base + kScanItems >= bins && base < bins) offsets[bins] = running;
  if (bins == 0 && blockIdx.x == 0 && threadIdx.x == 0) offsets[0] = 0;
}

__global__ void __launch_bounds__(256) place_kernel(const int32_t* __restrict__ keys, uint32_t count,
                                                    uint32_t* cursor, uint32_t* perm,
                                                    const uint32_t* flag, const uint32_t* gate) {
  if (closed(gate) || *flag) return;
  const uint32_t stride = gridDim.x * blockDim.x;
  for (uint32_t base = blockIdx.x * blockDim.x + (threadIdx.x & ~31u); base < count; base += stride) {
    const uint32_t i = base + (threadIdx.x & 31);
    const bool valid = i < count;
    const int32_t key = valid ? keys[i] : -1;
    uint32_t position = 0;
    aggregated_add(cursor, key, valid, position);
    if (valid) perm[position] = i;
  }
}

// Warp-level bitonic sort of up to kWarpBinCapacity indices in shared memory.
__device__ __forceinline__ void warp_bitonic(uint32_t* s, int size) {
  const int lane = threadIdx.x & 31;
  for (int k = 2; k <= size; k <<= 1)
    for (int j = k >> 1; j > 0; j >>= 1) {
      for (int t = lane; t < size; t += 32) {
        const int partner = t ^ j;
        if (partner > t) {
          const uint32_t a = s[t], b = s[partner];
          const bool up = (t & k) == 0;
          if ((a > b) == up) { s[t] = b; s[partner] = a; }
        }
      }
      __syncwarp();
    }
}

__global__ void __launch_bounds__(256) fixup_small_kernel(const uint32_t* __restrict__ counts,
                                                          const uint32_t* __restrict__ offsets,
                                                          long long bins, uint32_t* perm,
                                                          uint32_t* large_count, uint32_t* large_bins,
                                                          const uint32_t* flag, const uint32_t* gate) {
  __shared__ uint32_t buffer[8][kWarpBinCapacity];
  if (closed(gate) || *flag) return;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t* s = buffer[warp];
  const long long warps = (long long)gridDim.x * 8;
  for (long long bin = (long long)blockIdx.x * 8 + warp; bin < bins; bin += warps) {
    const uint32_t n = counts[bin];
    if (n <= 1) continue;
    if (n > (uint32_t)kWarpBinCapacity) {
      if (lane == 0) large_bins[atomicAdd(large_count, 1u)] = (uint32_t)bin;
      continue;
    }
    const uint32_t first = offsets[bin];
    bool sorted = true;
    for (uint32_t t = lane; t < n; t += 32) {
      const uint32_t value = perm[first + t];
      s[t] = value;
      if (t > 0 && perm[first + t - 1] > value) sorted = false;
    }
    if (__all_sync(0xffffffffu, sorted)) continue;
    int size = 1;
    while (size < (int)n) size <<= 1;
    for (int t = n + lane; t < size; t += 32) s[t] = 0xffffffffu;
    __syncwarp();
    warp_bitonic(s, size);
    for (uint32_t t = lane; t < n; t += 32) perm[first + t] = s[t];
    __syncwarp();
  }
}

// One block per large bin. Up to kBlockBinCapacity entries sort in shared
// memory; larger bins merge runs in global memory with merge-path splits,
// ping-ponging with `scratch` (a free array of the output records).
__global__ void __launch_bounds__(1024) fixup_large_kernel(const uint32_t* __restrict__ counts,
                                                           const uint32_t* __restrict__ offsets,
                                                           uint32_t* perm, uint32_t* scratch,
                                                           const uint32_t* large_count,
                                                           const uint32_t* large_bins,
                                                           const uint32_t* flag, const uint32_t* gate) {
  __shared__ uint32_t s[kBlockBinCapacity];
  if (closed(gate) || *flag) return;
  const uint32_t nlarge = *large_count;
  for (uint32_t item = blockIdx.x; item < nlarge; item += gridDim.x) {
    const uint32_t bin = large_bins[item];
    const uint32_t n = counts[bin], first = offsets[bin];
    if (n <= (uint32_t)kBlockBinCapacity) {
      int size = 1;
      while (size < (int)n) size <<= 1;
      for (int t = threadIdx.x; t < size; t += blockDim.x) s[t] = t < (int)n ? perm[first + t] : 0xffffffffu;
      __syncthreads();
      for (int k = 2; k <= size; k <<= 1)
        for (int j = k >> 1; j > 0; j >>= 1) {
          for (int t = threadIdx.x; t < size; t += blockDim.x) {
            const int partner = t ^ j;
            if (partner > t) {
              const uint32_t a = s[t], b = s[partner];
              const bool up = (t & k) == 0;
              if ((a > b) == up) { s[t] = b; s[partner] = a; }
            }
          }
          __syncthreads();
        }
      for (int t = threadIdx.x; t < (int)n; t += blockDim.x) perm[first + t] = s[t];
      __syncthreads();
      continue;
    }
    // Bottom-up merge sort in global memory, width doubling.
    uint32_t* src = perm + first;
    uint32_t* dst = scratch + first;
    for (uint32_t width = 1; width < n; width <<= 1) {
      for (uint32_t t = threadIdx.x; t < n; t += blockDim.x) {
        const uint32_t run = t / (2 * width) * (2 * width);
        const uint32_t a0 = run, a1 = min(run + width, n), b1 = min(run + 2 * width, n);
        const uint32_t la = a1 - a0, lb = b1 - a1, d = t - run;
        // Merge path: i elements from A and d - i from B precede output d.
        uint32_t lo = d > lb ? d - lb : 0, hi = d < la ? d : la;
        while (lo < hi) {
          const uint32_t mid = (lo + hi) >> 1;
          if (src[a0 + mid] < src[a1 + d - mid - 1]) lo = mid + 1;
          else hi = mid;
        }
        const uint32_t i = lo, jb = d - i;
        uint32_t value;
        if (i < la && (jb >= lb || src[a0 + i] < src[a1 + jb])) value = src[a0 + i];
        else value = src[a1 + jb];
        dst[t] = value;
      }
      __syncthreads();
      uint32_t* tmp = src; src = dst; dst = tmp;
    }
    if (src != perm + first)
      for (uint32_t t = threadIdx.x; t < n; t += blockDim.x) perm[first + t] = src[t];
    __syncthreads();
  }
}

template <class Vel>
__global__ void __launch_bounds__(256) gather_kernel(const uint32_t* __restrict__ perm, uint32_t count,
    const double* __restrict__ irx, const double* __restrict__ iry, const double* __restrict__ irz,
    const Vel* __restrict__ iu, const Vel* __restrict__ iv, const Vel* __restrict__ iw,
    const double* __restrict__ iq, const int32_t* __restrict__ ikey, const uint64_t* __restrict__ iid,
    double* __restrict__ orx, double* __restrict__ ory, double* __restrict__ orz,
    Vel* __restrict__ ou, Vel* __restrict__ ov, Vel* __restrict__ ow, double* __restrict__ oq,
    int32_t* __restrict__ okey, uint64_t* __restrict__ oid, const uint32_t* flag, const uint32_t* gate) {
  if (closed(gate) || (flag && *flag)) return;
  for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < count; p += gridDim.x * blockDim.x) {
    const uint32_t s = perm[p];
    orx[p] = irx[s]; ory[p] = iry[s]; orz[p] = irz[s];
    ou[p] = iu[s]; ov[p] = iv[s]; ow[p] = iw[s];
    oq[p] = iq[s];
    okey[p] = ikey[s];
    if (oid) oid[p] = iid[s];
  }
}

__global__ void report_kernel(const uint32_t* flag, uint32_t* invalid, const uint32_t* gate) {
  if (closed(gate)) return;
  if (*flag && invalid) atomicAdd(invalid, 1u);
}

}  // namespace

size_t sort_scan_words(long long bins) {
  const long long nblocks = (bins + kScanTile - 1) / kScanTile;
  return size_t(nblocks) + 2 + size_t(bins);
}

namespace {

// The general sort; with a gate, every step runs only when *gate != 0.
cudaError_t enqueue_general(int precision, const Geom& g, const tpicb200_particles* in, tpicb200_particles* out,
                            uint32_t* counts, uint32_t* offsets, uint32_t* cursor, uint32_t* perm,
                            uint32_t* scan_scratch, uint32_t* invalid, const uint32_t* gate, cudaStream_t s) {
  const long long bins = g.bins;
  const int nblocks = int((bins + kScanTile - 1) / kScanTile);
  ScanScratch sc{scan_scratch, scan_scratch + nblocks, scan_scratch + nblocks + 1,
                 scan_scratch + nblocks + 2};
  const uint32_t n = in->count;
  cudaError_t e;
  if ((e = cudaMemsetAsync(sc.flag, 0, 2 * sizeof(uint32_t), s)) != cudaSuccess) return e;
  fill_kernel<<<grid_for(bins, 256, 148u * 8u), 256, 0, s>>>(counts, bins, 0u, gate);
  if (n) histogram_kernel<<<grid_for(n, 256, 148u * 8u), 256, 0, s>>>(g, in->cell, n, counts, sc.flag, gate);
  scan_reduce_kernel<<<nblocks, kScanThreads, 0, s>>>(counts, bins, sc.block_sums, sc.flag, gate);
  scan_block_sums_kernel<<<1, 1024, 0, s>>>(sc.block_sums, nblocks, sc.flag, gate);
  scan_down_kernel<<<nblocks, kScanThreads, 0, s>>>(counts, bins, sc.block_sums, offsets, sc.flag, gate);
  copy_kernel<<<grid_for(bins, 256, 148u * 8u), 256, 0, s>>>(cursor, offsets, bins, gate);
  int launches = 7;
  if (n) {
    place_kernel<<<grid_for(n, 256, 148u * 8u), 256, 0, s>>>(in->cell, n, cursor, perm, sc.flag, gate);
    fixup_small_kernel<<<grid_for(bins, 256, 148u * 16u), 256, 0, s>>>(
        counts, offsets, bins, perm, sc.large_count, sc.large_bins, sc.flag, gate);
    fixup_large_kernel<<<148, 1024, 0, s>>>(counts, offsets, perm, (uint32_t*)out->cell,
                                            sc.large_count, sc.large_bins, sc.flag, gate);
    const unsigned gb = grid_for(n, 256, 148u * 8u);
    if (precision == TPICB200_PRECISION_DOUBLE)
      gather_kernel<double><<<gb, 256, 0, s>>>(perm, n, (const double*)in->rx, (const double*)in->ry,
          (const double*)in->rz, (const double*)in->u, (const double*)in->v, (const double*)in->w,
          in->q, in->cell, in->id, (double*)out->rx, (double*)out->ry, (double*)out->rz,
          (double*)out->u, (double*)out->v, (double*)out->w, out->q, out->cell,
          in->id ? out->id : nullptr, sc.flag, gate);
    else
      gather_kernel<float><<<gb, 256, 0, s>>>(perm, n, (const double*)in->rx, (const double*)in->ry,
          (const double*)in->rz, (const float*)in->u, (const float*)in->v, (const float*)in->w,
          in->q, in->cell, in->id, (double*)out->rx, (double*)out->ry, (double*)out->rz,
          (float*)out->u, (float*)out->v, (float*)out->w, out->q, out->cell,
          in->id ? out->id : nullptr, sc.flag, gate);
    launches += 4;
  }
  report_kernel<<<1, 1, 0, s>>>(sc.flag, invalid, gate);
  count_launches(launches + 1);
  return cudaGetLastError();
}

// ---- Binned sort: the input is grouped by the bins of an earlier sort ----
//
// After the mover a species' records are still grouped by the cells of the
// previous sort, in increasing key order, and almost every record moved to
// one of the 27 cells around its old one. The stable order of a destination
// bin is then: its source cells in increasing key order and, within one
// source, the records in input order. So
//   1. direction codes d < 27 of every record and transfer counts T[d][c]
//      per old interior cell c: from the mover itself (it knows both cells)
//      or from classify_kernel (old cell from the bins, new from the key);
//      periodic_step gives each (source, destination) pair one code on
//      any extent (on an axis of two cells 0 -> 1 is -1 and 1 -> 0 is +1; on
//      an axis of one cell every step is 0);
//   2. validation: the old bins must tile the records in key order;
//   3. counts (thread per bin): counts'[b] = sum_d T[d][b - d];
//   4. scan of the counts;
//   5. bases (thread per interior bin): walking the 27 sources of b in key
//      order, T[d][c] becomes the first output position of c's records that
//      moved by d;
//   6. rank (a warp per run of up to 32 old cells of an x-row): a record's
//      position is its base plus its rank among the earlier records of its
//      cell with the same d, after checking that old cell + d is the cell of
//      its key; one gather then writes the sorted records.
// Any record that did not move to a neighbour, any invalid key, bins that do
// not tile the records or a failed scatter check raise the fallback flag,
// and the general sort, enqueued last and gated on the flag, rewrites the
// whole output (the binned gather is skipped). The output is the same stable
// order either way.

constexpr int kBinnedThreads = 256;
constexpr int kBinnedWarps = kBinnedThreads / 32;

// A warp takes a run (up to g.run_len <= 32 consecutive old interior cells
// of one x-row, run_cells) at a time. The run's records form one contiguous range; lane l
// holds cell l's record range. Writes the cells' first records to `start`
// (empty cells share their successor's start; unused entries are ~0) and
// returns the run's record range.
__device__ __forceinline__ void load_run_bins(const Geom& g, int i0, int len, int j, int k,
                                              const uint32_t* __restrict__ old_counts,
                                              const uint32_t* __restrict__ old_offsets, uint32_t* start,
                                              uint32_t& begin, uint32_t& end) {
  const int lane = threadIdx.x & 31;
  uint32_t off = 0xffffffffu, stop = 0;
  if (lane < len) {
    const int32_t key = g.encode(i0 + lane, j, k);
    off = old_offsets[key];
    stop = off + old_counts[key];
  }
  start[lane] = off;
  begin = __shfl_sync(0xffffffffu, off, 0);
  end = __shfl_sync(0xffffffffu, stop, len - 1);
  __syncwarp();
}

// Cell (offset in the run) of record p: the last cell whose start is at most p.
__device__ __forceinline__ int run_cell(const uint32_t* start, uint32_t p) {
  int c = 0;
#pragma unroll
  for (int step = 16; step > 0; step >>= 1)
    if (start[c + step] <= p) c += step;
  return c;
}

// Direction code of a record of old interior cell (i, j, k) whose key is now
// `key`, or -1 when the key is invalid or not one of the 27 neighbours.
__device__ __forceinline__ int key_move_code(const Geom& g, int i, int j, int k, int32_t key) {
  if (key < 0 || key >= g.bins) return -1;
  int a, b, c;
  g.decode(key, a, b, c);
  if (!g.interior_cell(a, b, c)) return -1;
  return move_code(g, i, j, k, a, b, c);
}

// The old bins must tile the records in key order: disjoint ranges in
// increasing key order, records only in interior cells, n records in all.
__global__ void __launch_bounds__(256) validate_bins_kernel(Geom g, uint32_t n,
                                                            const uint32_t* __restrict__ old_counts,
                                                            const uint32_t* __restrict__ old_offsets,
                                                            BinnedState* state) {
  __shared__ unsigned long long partial[8];
  bool bad = false;
  unsigned long long total = 0;
  for (long long b = blockIdx.x * (long long)blockDim.x + threadIdx.x; b < g.bins;
       b += (long long)gridDim.x * blockDim.x) {
    const uint32_t off = old_offsets[b], cnt = old_counts[b];
    if ((unsigned long long)off + cnt > old_offsets[b + 1]) bad = true;
    if (cnt) {
      int i, j, k;
      g.decode(int32_t(b), i, j, k);
      if (!g.interior_cell(i, j, k)) bad = true;
    }
    total += cnt;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0 && old_offsets[g.bins] > n) bad = true;
  total = warp_sum(total);
  if ((threadIdx.x & 31) == 0) partial[threadIdx.x >> 5] = total;
  const bool any_bad = __syncthreads_or(bad);
  if (threadIdx.x == 0) {
    unsigned long long block_total = 0;
    for (int w = 0; w < 8; ++w) block_total += partial[w];
    atomicAdd(&state->total, block_total);
    if (any_bad) {
      atomicExch(&state->bins_bad, 1u);
      atomicExch(&state->fallback, 1u);
    }
  }
}

__global__ void decide_kernel(uint32_t n, BinnedState* state) {
  if (state->total != (unsigned long long)n) {
    state->bins_bad = 1;
    state->fallback = 1;
  }
}

__global__ void __launch_bounds__(kBinnedThreads) classify_kernel(Geom g, const int32_t* __restrict__ keys,
    uint32_t n, const uint32_t* __restrict__ old_counts, const uint32_t* __restrict__ old_offsets,
    uint32_t* __restrict__ transfer, uint16_t* __restrict__ code, BinnedState* state) {
  __shared__ uint32_t starts[kBinnedWarps][kRunCells];
  __shared__ uint32_t hist[kBinnedWarps][27][33];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const long long cells = (long long)g.nx * g.ny * g.nz;
  const long long runs = run_count(g);
  bool bad = false;
  uint32_t* start = starts[warp];
  for (long long run = (long long)blockIdx.x * kBinnedWarps + warp; run < runs;
       run += (long long)gridDim.x * kBinnedWarps) {
    int i0, len, j, k;
    run_cells(g, run, i0, len, j, k);
    uint32_t begin, end;
    load_run_bins(g, i0, len, j, k, old_counts, old_offsets, start, begin, end);
#pragma unroll
    for (int d = 0; d < 27; ++d) hist[warp][d][lane] = 0;
    __syncwarp();
    if (begin > end || end > n) {  // bins that do not describe the records: no walk over them
      bad = true;
      continue;
    }
    // Four chunks per step: the key loads of all four are in flight together.
    for (uint32_t p0 = begin; p0 < end; p0 += 128) {
      int32_t key[4];
#pragma unroll
      for (int m = 0; m < 4; ++m) {
        const uint32_t p = p0 + 32 * m + lane;
        key[m] = p < end ? keys[p] : 0;
      }
#pragma unroll
      for (int m = 0; m < 4; ++m) {
        if (p0 + 32 * m >= end) break;
        const uint32_t p = p0 + 32 * m + lane;
        const bool live = p < end;
        int c = 0, d = -1;
        if (live) {
          c = run_cell(start, p);
          d = key_move_code(g, i0 + c, j, k, key[m]);
          if (d < 0) bad = true;
          code[p] = d < 0 ? kNoMove : uint16_t(d | (c << 5));
        }
        const int slot = d < 0 ? -1 : c * 27 + d;
        const unsigned peers = __match_any_sync(0xffffffffu, slot);
        if (slot >= 0 && lane == __ffs(peers) - 1) hist[warp][d][c] += __popc(peers);
        __syncwarp();
      }
    }
    if (lane < len) {
      const long long u = i0 + lane + (long long)g.nx * (j + (long long)g.ny * k);
#pragma unroll
      for (int d = 0; d < 27; ++d) transfer[(long long)d * cells + u] = hist[warp][d][lane];
    }
    __syncwarp();
  }
  if (__syncthreads_or(bad) && threadIdx.x == 0) atomicExch(&state->fallback, 1u);
}

__global__ void __launch_bounds__(256) binned_counts_kernel(Geom g, const uint32_t* __restrict__ transfer,
                                                            uint32_t* counts, const BinnedState* state) {
  if (state->fallback) return;
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const long long cells = (long long)nx * ny * nz;
  for (long long b = blockIdx.x * (long long)blockDim.x + threadIdx.x; b < g.bins;
       b += (long long)gridDim.x * blockDim.x) {
    int i, j, k;
    g.decode(int32_t(b), i, j, k);
    uint32_t sum = 0;
    if (g.interior_cell(i, j, k)) {
#pragma unroll
      for (int dz = -1; dz <= 1; ++dz)
#pragma unroll
        for (int dy = -1; dy <= 1; ++dy)
#pragma unroll
          for (int dx = -1; dx <= 1; ++dx) {
            // Neighbour offsets are -1..1: a conditional wrap (no modulo).
            int si = i - dx, sj = j - dy, sk = k - dz;
            si = si < 0 ? si + nx : (si >= nx ? si - nx : si);
            sj = sj < 0 ? sj + ny : (sj >= ny ? sj - ny : sj);
            sk = sk < 0 ? sk + nz : (sk >= nz ? sk - nz : sk);
            const int d = (dx + 1) + 3 * (dy + 1) + 9 * (dz + 1);
            sum += transfer[d * cells + si + (long long)nx * (sj + (long long)ny * sk)];
          }
    }
    counts[b] = sum;
  }
}

// Directions along one axis in increasing source coordinate: the sources of
// destination x are x - d (periodic).
__device__ __forceinline__ void source_order(int x, int n, int (&d)[3]) {
  if (x == 0) { d[0] = 0; d[1] = -1; d[2] = 1; }
  else if (x == n - 1) { d[0] = -1; d[1] = 1; d[2] = 0; }
  else { d[0] = 1; d[1] = 0; d[2] = -1; }
}

__global__ void __launch_bounds__(256) binned_bases_kernel(Geom g, const uint32_t* __restrict__ offsets,
                                                           uint32_t* transfer, const BinnedState* state) {
  if (state->fallback) return;
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const long long cells = (long long)nx * ny * nz;
  for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < cells;
       v += (long long)gridDim.x * blockDim.x) {
    const int i = int(v % nx);
    const long long r = v / nx;
    const int j = int(r % ny), k = int(r / ny);
    int ox[3], oy[3], oz[3];
    source_order(i, nx, ox);
    source_order(j, ny, oy);
    source_order(k, nz, oz);
    // Sources (periodic neighbours x - d) in increasing key order.
    long long index[27];
    uint32_t count[27];
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
      for (int b = 0; b < 3; ++b)
#pragma unroll
        for (int a = 0; a < 3; ++a) {
          const int dx = ox[a], dy = oy[b], dz = oz[c];
          int si = i - dx, sj = j - dy, sk = k - dz;
          si = si < 0 ? si + nx : (si >= nx ? si - nx : si);
          sj = sj < 0 ? sj + ny : (sj >= ny ? sj - ny : sj);
          sk = sk < 0 ? sk + nz : (sk >= nz ? sk - nz : sk);
          const int e = a + 3 * b + 9 * c;
          index[e] = ((dx + 1) + 3 * (dy + 1) + 9 * (dz + 1)) * cells + si + (long long)nx * (sj + (long long)ny * sk);
          count[e] = transfer[index[e]];
        }
    uint32_t base = offsets[g.encode(i, j, k)];
#pragma unroll
    for (int e = 0; e < 27; ++e) {
      transfer[index[e]] = base;
      base += count[e];
    }
  }
}

// The lane mask of a live lane's slot: the live lanes with the same slot
// value (one match instruction; a lane that is not live matches only itself).
__device__ __forceinline__ unsigned slot_group(int slot, bool live) {
  return __match_any_sync(0xffffffffu, live ? slot : -1 - int(threadIdx.x & 31));
}

// Output position of every record: perm[position] = record. The record goes
// to its base plus its rank among the earlier records of its cell with the
// same direction, after the check that its old cell + d is the cell of its
// key; the sorted records are then written by gather_kernel, whose stores
// are coalesced (records that changed cell would otherwise each write
// partial sectors of nine arrays).
__global__ void __launch_bounds__(kBinnedThreads) binned_rank_kernel(Geom g, uint32_t n,
    const uint32_t* __restrict__ old_counts, const uint32_t* __restrict__ old_offsets,
    const uint32_t* __restrict__ transfer, const uint16_t* __restrict__ code, const int32_t* __restrict__ keys,
    uint32_t* __restrict__ perm, BinnedState* state) {
  __shared__ uint32_t starts[kBinnedWarps][kRunCells];
  __shared__ uint32_t cursor[kBinnedWarps][27][33];
  if (state->fallback) return;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const long long cells = (long long)nx * ny * nz;
  const long long runs = run_count(g);
  const unsigned below = (1u << lane) - 1u;
  bool bad = false;
  for (long long run = (long long)blockIdx.x * kBinnedWarps + warp; run < runs;
       run += (long long)gridDim.x * kBinnedWarps) {
    int i0, len, j, k;
    run_cells(g, run, i0, len, j, k);
    uint32_t begin, end;
    load_run_bins(g, i0, len, j, k, old_counts, old_offsets, starts[warp], begin, end);
    if (lane < len) {
      const long long u = i0 + lane + (long long)nx * (j + (long long)ny * k);
#pragma unroll
      for (int d = 0; d < 27; ++d) cursor[warp][d][lane] = transfer[(long long)d * cells + u];
    }
    __syncwarp();
    // Four chunks per step: their loads are in flight together.
    for (uint32_t p0 = begin; p0 < end; p0 += 128) {
      uint16_t cd[4];
      int32_t key[4];
#pragma unroll
      for (int m = 0; m < 4; ++m) {
        const uint32_t p = p0 + 32 * m + lane;
        cd[m] = p < end ? code[p] : kNoMove;
        key[m] = p < end ? keys[p] : 0;
      }
#pragma unroll
      for (int m = 0; m < 4; ++m) {
        if (p0 + 32 * m >= end) break;
        const uint32_t p = p0 + 32 * m + lane;
        bool live = p < end;
        const int d = cd[m] & 31, c = (cd[m] >> 5) & 31;
        if (live) {
          // The record must land in the cell of its key: its old cell + d.
          int a = i0 + c + (d % 3) - 1, b = j + (d / 3) % 3 - 1, e = k + d / 9 - 1;
          a = a < 0 ? a + nx : (a >= nx ? a - nx : a);
          b = b < 0 ? b + ny : (b >= ny ? b - ny : b);
          e = e < 0 ? e + nz : (e >= nz ? e - nz : e);
          if (cd[m] == kNoMove || d >= 27 || c >= len || g.encode(a, b, e) != key[m]) {
            bad = true;
            live = false;
          }
        }
        const unsigned group = slot_group(c * 27 + d, live);
        if (live) {
          const uint32_t o = cursor[warp][d][c] + __popc(group & below);
          if (o < n) perm[o] = p;
          else bad = true;
        }
        __syncwarp();
        if (live && lane == __ffs(group) - 1) cursor[warp][d][c] += __popc(group);
        __syncwarp();
      }
    }
  }
  if (__any_sync(0xffffffffu, bad) && lane == 0) atomicExch(&state->fallback, 1u);
}

}  // namespace

cudaError_t launch_sort(int precision, const Geom& g, const tpicb200_particles* in,
                        tpicb200_particles* out, uint32_t* counts, uint32_t* offsets,
                        uint32_t* cursor, uint32_t* perm, uint32_t* scan_scratch,
                        uint32_t* invalid, cudaStream_t s) {
  out->count = in->count;
  return enqueue_general(precision, g, in, out, counts, offsets, cursor, perm, scan_scratch, invalid, nullptr, s);
}

cudaError_t launch_sorted_gather(int precision, const uint32_t* perm, const tpicb200_particles* in,
                                 tpicb200_particles* out, cudaStream_t s) {
  const uint32_t n = in->count;
  out->count = n;
  if (!n) return cudaSuccess;
  const unsigned gb = grid_for(n, 256, 148u * 8u);
  const uint32_t* zero = nullptr;  // no stop flag
  if (precision == TPICB200_PRECISION_DOUBLE)
    gather_kernel<double><<<gb, 256, 0, s>>>(perm, n, (const double*)in->rx, (const double*)in->ry,
        (const double*)in->rz, (const double*)in->u, (const double*)in->v, (const double*)in->w, in->q, in->cell,
        in->id, (double*)out->rx, (double*)out->ry, (double*)out->rz, (double*)out->u, (double*)out->v,
        (double*)out->w, out->q, out->cell, in->id ? out->id : nullptr, zero, nullptr);
  else
    gather_kernel<float><<<gb, 256, 0, s>>>(perm, n, (const double*)in->rx, (const double*)in->ry,
        (const double*)in->rz, (const float*)in->u, (const float*)in->v, (const float*)in->w, in->q, in->cell,
        in->id, (double*)out->rx, (double*)out->ry, (double*)out->rz, (float*)out->u, (float*)out->v,
        (float*)out->w, out->q, out->cell, in->id ? out->id : nullptr, zero, nullptr);
  count_launches(1);
  return cudaGetLastError();
}

size_t binned_scratch_words(const Geom& g) {
  const long long cells = (long long)g.nx * g.ny * g.nz;
  return 4 + size_t(2 * g.bins + 1) + size_t(27 * cells);
}

// Every periodic grid: on an axis of one or two cells each (source, destination)
// pair still has exactly one direction code (periodic_step), so the sources
// of a destination stay in increasing key order with no two nonempty
// directions sharing a source.
bool binned_sort_applies(const Geom& g) { return g.nx >= 1 && g.ny >= 1 && g.nz >= 1; }

BinnedScratch binned_scratch(const Geom& g, uint32_t* words, uint16_t* codes) {
  BinnedScratch b;
  b.state = reinterpret_cast<BinnedState*>(words);  // 4 words, 8-byte aligned
  b.old_counts = words + 4;
  b.old_offsets = b.old_counts + g.bins;
  b.transfer = b.old_offsets + g.bins + 1;
  b.code = codes;
  return b;
}

cudaError_t binned_begin(const Geom& g, const BinnedScratch& b, const uint32_t* in_counts,
                         const uint32_t* in_offsets, bool zero_transfer, cudaStream_t s) {
  // The old bins are copied first: the new ones may overwrite them in place.
  cudaError_t e;
  if ((e = cudaMemsetAsync(b.state, 0, sizeof(BinnedState), s)) != cudaSuccess) return e;
  if ((e = cudaMemcpyAsync(b.old_counts, in_counts, size_t(g.bins) * 4, cudaMemcpyDeviceToDevice, s)) !=
      cudaSuccess)
    return e;
  if ((e = cudaMemcpyAsync(b.old_offsets, in_offsets, size_t(g.bins + 1) * 4, cudaMemcpyDeviceToDevice, s)) !=
      cudaSuccess)
    return e;
  if (zero_transfer)
    e = cudaMemsetAsync(b.transfer, 0, size_t(27) * size_t((long long)g.nx * g.ny * g.nz) * 4, s);
  return e;
}

cudaError_t binned_validate(const Geom& g, const BinnedScratch& b, uint32_t n, cudaStream_t s) {
  validate_bins_kernel<<<grid_for(g.bins, 256, 148u * 8u), 256, 0, s>>>(g, n, b.old_counts, b.old_offsets, b.state);
  decide_kernel<<<1, 1, 0, s>>>(n, b.state);
  count_launches(2);
  return cudaGetLastError();
}

cudaError_t binned_finish(int precision, const Geom& g, const BinnedScratch& b, bool classify, bool materialize,
                          const tpicb200_particles* in, tpicb200_particles* out, uint32_t* counts,
                          uint32_t* offsets, uint32_t* cursor, uint32_t* perm, uint32_t* scan_scratch,
                          uint32_t* invalid, cudaStream_t s) {
  const long long bins = g.bins;
  const long long cells = (long long)g.nx * g.ny * g.nz;
  const uint32_t n = in->count;
  out->count = n;
  // One warp per run (up to 32 cells of an x-row).
  const unsigned runs_grid = grid_for(run_count(g) * 32, kBinnedThreads, 148u * 8u);
  int launches = 0;
  if (classify) {
    classify_kernel<<<runs_grid, kBinnedThreads, 0, s>>>(g, in->cell, n, b.old_counts, b.old_offsets, b.transfer,
                                                        b.code, b.state);
    ++launches;
  }
  binned_counts_kernel<<<grid_for(bins, 256, 148u * 16u), 256, 0, s>>>(g, b.transfer, counts, b.state);
  const int nblocks = int((bins + kScanTile - 1) / kScanTile);
  // The scan kernels take the fallback flag as their stop flag: they run only
  // when it is clear.
  ScanScratch sc{scan_scratch, scan_scratch + nblocks, scan_scratch + nblocks + 1, scan_scratch + nblocks + 2};
  scan_reduce_kernel<<<nblocks, kScanThreads, 0, s>>>(counts, bins, sc.block_sums, &b.state->fallback, nullptr);
  scan_block_sums_kernel<<<1, 1024, 0, s>>>(sc.block_sums, nblocks, &b.state->fallback, nullptr);
  scan_down_kernel<<<nblocks, kScanThreads, 0, s>>>(counts, bins, sc.block_sums, offsets, &b.state->fallback,
                                                    nullptr);
  binned_bases_kernel<<<grid_for(cells, 256, 148u * 16u), 256, 0, s>>>(g, offsets, b.transfer, b.state);
  binned_rank_kernel<<<runs_grid, kBinnedThreads, 0, s>>>(g, n, b.old_counts, b.old_offsets, b.transfer, b.code,
                                                           in->cell, perm, b.state);
  // The gather writes the records unless a check raised the fallback flag
  // (without `materialize` the caller reads the records through perm).
  if (n && materialize) {
    const unsigned gb = grid_for(n, 256, 148u * 8u);
    if (precision == TPICB200_PRECISION_DOUBLE)
      gather_kernel<double><<<gb, 256, 0, s>>>(perm, n, (const double*)in->rx, (const double*)in->ry,
          (const double*)in->rz, (const double*)in->u, (const double*)in->v, (const double*)in->w,
          in->q, in->cell, in->id, (double*)out->rx, (double*)out->ry, (double*)out->rz,
          (double*)out->u, (double*)out->v, (double*)out->w, out->q, out->cell,
          in->id ? out->id : nullptr, &b.state->fallback, nullptr);
    else
      gather_kernel<float><<<gb, 256, 0, s>>>(perm, n, (const double*)in->rx, (const double*)in->ry,
          (const double*)in->rz, (const float*)in->u, (const float*)in->v, (const float*)in->w,
          in->q, in->cell, in->id, (double*)out->rx, (double*)out->ry, (double*)out->rz,
          (float*)out->u, (float*)out->v, (float*)out->w, out->q, out->cell,
          in->id ? out->id : nullptr, &b.state->fallback, nullptr);
    ++launches;
  }
  count_launches(launches + 6);
  if (cudaError_t e = cudaGetLastError(); e != cudaSuccess) return e;
  // General sort, gated on the fallback flag: it rewrites every output.
  return enqueue_general(precision, g, in, out, counts, offsets, cursor, perm, scan_scratch, invalid,
                         &b.state->fallback, s);
}

cudaError_t launch_sort_binned(int precision, const Geom& g, const tpicb200_particles* in,
                               const uint32_t* in_counts, const uint32_t* in_offsets, tpicb200_particles* out,
                               uint32_t* counts, uint32_t* offsets, uint32_t* cursor, uint32_t* perm,
                               uint32_t* scan_scratch, uint32_t* binned_words, uint16_t* codes,
                               uint32_t* invalid, cudaStream_t s) {
  const BinnedScratch b = binned_scratch(g, binned_words, codes);
  if (cudaError_t e = binned_begin(g, b, in_counts, in_offsets, false, s); e != cudaSuccess) return e;
  if (cudaError_t e = binned_validate(g, b, in->count, s); e != cudaSuccess) return e;
  return binned_finish(precision, g, b, true, true, in, out, counts, offsets, cursor, perm, scan_scratch, invalid,
                       s);
}

// ---- Sort without a context and without allocation ----
//
// Some callers cannot allocate device memory for a sort: a caller that owns
// no context (the sort needs one only for its scratch), a caller whose device
// memory is held by another allocator's pool, or a loop that must not pay
// cudaMalloc's implicit device synchronisation. For them the general sort runs
// on a fixed file-scope scratch array instead of context buffers, for inputs
// up to TPICB200_SORT_STATIC_MAX_RECORDS records over up to
// TPICB200_SORT_STATIC_MAX_BINS bins; larger inputs are rejected. Every call
// shares the one array, so calls that overlap in time (other streams, other
// host threads) race on it; they must be ordered on one stream.

namespace {

constexpr long long kStaticRecords = TPICB200_SORT_STATIC_MAX_RECORDS;
constexpr long long kStaticBins = TPICB200_SORT_STATIC_MAX_BINS;
constexpr long long kStaticScanWords = (kStaticBins + kScanTile - 1) / kScanTile + 2 + kStaticBins;
// Permutation, cursors, then the scan block sums, flags and large-bin list.
constexpr long long kStaticWords = kStaticRecords + kStaticBins + kStaticScanWords;

static __device__ __align__(256) uint32_t g_static_scratch[kStaticWords];

// The array's address is resolved once per CUDA context: a device's primary
// context, a driver context a caller made current, or the primary context
// created again after cudaDeviceReset each hold their own copy of the array.
// A context's id (cuCtxGetId) is unique for the life of the process, so a
// context created after another was destroyed never reuses its cached
// address. The driver functions are fetched through the runtime, so the
// library needs no link against the driver library.
using CtxGetCurrentFn = CUresult (*)(CUcontext*);
using CtxGetIdFn = CUresult (*)(CUcontext, unsigned long long*);
constexpr int kStaticMaxContexts = 64;
std::mutex g_static_mutex;
struct StaticAddress {
  unsigned long long context_id;
  uint32_t* address;
};
StaticAddress g_static_address[kStaticMaxContexts] = {};
int g_static_used = 0;
CtxGetCurrentFn g_ctx_get_current = nullptr;
CtxGetIdFn g_ctx_get_id = nullptr;

cudaError_t current_context_id(unsigned long long* id) {
  CUcontext ctx = nullptr;
  if (g_ctx_get_current(&ctx) != CUDA_SUCCESS) return cudaErrorInvalidResourceHandle;
  if (!ctx) return cudaErrorContextIsDestroyed;
  return g_ctx_get_id(ctx, id) == CUDA_SUCCESS ? cudaSuccess : cudaErrorInvalidResourceHandle;
}

}  // namespace

long long sort_static_scratch_bytes() { return kStaticWords * 4; }

cudaError_t sort_static_setup(uint32_t** scratch) {
  std::lock_guard<std::mutex> lock(g_static_mutex);
  if (!g_ctx_get_current || !g_ctx_get_id) {
    cudaDriverEntryPointQueryResult found = cudaDriverEntryPointSymbolNotFound;
    void* fn = nullptr;
    cudaError_t e = cudaGetDriverEntryPoint("cuCtxGetCurrent", &fn, cudaEnableDefault, &found);
    if (e != cudaSuccess || found != cudaDriverEntryPointSuccess || !fn) return e != cudaSuccess ? e : cudaErrorNotSupported;
    g_ctx_get_current = reinterpret_cast<CtxGetCurrentFn>(fn);
    e = cudaGetDriverEntryPoint("cuCtxGetId", &fn, cudaEnableDefault, &found);
    if (e != cudaSuccess || found != cudaDriverEntryPointSuccess || !fn) return e != cudaSuccess ? e : cudaErrorNotSupported;
    g_ctx_get_id = reinterpret_cast<CtxGetIdFn>(fn);
  }
  unsigned long long id = 0;
  cudaError_t e = current_context_id(&id);
  uint32_t* fresh = nullptr;
  if (e == cudaErrorContextIsDestroyed) {
    // No context is current yet: resolving the symbol initialises the
    // current device's primary context and makes it current.
    e = cudaGetSymbolAddress((void**)&fresh, g_static_scratch);
    if (e != cudaSuccess) return e;
    e = current_context_id(&id);
  }
  if (e != cudaSuccess) return e;
  for (int i = 0; i < g_static_used; ++i)
    if (g_static_address[i].context_id == id) {
      *scratch = g_static_address[i].address;
      return cudaSuccess;
    }
  // Once per context, with that context current: the array's device address.
  if (!fresh) {
    e = cudaGetSymbolAddress((void**)&fresh, g_static_scratch);
    if (e != cudaSuccess) return e;
  }
  // Contexts beyond the table's size replace the oldest entry.
  const int slot = g_static_used < kStaticMaxContexts ? g_static_used++ : int(id % kStaticMaxContexts);
  g_static_address[slot] = {id, fresh};
  *scratch = fresh;
  return cudaSuccess;
}

cudaError_t launch_sort_static(int precision, const Geom& g, const tpicb200_particles* in, tpicb200_particles* out,
                               uint32_t* counts, uint32_t* offsets, uint32_t* invalid, uint32_t* scratch,
                               cudaStream_t s) {
  if ((long long)in->count > kStaticRecords || g.bins > kStaticBins) return cudaErrorInvalidValue;
  uint32_t* perm = scratch;
  uint32_t* cursor = perm + kStaticRecords;
  uint32_t* scan = cursor + kStaticBins;
  // The general sort clears what must start at zero on every call: its
  // flags and large-bin count (memset), the counts (fill); the cursors are
  // copied from the offsets and the permutation is fully written.
  out->count = in->count;
  return enqueue_general(precision, g, in, out, counts, offsets, cursor, perm, scan, invalid, nullptr, s);
}

}  // namespace tpicb200
