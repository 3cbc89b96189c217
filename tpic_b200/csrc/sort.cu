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

__global__ void __launch_bounds__(256) histogram_kernel(Geom g, const int32_t* __restrict__ keys,
                                                        uint32_t count, uint32_t* counts,
                                                        uint32_t* flag) {
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
                                                                   const uint32_t* flag) {
  __shared__ uint32_t scratch[kScanThreads / 32];
  if (*flag) return;
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
                                                               const uint32_t* flag) {
  __shared__ uint32_t warp_totals[32];
  if (*flag) return;
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
                                                                 uint32_t* offsets, const uint32_t* flag) {
  __shared__ uint32_t warp_totals[kScanThreads / 32];
  if (*flag) return;
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
                                                    const uint32_t* flag) {
  if (*flag) return;
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
                                                          const uint32_t* flag) {
  __shared__ uint32_t buffer[8][kWarpBinCapacity];
  if (*flag) return;
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
                                                           const uint32_t* flag) {
  __shared__ uint32_t s[kBlockBinCapacity];
  if (*flag) return;
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
    int32_t* __restrict__ okey, uint64_t* __restrict__ oid, const uint32_t* flag) {
  if (*flag) return;
  for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < count; p += gridDim.x * blockDim.x) {
    const uint32_t s = perm[p];
    orx[p] = irx[s]; ory[p] = iry[s]; orz[p] = irz[s];
    ou[p] = iu[s]; ov[p] = iv[s]; ow[p] = iw[s];
    oq[p] = iq[s];
    okey[p] = ikey[s];
    if (oid) oid[p] = iid[s];
  }
}

__global__ void report_kernel(const uint32_t* flag, uint32_t* invalid) {
  if (*flag && invalid) atomicAdd(invalid, 1u);
}

}  // namespace

size_t sort_scan_words(long long bins) {
  const long long nblocks = (bins + kScanTile - 1) / kScanTile;
  return size_t(nblocks) + 2 + size_t(bins);
}

cudaError_t launch_sort(int precision, const Geom& g, const tpicb200_particles* in,
                        tpicb200_particles* out, uint32_t* counts, uint32_t* offsets,
                        uint32_t* cursor, uint32_t* perm, uint32_t* scan_scratch,
                        uint32_t* invalid, cudaStream_t s) {
  const long long bins = g.bins;
  const int nblocks = int((bins + kScanTile - 1) / kScanTile);
  ScanScratch sc{scan_scratch, scan_scratch + nblocks, scan_scratch + nblocks + 1,
                 scan_scratch + nblocks + 2};
  const uint32_t n = in->count;
  cudaError_t e;
  if ((e = cudaMemsetAsync(sc.flag, 0, 2 * sizeof(uint32_t), s)) != cudaSuccess) return e;
  if ((e = cudaMemsetAsync(counts, 0, size_t(bins) * sizeof(uint32_t), s)) != cudaSuccess) return e;
  if (n) histogram_kernel<<<grid_for(n, 256, 148u * 8u), 256, 0, s>>>(g, in->cell, n, counts, sc.flag);
  scan_reduce_kernel<<<nblocks, kScanThreads, 0, s>>>(counts, bins, sc.block_sums, sc.flag);
  scan_block_sums_kernel<<<1, 1024, 0, s>>>(sc.block_sums, nblocks, sc.flag);
  scan_down_kernel<<<nblocks, kScanThreads, 0, s>>>(counts, bins, sc.block_sums, offsets, sc.flag);
  if ((e = cudaMemcpyAsync(cursor, offsets, size_t(bins) * sizeof(uint32_t), cudaMemcpyDeviceToDevice,
                           s)) != cudaSuccess)
    return e;
  if (n) {
    place_kernel<<<grid_for(n, 256, 148u * 8u), 256, 0, s>>>(in->cell, n, cursor, perm, sc.flag);
    fixup_small_kernel<<<grid_for(bins, 256, 148u * 16u), 256, 0, s>>>(
        counts, offsets, bins, perm, sc.large_count, sc.large_bins, sc.flag);
    fixup_large_kernel<<<148, 1024, 0, s>>>(counts, offsets, perm, (uint32_t*)out->cell,
                                            sc.large_count, sc.large_bins, sc.flag);
    const unsigned gb = grid_for(n, 256, 148u * 8u);
    if (precision == TPICB200_PRECISION_DOUBLE)
      gather_kernel<double><<<gb, 256, 0, s>>>(perm, n, (const double*)in->rx, (const double*)in->ry,
          (const double*)in->rz, (const double*)in->u, (const double*)in->v, (const double*)in->w,
          in->q, in->cell, in->id, (double*)out->rx, (double*)out->ry, (double*)out->rz,
          (double*)out->u, (double*)out->v, (double*)out->w, out->q, out->cell,
          in->id ? out->id : nullptr, sc.flag);
    else
      gather_kernel<float><<<gb, 256, 0, s>>>(perm, n, (const double*)in->rx, (const double*)in->ry,
          (const double*)in->rz, (const float*)in->u, (const float*)in->v, (const float*)in->w,
          in->q, in->cell, in->id, (double*)out->rx, (double*)out->ry, (double*)out->rz,
          (float*)out->u, (float*)out->v, (float*)out->w, out->q, out->cell,
          in->id ? out->id : nullptr, sc.flag);
  }
  report_kernel<<<1, 1, 0, s>>>(sc.flag, invalid);
  count_launches(n ? 9 : 4);
  out->count = n;
  return cudaGetLastError();
}

}  // namespace tpicb200
