// Shared-memory radix sort + unique of one tile of 4096 uint64 keys.
//
// LSD radix sort with 4-bit digits: each of the 256 threads owns a contiguous
// run of 16 keys; per pass every thread counts its digits, a block-wide
// exclusive scan (16-bit lanes, two bins per register, warp shuffles, then a
// scan over the 8 warp totals) gives each (digit, thread) its output offset,
// and the thread scatters its keys in order, which keeps the sort stable.
// Unique marks the first key of every run of equal keys and compacts them
// with a block scan.  Padding keys are ~0 and are dropped by unique.
//
// The reference does the same stage device-wide with CUB
// (cuda/permutation_bitmap_batch.cu:148, cuda/segmented_hash_batch.cu:174,
// gpu/sort_unique_visited.cu:122-290); here it runs per tile, in shared memory,
// so it fuses with generation and the visited claim.
#pragma once
#include "device.cuh"

namespace mgbfs2 {

constexpr uint32_t kSortTile = 4096;
constexpr uint32_t kSortThreads = 256;
constexpr uint32_t kSortPerThread = kSortTile / kSortThreads;  // 16

struct SortScratch {
  unsigned long long keys[kSortTile];
  uint32_t warp_sums[kSortThreads / 32][8];
  uint32_t bin_base[16];
  uint32_t unique_count;
};

// Inclusive warp scan of eight packed registers (two 16-bit lanes each).
__device__ __forceinline__ void warp_scan8(uint32_t (&v)[8]) {
  const uint32_t lane = lane_id();
#pragma unroll
  for (int off = 1; off < 32; off <<= 1) {
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const uint32_t up = __shfl_up_sync(kFullMask, v[j], off);
      if (lane >= static_cast<uint32_t>(off)) v[j] += up;
    }
  }
}

// Sorts s.keys[0..kSortTile) ascending on the low key_bits bits.  Must be
// called by all kSortThreads threads of the block.
__device__ __forceinline__ void block_radix_sort(SortScratch& s, uint32_t key_bits) {
  const uint32_t tid = threadIdx.x, warp = tid >> 5, lane = lane_id();
  unsigned long long mine[kSortPerThread];
#pragma unroll
  for (uint32_t k = 0; k < kSortPerThread; ++k) mine[k] = s.keys[tid * kSortPerThread + k];
  for (uint32_t shift = 0; shift < key_bits; shift += 4) {
    uint32_t packed[8] = {0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll
    for (uint32_t k = 0; k < kSortPerThread; ++k) {
      const uint32_t d = static_cast<uint32_t>(mine[k] >> shift) & 15u;
      packed[d >> 1] += 1u << (16 * (d & 1));
    }
    uint32_t incl[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) incl[j] = packed[j];
    warp_scan8(incl);
    if (lane == 31) {
#pragma unroll
      for (int j = 0; j < 8; ++j) s.warp_sums[warp][j] = incl[j];
    }
    __syncthreads();
    if (tid < 16) {
      // Total per digit over the block, then exclusive scan over digits.
      uint32_t total = 0;
      for (uint32_t w = 0; w < kSortThreads / 32; ++w) total += (s.warp_sums[w][tid >> 1] >> (16 * (tid & 1))) & 0xffffu;
      s.bin_base[tid] = total;
    }
    __syncthreads();
    if (tid == 0) {
      uint32_t run = 0;
      for (int d = 0; d < 16; ++d) {
        const uint32_t t = s.bin_base[d];
        s.bin_base[d] = run;
        run += t;
      }
    }
    __syncthreads();
    uint32_t offset[16];
#pragma unroll
    for (int d = 0; d < 16; ++d) {
      uint32_t before_warps = 0;
      for (uint32_t w = 0; w < warp; ++w) before_warps += (s.warp_sums[w][d >> 1] >> (16 * (d & 1))) & 0xffffu;
      const uint32_t excl = ((incl[d >> 1] - packed[d >> 1]) >> (16 * (d & 1))) & 0xffffu;
      offset[d] = s.bin_base[d] + before_warps + excl;
    }
    __syncthreads();
#pragma unroll
    for (uint32_t k = 0; k < kSortPerThread; ++k) {
      const uint32_t d = static_cast<uint32_t>(mine[k] >> shift) & 15u;
      uint32_t pos = 0;
#pragma unroll
      for (int e = 0; e < 16; ++e)
        if (static_cast<uint32_t>(e) == d) pos = offset[e]++;
      s.keys[pos] = mine[k];
    }
    __syncthreads();
#pragma unroll
    for (uint32_t k = 0; k < kSortPerThread; ++k) mine[k] = s.keys[tid * kSortPerThread + k];
    __syncthreads();
  }
}

// Stable in-place compaction of s.keys: keeps the keys i with keep(i, key)
// at the front and returns their number (identical in every thread).  The
// predicate may read s.keys: every read happens before the first write.
template <typename Keep>
__device__ __forceinline__ uint32_t block_compact(SortScratch& s, Keep keep) {
  const uint32_t tid = threadIdx.x, warp = tid >> 5, lane = lane_id();
  unsigned long long mine[kSortPerThread];
  uint32_t flags = 0, count = 0;
#pragma unroll
  for (uint32_t k = 0; k < kSortPerThread; ++k) {
    const uint32_t i = tid * kSortPerThread + k;
    mine[k] = s.keys[i];
    if (keep(i, mine[k])) {
      flags |= 1u << k;
      ++count;
    }
  }
  uint32_t incl = count;
#pragma unroll
  for (int off = 1; off < 32; off <<= 1) {
    const uint32_t up = __shfl_up_sync(kFullMask, incl, off);
    if (lane >= static_cast<uint32_t>(off)) incl += up;
  }
  __syncthreads();
  if (lane == 31) s.warp_sums[warp][0] = incl;
  __syncthreads();
  uint32_t base = incl - count;
  for (uint32_t w = 0; w < warp; ++w) base += s.warp_sums[w][0];
  if (tid == kSortThreads - 1) s.unique_count = base + count;
  __syncthreads();
#pragma unroll
  for (uint32_t k = 0; k < kSortPerThread; ++k)
    if (flags & (1u << k)) s.keys[base++] = mine[k];
  __syncthreads();
  return s.unique_count;
}

// After block_radix_sort: compacts the distinct non-padding keys to the front
// of s.keys and returns their number.  Keys are compared on `mask` (bits
// outside it, such as a parent-edge tag, ride along with the first key of
// each run).
__device__ __forceinline__ uint32_t block_unique(SortScratch& s, unsigned long long mask = ~0ull) {
  return block_compact(s, [&](uint32_t i, unsigned long long key) {
    return key != kEmpty && (i == 0 || (s.keys[i - 1] & mask) != (key & mask));
  });
}

static __global__ void __launch_bounds__(kSortThreads) sort_unique_tiles_kernel(const unsigned long long* keys,
                                                                         unsigned long long count, uint32_t key_bits,
                                                                         unsigned long long* out, uint32_t* counts) {
  __shared__ SortScratch s;
  const unsigned long long tiles = (count + kSortTile - 1) / kSortTile;
  for (unsigned long long t = blockIdx.x; t < tiles; t += gridDim.x) {
    const unsigned long long base = t * kSortTile;
    for (uint32_t i = threadIdx.x; i < kSortTile; i += kSortThreads) {
      const unsigned long long idx = base + i;
      unsigned long long k = idx < count ? keys[idx] : kEmpty;
      if (key_bits < 64 && k != kEmpty) k &= (1ull << key_bits) - 1;
      s.keys[i] = k;
    }
    __syncthreads();
    // Padding (~0) fills the tail of the tile; its low key_bits bits are the
    // largest digit pattern, and the stable sort keeps it behind any real key
    // with the same low bits, so unique can drop it by value.
    block_radix_sort(s, key_bits);
    const uint32_t n = block_unique(s);
    for (uint32_t i = threadIdx.x; i < n; i += kSortThreads) out[base + i] = s.keys[i];
    if (threadIdx.x == 0) counts[t] = n;
    __syncthreads();
  }
}

}  // namespace mgbfs2
