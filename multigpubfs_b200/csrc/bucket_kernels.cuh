// Owner routing inside one GPU: the two-kernel bucketed layer expansion of
// the Lehmer-bitmap path.
//
// Shards are rank ranges fixed by the first `prefix` positions of the state:
// all permutations that start with the same k symbols occupy one contiguous
// block of (N-k)! Lehmer ranks, so
//     shard(state) = Horner of the first k Lehmer digits   (k cheap steps)
// and shard s owns bitmap bits [s * (N-k)!, (s + 1) * (N-k)!).  k is chosen so
// a shard's slice is a few MiB.
//
//   route  : parent -> successors (packed words) -> shard.  Every thread stages
//            its (at most kMaxEntries) successors in its own shared-memory
//            slots and counts them in its warp's shard histogram; one block
//            scan turns (shard, warp, rank-in-warp) into a position of the
//            block's shard-sorted run; one global atomicAdd per shard reserves
//            the bucket range; runs are written out coalesced.  No rank, no
//            visited-set access.
//   accept : work items = fixed-size chunks of the shard buckets, claimed in
//            shard-major order from a device-wide counter, so all resident
//            blocks work on the same one or two slices, which stay in L2.  Each
//            state is ranked and test-and-set (eight in flight per thread);
//            the winners -- already packed states -- are block-compacted and
//            appended to the next frontier with one reservation per item.
//
// The visited test thus costs 8 B written + 8 B read of streaming bucket
// traffic per successor plus L2-resident atomics, instead of a random DRAM
// sector read-modify-write (the reference routes by owner and claims with
// random atomics: cuda/permutation_bitmap.cu:27-48 and :105-205).
//
// Exactness: a shard bucket that overflows only sets ERR_BUCKET_OVERFLOW while
// its count keeps the exact total; accept then returns before touching the
// bitmap and the host redoes the layer with exact per-shard capacities.
#pragma once
#include "packed_kernels.cuh"

namespace mgbfs2 {

constexpr uint32_t kMaxShards = 256;
constexpr uint32_t kMaxEntries = 12;                 // staged successors per thread per flush
constexpr uint32_t kWarpsPerBlock = kBlock / 32;
constexpr uint32_t kStageCap = kBlock * kMaxEntries;  // 3072
constexpr uint32_t kAcceptChunk = 4096;               // bucket entries per accept work item
// Template N of the route / accept kernels for packed modular matrices: shard
// = the top entry (the most significant digit of the radix rank), so shard s
// owns the rank range [s * m^(E-1), (s + 1) * m^(E-1)).
constexpr int kRadixDomain = kMatrixN;

struct RouteParams {
  const unsigned long long* frontier;
  unsigned long long count;
  const Term* terms;
  const uint32_t* term_begin;
  uint32_t gens, total_terms, ppt, group;  // group: generators per flush (group * ppt <= kMaxEntries)
  uint32_t gen_shift, pad0;                // parent-edge tags, as in ExpandParams
  uint32_t shards, prefix;                 // shard = Horner of the first `prefix` Lehmer digits
  unsigned long long* buckets;             // all shards, shard s at [begin[s], begin[s] + cap[s])
  const unsigned long long* shard_begin;   // per shard
  const unsigned long long* shard_cap;     // per shard
  unsigned long long* shard_count;         // per shard, exact
  Control* control;
  // Hash routing (route_lehmer<0, 0>): shard = the region of the key's home
  // slot, (mix64(key) & table_mask) >> region_shift.
  unsigned long long table_mask, key_mask;
  uint32_t region_shift, pad1;
  // Owner routing across ranks (owners > 1): prefix block s belongs to rank
  // s mod owners and goes to bucket (s mod owners) * owner_blocks + s / owners,
  // so each rank's buckets are contiguous (owner-major, block-minor).
  uint32_t owners, owner_blocks;
  MatrixAction mat;  // packed modular matrices (route_lehmer<kRadixDomain, 1>)
};

struct AcceptParams {
  const unsigned long long* buckets;
  const unsigned long long* shard_begin;
  const unsigned long long* shard_count;
  uint32_t shards, pad;
  unsigned long long* bitmap;
  unsigned long long* next;
  unsigned long long capacity;
  unsigned long long* work;                // device work-item counter, zero at launch
  Control* control;
  // accept_hash: the all-visited table.
  unsigned long long* table;
  unsigned long long table_mask, key_mask;
  uint32_t probe_limit, pad1;
  // Owner slices (owners > 1): bucket b holds states of this rank's local
  // block b / owners, i.e. of prefix block (b / owners) * owners + owner, and
  // `bitmap` is the rank's slice: bit = local block * (N-K)! + rank in block.
  uint32_t owners, owner;
  MatrixAction mat;  // accept_lehmer<kRadixDomain, 1>: the radix rank's digits
};

// Shard of a successor: its rank range for the Lehmer bitmap, or (N = 0) the
// table region of its home slot for the hash.
template <int N, int K>
__device__ __forceinline__ uint32_t route_shard(const RouteParams& p, uint64_t c);

// Dynamic shared memory of route_lehmer (after the generator program).
struct RouteSmem {
  unsigned long long state[kStageCap];        // staged successors, slot [e][thread]; then the sorted run
  uint32_t tag[kStageCap];                    // shard | rank-in-warp-and-shard << 8; then the run's shard
  uint32_t hist[kWarpsPerBlock][kMaxShards];  // per-warp counts, then per-warp exclusive offsets
  uint32_t total[kMaxShards];
  uint32_t start[kMaxShards + 1];             // start of shard s in the sorted run
  unsigned long long gbase[kMaxShards];       // reserved bucket position of the run
};

// Shard of a packed permutation of N distinct 4-bit codes: the first K Lehmer
// digits in mixed radix N, N-1, ..., N-K+1.
template <int N, int K>
__device__ __forceinline__ uint32_t prefix_shard(uint64_t w) {
  uint32_t used = 0, shard = 0;
#pragma unroll
  for (int i = 0; i < K; ++i) {
    const uint32_t s = static_cast<uint32_t>(w >> (4 * i)) & 15u;
    shard = shard * static_cast<uint32_t>(N - i) + (s - __popc(used & ((1u << s) - 1u)));
    used |= 1u << s;
  }
  return shard;
}

template <int N, int K>
__device__ __forceinline__ uint32_t route_shard(const RouteParams& p, uint64_t c) {
  if constexpr (N == kRadixDomain) {
    const uint32_t top = p.mat.rows * p.mat.cols - 1;
    return static_cast<uint32_t>((c >> (p.mat.bits * top)) & ((1ull << p.mat.bits) - 1));
  } else if constexpr (N == 0) {
    return static_cast<uint32_t>((mix64(c & p.key_mask) & p.table_mask) >> p.region_shift);
  } else {
    const uint32_t s = prefix_shard<N, K>(c);
    return p.owners > 1 ? (s % p.owners) * p.owner_blocks + s / p.owners : s;
  }
}

template <int N, int K>
__global__ void __launch_bounds__(kBlock, 3) route_lehmer(RouteParams p) {
  extern __shared__ __align__(16) unsigned char dyn_smem[];
  RouteSmem& sm = *reinterpret_cast<RouteSmem*>(dyn_smem);
  Term* terms = reinterpret_cast<Term*>(dyn_smem + sizeof(RouteSmem));
  uint32_t* tbegin = reinterpret_cast<uint32_t*>(dyn_smem + sizeof(RouteSmem) + p.total_terms * sizeof(Term));
  for (uint32_t i = threadIdx.x; i < p.total_terms; i += blockDim.x) terms[i] = p.terms[i];
  for (uint32_t i = threadIdx.x; i <= 2 * p.gens; i += blockDim.x) tbegin[i] = p.term_begin[i];
  const uint32_t* inverse = tbegin + p.gens + 1;
  for (uint32_t i = threadIdx.x; i < kWarpsPerBlock * kMaxShards; i += blockDim.x) (&sm.hist[0][0])[i] = 0;
  __syncthreads();
  const uint32_t tid = threadIdx.x, warp = tid >> 5;
  const uint32_t tile = kBlock * p.ppt;
  const unsigned long long tiles = (p.count + tile - 1) / tile;
  for (unsigned long long t = blockIdx.x; t < tiles; t += gridDim.x) {
    const unsigned long long base = t * tile;
    uint64_t par[4] = {0, 0, 0, 0};
    bool val[4] = {false, false, false, false};
    if (p.ppt == 1) {
      const unsigned long long i0 = base + tid;
      if (i0 < p.count) {
        par[0] = p.frontier[i0];
        val[0] = true;
      }
    } else {
#pragma unroll
      for (int j = 0; j < 2; ++j) {
        if (2 * j >= static_cast<int>(p.ppt)) break;
        const unsigned long long i0 = base + 2ull * (j * kBlock + tid);
        if (i0 + 1 < p.count) {
          const ulonglong2 v = *reinterpret_cast<const ulonglong2*>(p.frontier + i0);
          par[2 * j] = v.x;
          par[2 * j + 1] = v.y;
          val[2 * j] = val[2 * j + 1] = true;
        } else if (i0 < p.count) {
          par[2 * j] = p.frontier[i0];
          val[2 * j] = true;
        }
      }
    }
    uint32_t skip[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const uint32_t tag = p.gen_shift ? static_cast<uint32_t>(par[k] >> p.gen_shift) : 0u;
      skip[k] = tag ? inverse[tag - 1] : 0xffffffffu;
    }
    for (uint32_t g0 = 0; g0 < p.gens; g0 += p.group) {
      const uint32_t g1 = min(p.gens, g0 + p.group);
      // Produce: successor, its shard, its rank within (warp, shard).  Only
      // live successors take a slot: slot m of this thread is m*kBlock + tid.
      uint32_t live = 0;
      for (uint32_t g = g0; g < g1; ++g) {
        const uint32_t tb = tbegin[g], te = tbegin[g + 1];
        const unsigned long long gtag = p.gen_shift ? static_cast<unsigned long long>(g + 1) << p.gen_shift : 0ull;
#pragma unroll
        for (int k = 0; k < 4; ++k) {
          if (k >= static_cast<int>(p.ppt)) break;
          if (val[k] && g != skip[k]) {
            uint64_t c;
            if constexpr (N == kRadixDomain) c = apply_matrix(p.mat, par[k], terms, tb, te);
            else c = apply_terms(par[k], terms, tb, te);
            const uint32_t s = route_shard<N, K>(p, c);
            const uint32_t slot = live * kBlock + tid;
            sm.state[slot] = c | gtag;
            sm.tag[slot] = s | (atomicAdd(&sm.hist[warp][s], 1u) << 8);
            ++live;
          }
        }
      }
      __syncthreads();
      // Per-shard column scan over warps, then an exclusive scan over shards.
      for (uint32_t s = tid; s < p.shards; s += kBlock) {
        uint32_t run = 0;
#pragma unroll
        for (uint32_t w = 0; w < kWarpsPerBlock; ++w) {
          const uint32_t c = sm.hist[w][s];
          sm.hist[w][s] = run;
          run += c;
        }
        sm.total[s] = run;
      }
      __syncthreads();
      if (tid < 32) {
        uint32_t carry = 0;
        for (uint32_t b = 0; b < p.shards; b += 32) {
          const uint32_t s = b + tid;
          const uint32_t v = s < p.shards ? sm.total[s] : 0u;
          uint32_t incl = v;
#pragma unroll
          for (int o = 1; o < 32; o <<= 1) {
            const uint32_t up = __shfl_up_sync(kFullMask, incl, o);
            if (tid >= static_cast<uint32_t>(o)) incl += up;
          }
          if (s < p.shards) sm.start[s] = carry + incl - v;
          carry += __shfl_sync(kFullMask, incl, 31);
        }
        if (tid == 0) sm.start[p.shards] = carry;
      }
      for (uint32_t s = tid; s < p.shards; s += kBlock)
        sm.gbase[s] = sm.total[s] ? atomicAdd(&p.shard_count[s], static_cast<unsigned long long>(sm.total[s])) : 0ull;
      __syncthreads();
      // Own entries to registers, then scatter them into the sorted run.
      unsigned long long st[kMaxEntries];
      uint32_t tg[kMaxEntries], pos[kMaxEntries];
#pragma unroll
      for (uint32_t e = 0; e < kMaxEntries; ++e) {
        if (e < live) {
          const uint32_t slot = e * kBlock + tid;
          tg[e] = sm.tag[slot];
          st[e] = sm.state[slot];
          const uint32_t s = tg[e] & 0xffu;
          pos[e] = sm.start[s] + sm.hist[warp][s] + (tg[e] >> 8);
        }
      }
      __syncthreads();
#pragma unroll
      for (uint32_t e = 0; e < kMaxEntries; ++e) {
        if (e < live) {
          sm.state[pos[e]] = st[e];
          sm.tag[pos[e]] = tg[e] & 0xffu;
        }
      }
      __syncthreads();
      const uint32_t n = sm.start[p.shards];
      bool overflow = false;
      for (uint32_t i = tid; i < n; i += kBlock) {
        const uint32_t s = sm.tag[i];
        const unsigned long long at = sm.gbase[s] + (i - sm.start[s]);
        if (at < __ldg(&p.shard_cap[s])) p.buckets[__ldg(&p.shard_begin[s]) + at] = sm.state[i];
        else overflow = true;
      }
      if (overflow) raise_error(&p.control->error, ERR_BUCKET_OVERFLOW);
      __syncthreads();
      for (uint32_t i = tid; i < kWarpsPerBlock * kMaxShards; i += kBlock) (&sm.hist[0][0])[i] = 0;
      __syncthreads();
    }
  }
}

// Lehmer rank of a state of shard `shard` (its first K digits): the shard's
// base rank shard * (N-K)! plus the Horner sum of the remaining digits, which
// stays below (N-K)! and so in 32 bits while N-K <= 12.
template <int N, int K>
__device__ __forceinline__ uint64_t lehmer_rank4_in_shard(uint64_t w, uint32_t shard) {
  if constexpr (N - K > 12) {
    return lehmer_rank4<N>(w);
  } else {
    constexpr uint32_t kFact[13] = {1u, 1u, 2u, 6u, 24u, 120u, 720u, 5040u, 40320u, 362880u, 3628800u, 39916800u,
                                    479001600u};
    const uint32_t lo_word = static_cast<uint32_t>(w), hi_word = static_cast<uint32_t>(w >> 32);
    uint32_t used = 0, tail = 0;
#pragma unroll
    for (int i = 0; i < N - 1; ++i) {
      const uint32_t s = (i < 8 ? (lo_word >> (4 * i)) : (hi_word >> (4 * (i - 8)))) & 15u;
      if (i >= K) tail = tail * static_cast<uint32_t>(N - i) + (s - __popc(used & ((1u << s) - 1u)));
      used |= 1u << s;
    }
    return static_cast<uint64_t>(shard) * kFact[N - K] + tail;
  }
}

// Counting pass for exactly sized buckets: the shard histogram of all
// successors of the frontier (same generation and shard rule as route).
template <int N, int K>
__global__ void __launch_bounds__(kBlock) count_lehmer(RouteParams p) {
  extern __shared__ __align__(16) unsigned char dyn_smem[];
  uint32_t* hist = reinterpret_cast<uint32_t*>(dyn_smem);
  Term* terms = reinterpret_cast<Term*>(dyn_smem + kMaxShards * sizeof(uint32_t));
  uint32_t* tbegin = reinterpret_cast<uint32_t*>(reinterpret_cast<unsigned char*>(terms) + p.total_terms * sizeof(Term));
  for (uint32_t i = threadIdx.x; i < p.total_terms; i += blockDim.x) terms[i] = p.terms[i];
  for (uint32_t i = threadIdx.x; i <= 2 * p.gens; i += blockDim.x) tbegin[i] = p.term_begin[i];
  for (uint32_t s = threadIdx.x; s < p.shards; s += blockDim.x) hist[s] = 0;
  __syncthreads();
  const uint32_t* inverse = tbegin + p.gens + 1;
  for (unsigned long long i = blockIdx.x * static_cast<unsigned long long>(blockDim.x) + threadIdx.x; i < p.count;
       i += static_cast<unsigned long long>(gridDim.x) * blockDim.x) {
    const unsigned long long w = p.frontier[i];
    const uint32_t tag = p.gen_shift ? static_cast<uint32_t>(w >> p.gen_shift) : 0u;
    const uint32_t skip = tag ? inverse[tag - 1] : 0xffffffffu;
    for (uint32_t g = 0; g < p.gens; ++g)
      if (g != skip) {
        uint64_t c;
        if constexpr (N == kRadixDomain) c = apply_matrix(p.mat, w, terms, tbegin[g], tbegin[g + 1]);
        else c = apply_terms(w, terms, tbegin[g], tbegin[g + 1]);
        atomicAdd(&hist[route_shard<N, K>(p, c)], 1u);
      }
  }
  __syncthreads();
  for (uint32_t s = threadIdx.x; s < p.shards; s += blockDim.x)
    if (hist[s]) atomicAdd(&p.shard_count[s], static_cast<unsigned long long>(hist[s]));
}

template <int N, int K>
__global__ void __launch_bounds__(kBlock) accept_lehmer(AcceptParams p) {
  __shared__ unsigned long long win[kAcceptChunk];
  __shared__ unsigned long long item_prefix[kMaxShards + 1];
  __shared__ unsigned long long item_s;
  __shared__ uint32_t win_count;
  __shared__ unsigned long long win_base;
  // A routed layer whose buckets overflowed is redone by the host: leave the
  // bitmap untouched.
  if (*reinterpret_cast<volatile unsigned int*>(&p.control->error) & ERR_BUCKET_OVERFLOW) return;
  if (threadIdx.x == 0) {
    unsigned long long run = 0;
    for (uint32_t s = 0; s < p.shards; ++s) {
      item_prefix[s] = run;
      run += (p.shard_count[s] + kAcceptChunk - 1) / kAcceptChunk;
    }
    item_prefix[p.shards] = run;
    win_count = 0;
  }
  __syncthreads();
  const uint32_t tid = threadIdx.x, lane = lane_id();
  const unsigned long long items = item_prefix[p.shards];
  for (;;) {
    // Items are claimed in shard-major order by all blocks together.
    if (tid == 0) item_s = atomicAdd(p.work, 1ull);
    __syncthreads();
    const unsigned long long item = item_s;
    if (item >= items) break;
    uint32_t lo = 0, hi = p.shards;
    while (hi - lo > 1) {
      const uint32_t mid = (lo + hi) >> 1;
      if (item_prefix[mid] <= item) lo = mid;
      else hi = mid;
    }
    const uint32_t s = lo;
    const unsigned long long first = (item - item_prefix[s]) * kAcceptChunk;
    const uint32_t n = static_cast<uint32_t>(min(static_cast<unsigned long long>(kAcceptChunk), p.shard_count[s] - first));
    const unsigned long long* src = p.buckets + p.shard_begin[s] + first;
    // Prefix block of the bucket's states and the offset of its bits: on one
    // GPU the bucket is the block and its bits are its ranks; on an owner
    // slice, local block j = s / owners holds prefix block j * owners + owner.
    const bool sliced = N > 0 && p.owners > 1;
    const uint32_t local = sliced ? s / p.owners : s;
    const uint32_t block = sliced ? local * p.owners + p.owner : s;
    uint64_t shift = 0;
    if constexpr (N > 0) {
      constexpr uint64_t kBlockRanks = factorial_u64(N - K);
      shift = static_cast<uint64_t>(block - local) * kBlockRanks;
    }
    for (uint32_t round = 0; round < n; round += 8 * kBlock) {
      unsigned long long w[8], old[8];
      uint64_t r[8];
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        const uint32_t i = round + k * kBlock + tid;
        w[k] = i < n ? src[i] : 0ull;
      }
      bool bad = false;
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        const uint32_t i = round + k * kBlock + tid;
        // A state routed to a rank that does not own it is never claimed.
        bool mine = true;
        if constexpr (N > 0) {
          mine = !sliced || prefix_shard<N, K>(w[k]) == block;
          r[k] = lehmer_rank4_in_shard<N, K>(w[k], block) - shift;
        } else {
          r[k] = radix_rank(w[k], p.mat);
        }
        bad = bad || (i < n && !mine);
        old[k] = i < n && mine ? atomicOr(&p.bitmap[r[k] >> 6], 1ull << (r[k] & 63)) : ~0ull;
      }
      if (bad) raise_error(&p.control->error, ERR_BAD_REFERENCE);
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        const bool won = !(old[k] & (1ull << (r[k] & 63)));
        const unsigned m = __ballot_sync(kFullMask, won);
        if (m) {
          const int leader = __ffs(m) - 1;
          uint32_t wb = 0;
          if (static_cast<int>(lane) == leader) wb = atomicAdd(&win_count, static_cast<uint32_t>(__popc(m)));
          wb = __shfl_sync(kFullMask, wb, leader);
          if (won) win[wb + __popc(m & lanemask_lt())] = w[k];
        }
      }
    }
    __syncthreads();
    const uint32_t nw = win_count;
    if (tid == 0 && nw) win_base = atomicAdd(&p.control->next_count, static_cast<unsigned long long>(nw));
    __syncthreads();
    bool overflow = false;
    for (uint32_t i = tid; i < nw; i += kBlock) {
      const unsigned long long at = win_base + i;
      if (at < p.capacity) p.next[at] = win[i];
      else overflow = true;
    }
    if (overflow) raise_error(&p.control->error, ERR_FRONTIER_OVERFLOW);
    __syncthreads();
    if (tid == 0) win_count = 0;
  }
}

// Accept for hash-routed layers: items are chunks of one table region, claimed
// region-major from a device counter, so the resident blocks insert into one or
// two L2-sized regions.  The home slots of eight keys per thread are read
// before any result is used; a key found there is done, the others insert
// (CAS, probing on).  Winners are appended like accept_lehmer's.
static __global__ void __launch_bounds__(kBlock) accept_hash(AcceptParams p) {
  __shared__ unsigned long long win[kAcceptChunk];
  __shared__ unsigned long long item_prefix[kMaxShards + 1];
  __shared__ unsigned long long item_s;
  __shared__ uint32_t win_count;
  __shared__ unsigned long long win_base;
  if (*reinterpret_cast<volatile unsigned int*>(&p.control->error) & ERR_BUCKET_OVERFLOW) return;
  if (threadIdx.x == 0) {
    unsigned long long run = 0;
    for (uint32_t s = 0; s < p.shards; ++s) {
      item_prefix[s] = run;
      run += (p.shard_count[s] + kAcceptChunk - 1) / kAcceptChunk;
    }
    item_prefix[p.shards] = run;
    win_count = 0;
  }
  __syncthreads();
  const uint32_t tid = threadIdx.x, lane = lane_id();
  const unsigned long long items = item_prefix[p.shards];
  for (;;) {
    if (tid == 0) item_s = atomicAdd(p.work, 1ull);
    __syncthreads();
    const unsigned long long item = item_s;
    if (item >= items) break;
    uint32_t lo = 0, hi = p.shards;
    while (hi - lo > 1) {
      const uint32_t mid = (lo + hi) >> 1;
      if (item_prefix[mid] <= item) lo = mid;
      else hi = mid;
    }
    const uint32_t s = lo;
    const unsigned long long first = (item - item_prefix[s]) * kAcceptChunk;
    const uint32_t n = static_cast<uint32_t>(min(static_cast<unsigned long long>(kAcceptChunk), p.shard_count[s] - first));
    const unsigned long long* src = p.buckets + p.shard_begin[s] + first;
    for (uint32_t round = 0; round < n; round += 8 * kBlock) {
      unsigned long long w[8], prev[8];
      uint64_t slot[8];
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        const uint32_t i = round + k * kBlock + tid;
        w[k] = i < n ? src[i] : 0ull;
      }
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        const uint32_t i = round + k * kBlock + tid;
        const uint64_t key = w[k] & p.key_mask;
        slot[k] = mix64(key) & p.table_mask;
        prev[k] = i < n ? *reinterpret_cast<volatile unsigned long long*>(&p.table[slot[k]]) : key;
      }
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        const uint32_t i = round + k * kBlock + tid;
        const uint64_t key = w[k] & p.key_mask;
        bool won = false;
        if (i < n && (prev[k] & p.key_mask) != key) {
          // Empty or another key in the home slot: insert (CAS and probe on).
          const int rc = hash_insert(p.table, p.table_mask, key, p.key_mask, 0, p.probe_limit);
          if (rc < 0) raise_error(&p.control->error, ERR_TABLE_FULL);
          won = rc == 1;
        }
        const unsigned m = __ballot_sync(kFullMask, won);
        if (m) {
          const int leader = __ffs(m) - 1;
          uint32_t wb = 0;
          if (static_cast<int>(lane) == leader) wb = atomicAdd(&win_count, static_cast<uint32_t>(__popc(m)));
          wb = __shfl_sync(kFullMask, wb, leader);
          if (won) win[wb + __popc(m & lanemask_lt())] = w[k];
        }
      }
    }
    __syncthreads();
    const uint32_t nw = win_count;
    if (tid == 0 && nw) win_base = atomicAdd(&p.control->next_count, static_cast<unsigned long long>(nw));
    __syncthreads();
    bool overflow = false;
    for (uint32_t i = tid; i < nw; i += kBlock) {
      const unsigned long long at = win_base + i;
      if (at < p.capacity) p.next[at] = win[i];
      else overflow = true;
    }
    if (overflow) raise_error(&p.control->error, ERR_FRONTIER_OVERFLOW);
    __syncthreads();
    if (tid == 0) win_count = 0;
  }
}

}  // namespace mgbfs2
