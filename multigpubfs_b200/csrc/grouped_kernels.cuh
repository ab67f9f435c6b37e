// Grouped layers of the Lehmer-bitmap path: claim first, then route only the
// winners.
//
// The frontier is stored grouped by the first K symbols of the state (group =
// the first K Lehmer digits, so group g owns the bitmap bits
// [g * (N-K)!, (g + 1) * (N-K)!), 10! bits = 454 KB for K = N - 10).  A layer
// is ONE kernel:
//
//   work items = chunks of the current frontier's groups, claimed from a
//                device counter in a group visiting order chosen for the
//                generators, so the resident blocks expand parents of a few
//                neighbouring groups at a time and the target groups they
//                share are revisited while still in L2;
//   per parent = apply each generator, rank the child, atomicOr its bit;
//   per winner = stage (state, the slot of the child's group in the block's
//                group table, rank within that slot's run) in shared memory;
//                a flush reserves one range per (block, group) and writes
//                the runs to the next frontier's group regions.
//
// With generators that move only a few leading positions into or out of the
// first K (LRX, adjacent transpositions), the children of one parent group
// fall into a few tens of groups, so the bitmap words a block touches stay in
// L2 although the whole bitmap (778 MB at N = 13) does not.  Compared with
// route + accept (bucket_kernels.cuh) only the winners are sorted and the
// 16 B per successor of bucket traffic disappear.
//
// Exactness: group regions are sized from the previous layer's distribution;
// a winner whose group region is full goes to the spill region, whose
// capacity is the exact bound on the next layer, so no winner is ever lost and
// no layer is redone.  The spill is expanded after the groups, without
// locality.  (The reference claims with random atomics from a flat candidate
// list: cuda/permutation_bitmap.cu:105-205.)
#pragma once
#include "packed_kernels.cuh"

namespace mgbfs2 {

constexpr uint32_t kGroupStage = 1024;  // staged winners per block (one pass of 256 x 4 parents)
constexpr int kGroupBlocksPerSM = 8;    // resident blocks the shared-memory carveout is sized for
constexpr uint32_t kMaxGroups = 24024;  // region tables: 14!/10! groups at most (S13: 1,716)
constexpr uint32_t kGroupChunk = 4096;  // parents per work item unless the plan chooses another size
constexpr uint32_t kMaxTranspGens = 32;  // adjacent-transposition generators of the incremental-rank path
static_assert(kGroupStage >= kBlock * 4, "a pass stages up to kBlock * ppt winners, ppt <= 4");


struct GroupedParams {
  const unsigned long long* frontier;
  // Regions 0..groups-1 are the groups, region `groups` is the spill.
  const unsigned long long* region_begin;  // regions
  const unsigned long long* region_count;  // regions
  const unsigned long long* item_prefix;   // regions + 1: exclusive prefix of work items, in visiting order
  const uint32_t* region_order;            // regions: the region visited j-th (the spill last)
  uint32_t regions, groups;
  const Term* terms;
  const uint32_t* term_begin;
  uint32_t gens, total_terms, gen_shift, ppt;
  unsigned long long* bitmap;
  unsigned long long* next;
  const unsigned long long* next_begin;  // regions (spill last)
  const unsigned long long* next_cap;    // regions (spill last)
  unsigned long long* next_count;        // regions: winners reserved per region (may pass a group's cap)
  unsigned long long* work;              // work-item counter, zero at launch
  uint32_t chunk;                        // parents per work item
  // Claims load the bitmap word first and skip the atomic when the bit is
  // set (claim_bit32).  The host sets it from kTestFirstGens generators up and
  // in layers whose parents won under 40 % of their tests; the incremental-
  // rank path (adjacent transpositions) always tests first.
  uint32_t test_first;
  Control* control;
  // Incremental-rank path (every generator swaps positions t-1 and t): per
  // generator t and the weights of digits t-1 and t in the group part and in
  // the in-group rank (0 where the position lies in the other part).
  const uint32_t* transp;                // gens x 5: t, wg(t-1), wg(t), wi(t-1), wi(t)
};

// The groups a block stages winners for live in a small open-addressing
// table: a work item's children reach a few dozen groups (LRX: X keeps the
// group, L and R reach ten each), so 256 slots replace per-group arrays of
// all 1,716 groups and leave room for eight blocks per SM.  A winner whose
// group finds no slot (a full table) is staged with kNoSlot and written to
// the spill region.
constexpr uint32_t kGroupSlots = 256;
constexpr uint32_t kEmptySlot = 0xffffffffu;
constexpr uint16_t kNoSlot = 0xffff;
static_assert(kGroupSlots == 256, "group_slot hashes to the top 8 bits");

struct GroupedSmem {
  unsigned long long state[kGroupStage];
  unsigned long long sdst[kGroupSlots];  // per slot: index in `next` of the block's reserved run
  uint32_t skey[kGroupSlots];            // per slot: the group, or kEmptySlot
  uint32_t scnt[kGroupSlots];            // per slot: staged winners, then (after the reservation) how many fit
  uint16_t rank[kGroupStage];            // per winner: its position in its slot's run
  uint16_t slot[kGroupStage];            // per winner: its slot, or kNoSlot
  uint16_t used[kGroupSlots];            // the occupied slots, in first-use order
  unsigned long long item, src;          // the claimed work item and its first parent's index
  uint32_t count, nused, n;
};

// The slot of group g, claimed if new; -1 when the table has none free.
// Bounded: at most kGroupSlots probes.
__device__ __forceinline__ int group_slot(GroupedSmem& sm, uint32_t g) {
  uint32_t h = (g * 0x9E3779B1u) >> 24;
  for (uint32_t probe = 0; probe < kGroupSlots; ++probe, h = (h + 1) & (kGroupSlots - 1)) {
    const uint32_t k = *reinterpret_cast<volatile uint32_t*>(&sm.skey[h]);
    if (k == g) return static_cast<int>(h);
    if (k == kEmptySlot) {
      const uint32_t prev = atomicCAS(&sm.skey[h], kEmptySlot, g);
      if (prev == kEmptySlot) {
        sm.used[atomicAdd(&sm.nused, 1u)] = static_cast<uint16_t>(h);
        return static_cast<int>(h);
      }
      if (prev == g) return static_cast<int>(h);
    }
  }
  return -1;
}

// Writes the staged winners: one reservation per (block, group); positions
// past a group's capacity, and winners without a slot, go to the spill
// region.  All threads call it.
__device__ __forceinline__ void grouped_flush(const GroupedParams& p, GroupedSmem& sm) {
  __syncthreads();
  const uint32_t used = sm.nused;
  for (uint32_t t = threadIdx.x; t < used; t += blockDim.x) {
    const uint32_t s = sm.used[t];
    const uint32_t g = sm.skey[s];
    const uint32_t staged = sm.scnt[s];
    const unsigned long long at = atomicAdd(&p.next_count[g], static_cast<unsigned long long>(staged));
    const unsigned long long cap = __ldg(&p.next_cap[g]);
    const unsigned long long room = at < cap ? cap - at : 0ull;
    sm.scnt[s] = room < staged ? static_cast<uint32_t>(room) : staged;
    sm.sdst[s] = __ldg(&p.next_begin[g]) + at;
  }
  __syncthreads();
  const uint32_t n = sm.count;
  bool overflow = false;
  for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) {
    const uint32_t s = sm.slot[i], r = sm.rank[i];
    if (s != kNoSlot && r < sm.scnt[s]) {
      p.next[sm.sdst[s] + r] = sm.state[i];
    } else {
      const unsigned long long sp = atomicAdd(&p.next_count[p.groups], 1ull);
      if (sp < __ldg(&p.next_cap[p.groups])) p.next[__ldg(&p.next_begin[p.groups]) + sp] = sm.state[i];
      else overflow = true;
    }
  }
  if (overflow) raise_error(&p.control->error, ERR_FRONTIER_OVERFLOW);
  if (threadIdx.x == 0 && n) atomicAdd(&p.control->next_count, static_cast<unsigned long long>(n));
  __syncthreads();
  for (uint32_t t = threadIdx.x; t < used; t += blockDim.x) {
    const uint32_t s = sm.used[t];
    sm.skey[s] = kEmptySlot;
    sm.scnt[s] = 0;
  }
  if (threadIdx.x == 0) {
    sm.count = 0;
    sm.nused = 0;
  }
  __syncthreads();
}

// Eight blocks per SM for the plain kernel (32 registers, no spills); the
// incremental-rank kernel spills at 32 registers and runs five.
template <int N, int K, bool TRANSP>
__global__ void __launch_bounds__(kBlock, TRANSP ? 5 : kGroupBlocksPerSM) expand_grouped(GroupedParams p) {
  extern __shared__ __align__(16) unsigned char dyn_smem[];
  GroupedSmem& sm = *reinterpret_cast<GroupedSmem*>(dyn_smem);
  Term* terms = reinterpret_cast<Term*>(dyn_smem + sizeof(GroupedSmem));
  uint32_t* tbegin = reinterpret_cast<uint32_t*>(dyn_smem + sizeof(GroupedSmem) + p.total_terms * sizeof(Term));
  for (uint32_t i = threadIdx.x; i < p.total_terms; i += blockDim.x) terms[i] = p.terms[i];
  for (uint32_t i = threadIdx.x; i <= 2 * p.gens; i += blockDim.x) tbegin[i] = p.term_begin[i];
  const uint32_t* inverse = tbegin + p.gens + 1;
  // The transposition table sits after the term offsets in the dynamic tail, sized only for TRANSP
  // launches, so the plain kernel's footprint does not grow.
  uint32_t* transp = tbegin + 2 * p.gens + 1;
  for (uint32_t t = threadIdx.x; t < kGroupSlots; t += blockDim.x) {
    sm.skey[t] = kEmptySlot;
    sm.scnt[t] = 0;
  }
  if constexpr (TRANSP)
    for (uint32_t i = threadIdx.x; i < 5 * p.gens; i += blockDim.x) transp[i] = p.transp[i];
  if (threadIdx.x == 0) {
    sm.count = 0;
    sm.nused = 0;
  }
  __syncthreads();
  constexpr uint64_t kGroupSize = factorial_u64(N - K);  // bits per group
  constexpr bool kSplitRank = N - K >= 8 && N - K <= 12;  // 32-bit in-group rank, word-aligned groups
  static_assert(!TRANSP || kSplitRank, "the incremental-rank path needs the split rank");
  constexpr uint64_t kGroupWords32 = kGroupSize / 32;
  constexpr uint64_t kStateMask = N >= 16 ? ~0ull : (1ull << (4 * N)) - 1ull;  // the N packed symbols
  const uint32_t tid = threadIdx.x, lane = lane_id();
  const uint32_t round = kBlock * p.ppt;
  const unsigned long long items = __ldg(&p.item_prefix[p.regions]);
  for (;;) {
    if (tid == 0) {
      // Claim a work item and locate it: a binary search over the region
      // prefix (in visiting order), once per work item.
      const unsigned long long item = atomicAdd(p.work, 1ull);
      sm.item = item;
      if (item < items) {
        uint32_t lo = 0, hi = p.regions;
        while (hi - lo > 1) {
          const uint32_t mid = (lo + hi) >> 1;
          if (__ldg(&p.item_prefix[mid]) <= item) lo = mid;
          else hi = mid;
        }
        const unsigned long long first = (item - __ldg(&p.item_prefix[lo])) * p.chunk;
        const uint32_t region = __ldg(&p.region_order[lo]);
        const unsigned long long avail = __ldg(&p.region_count[region]) - first;
        sm.n = static_cast<uint32_t>(avail < p.chunk ? avail : p.chunk);
        sm.src = __ldg(&p.region_begin[region]) + first;
      }
    }
    __syncthreads();
    if (sm.item >= items) break;
    const uint32_t n = sm.n;
    const unsigned long long* src = p.frontier + sm.src;
    __syncthreads();  // every thread has the item before thread 0 claims the next
    for (uint32_t r0 = 0; r0 < n; r0 += round) {
      uint64_t par[4];
      uint32_t skip[4];
      bool val[4];
      bool untagged = false;
      // Incremental-rank path: the parent's digits and split rank, once per parent.
      uint64_t pdig[4];
      uint32_t pgrp[4], pinner[4];
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        const uint32_t i = r0 + k * kBlock + tid;
        val[k] = k < static_cast<int>(p.ppt) && i < n;
        par[k] = val[k] ? src[i] : 0ull;
        const uint32_t tag = p.gen_shift ? static_cast<uint32_t>(par[k] >> p.gen_shift) : 0u;
        skip[k] = tag ? inverse[tag - 1] : 0xffffffffu;
        untagged = untagged || (val[k] && !tag);
        if constexpr (TRANSP) {
          pdig[k] = 0;
          pgrp[k] = pinner[k] = 0;
          if (val[k]) lehmer_digits_split4<N, K>(par[k], &pdig[k], &pgrp[k], &pinner[k]);
        }
      }
      // Pass j applies to every parent its j-th generator other than the
      // skipped one, so a round of tagged parents is done after gens - 1
      // passes with no idle lanes.
      const uint32_t passes = __syncthreads_or(untagged) ? p.gens : p.gens - 1;
      for (uint32_t j = 0; j < passes; ++j) {
        // Room for this pass's winners (at most one per parent).
        // Also flush a half-full slot table, which keeps probes short.
        __syncthreads();
        const uint32_t pending = sm.count, slots_used = sm.nused;
        __syncthreads();
        if (pending + round > kGroupStage || slots_used > kGroupSlots / 2) grouped_flush(p, sm);
#pragma unroll
        for (int k = 0; k < 4; ++k) {
          const uint32_t g = j + (j >= skip[k] ? 1u : 0u);
          const bool live = val[k] && g < p.gens;
          const unsigned long long gtag = p.gen_shift ? static_cast<unsigned long long>(g + 1) << p.gen_shift : 0ull;
          bool won = false;
          uint64_t c = 0;
          uint32_t grp = 0;
          if (live && TRANSP) {
            // Swapping positions t-1 and t changes only those two Lehmer
            // digits: with a, b the two symbols and c1, c2 their digits,
            // the new digits are c2 + [a < b] and c1 - [b < a].
            const uint32_t* ti = transp + 5 * g;
            const uint32_t t = ti[0];
            const uint32_t a = static_cast<uint32_t>(par[k] >> (4 * (t - 1))) & 15u;
            const uint32_t b = static_cast<uint32_t>(par[k] >> (4 * t)) & 15u;
            const unsigned long long x = static_cast<unsigned long long>(a ^ b);
            c = (par[k] ^ (x << (4 * (t - 1))) ^ (x << (4 * t))) & kStateMask;
            const int c1 = static_cast<int>((pdig[k] >> (4 * (t - 1))) & 15u);
            const int c2 = static_cast<int>((pdig[k] >> (4 * t)) & 15u);
            const int lt = a < b ? 1 : 0;
            const int d1 = c2 + lt - c1, d2 = c1 - (1 - lt) - c2;
            grp = static_cast<uint32_t>(static_cast<int>(pgrp[k]) + d1 * static_cast<int>(ti[1]) +
                                        d2 * static_cast<int>(ti[2]));
            const uint32_t inner = static_cast<uint32_t>(static_cast<int>(pinner[k]) + d1 * static_cast<int>(ti[3]) +
                                                         d2 * static_cast<int>(ti[4]));
            if (grp < p.groups && inner < kGroupSize) {
              const uint32_t bit = 1u << (inner & 31);
              unsigned int* word = reinterpret_cast<unsigned int*>(p.bitmap) +
                                   (static_cast<unsigned long long>(grp) * kGroupWords32 + (inner >> 5));
              won = claim_bit32(word, bit, l2_policy_evict_last());
            } else {
              raise_error(&p.control->error, ERR_RANK_RANGE);
            }
          } else if (live) {
            c = apply_terms(par[k], terms, tbegin[g], tbegin[g + 1]);
            if constexpr (kSplitRank) {
              // Group = the first K Lehmer digits, and the rank inside the group
              // in 32 bits; (N-K)! is a multiple of 32, so group regions start
              // on 32-bit words and the claim is a 32-bit atomicOr.
              uint32_t inner = 0;
              lehmer_split4<N, K>(c, &grp, &inner);
              const uint32_t bit = 1u << (inner & 31);
              unsigned int* word = reinterpret_cast<unsigned int*>(p.bitmap) +
                                   (static_cast<unsigned long long>(grp) * kGroupWords32 + (inner >> 5));
              won = p.test_first ? claim_bit32(word, bit, l2_policy_evict_last())
                                 : !(atomic_or_hinted32(word, bit, l2_policy_evict_last()) & bit);
            } else {
              const uint64_t r = lehmer_rank4<N>(c);
              const unsigned long long bit = 1ull << (r & 63);
              won = !(atomic_or_hinted(&p.bitmap[r >> 6], bit, l2_policy_evict_last()) & bit);
              grp = static_cast<uint32_t>(r / kGroupSize);
            }
          }
          const unsigned m = __ballot_sync(kFullMask, won);
          if (m) {
            const int leader = __ffs(m) - 1;
            uint32_t base = 0;
            if (static_cast<int>(lane) == leader) base = atomicAdd(&sm.count, static_cast<uint32_t>(__popc(m)));
            base = __shfl_sync(kFullMask, base, leader);
            if (won) {
              const unsigned peers = __match_any_sync(m, grp);
              const int gl = __ffs(peers) - 1;
              uint32_t packed = 0;  // slot | first rank << 16 (ranks stay below kGroupStage)
              if (static_cast<int>(lane) == gl) {
                const int gs = group_slot(sm, grp);
                packed = gs < 0 ? kNoSlot
                                : (static_cast<uint32_t>(gs) |
                                   atomicAdd(&sm.scnt[gs], static_cast<uint32_t>(__popc(peers))) << 16);
              }
              packed = __shfl_sync(peers, packed, gl);
              const uint32_t at = base + __popc(m & lanemask_lt());
              sm.state[at] = c | gtag;
              sm.slot[at] = static_cast<uint16_t>(packed & 0xffffu);
              sm.rank[at] = static_cast<uint16_t>((packed >> 16) + __popc(peers & lanemask_lt()));
            }
          }
        }
      }
    }
  }
  grouped_flush(p, sm);
}

// Copies a grouped frontier into one contiguous array (regions in order).
static __global__ void gather_regions(const unsigned long long* src, const unsigned long long* begin,
                                      const unsigned long long* count, const unsigned long long* out_prefix,
                                      uint32_t regions, unsigned long long* dst) {
  for (uint32_t r = blockIdx.x; r < regions; r += gridDim.x) {
    const unsigned long long b = begin[r], c = count[r], o = out_prefix[r];
    for (unsigned long long i = threadIdx.x; i < c; i += blockDim.x) dst[o + i] = src[b + i];
  }
}

}  // namespace mgbfs2
