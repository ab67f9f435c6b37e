// Device building blocks shared by every BFS kernel of libmgbfs2.
//
// State encoding (packed path): a permutation state of n positions is one
// uint64 word; position i holds a dense symbol code in bits [b*i, b*i+b),
// b in {4, 8, 16, 32}, n*b <= 64.  Codes are the ranks of the distinct start
// labels (the permutation action only moves labels, so the label multiset is
// invariant and the code map is lossless).  This is the layout of
// scripts/cpu_small_bfs.py:21-27 and gpu/cayley_bfs.cu:50-55 in the reference.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace mgbfs2 {

// ---------------------------------------------------------------------------
// Sticky device status bits (the reference keeps the same idea in one
// uint32 error word: cuda/generic_visited.h:19, cuda/generic_route.h:15-16).
enum : uint32_t {
  ERR_FRONTIER_OVERFLOW = 1u << 0,  // next-frontier capacity exceeded (count stays exact)
  ERR_TABLE_FULL = 1u << 1,         // hash probe limit reached, key not inserted
  ERR_RANK_RANGE = 1u << 2,         // a state ranked outside the bitmap domain
  ERR_BUCKET_OVERFLOW = 1u << 3,    // a shard bucket overflowed
  ERR_WAIT_LIMIT = 1u << 4,         // a bounded wait gave up
  ERR_ARENA_OVERFLOW = 1u << 5,     // wide-key arena capacity exceeded
  ERR_BAD_STATE = 1u << 6,          // malformed input state
};

constexpr uint32_t kFullMask = 0xffffffffu;
constexpr uint64_t kEmpty = ~0ull;  // never a packed state: code 0 always occurs

// One displacement group of a generator: child |= ((p >> rshift) << lshift) & mask.
// A generator g (child[i] = parent[g[i]]) becomes one term per distinct
// displacement g[i] - i, so L/R cost 2 terms and a transposition 3.
struct Term {
  unsigned long long mask;
  uint32_t rshift, lshift;
};

struct Control {
  unsigned long long next_count;  // states appended to the next frontier (exact, may exceed capacity)
  unsigned long long aux;         // kernel-specific counter (bucket totals, probes)
  unsigned int error;             // sticky ERR_* bits
  unsigned int pad;
};

__device__ __forceinline__ void raise_error(unsigned int* error, uint32_t bits) {
  atomicOr(error, bits);
}

constexpr uint32_t kBarrierPolls = 1u << 22;

// Grid-wide barrier of a cooperative launch, with a bounded wait.  Thread 0
// of each block arrives on *count; the last to arrive resets it and advances
// *gen with a release store; the others poll *gen with acquire loads, at most
// kBarrierPolls times, after which they raise ERR_WAIT_LIMIT in *error and
// return false (the caller then ends the kernel: nothing waits forever).
// Every thread orders its later loads after the barrier.  *count and *gen
// start at zero for each launch.
__device__ __forceinline__ bool grid_barrier(unsigned int* count, unsigned int* gen, unsigned int* error) {
  __shared__ int barrier_ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    barrier_ok = 1;
    unsigned int g;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(g) : "l"(gen) : "memory");
    __threadfence();
    if (atomicAdd(count, 1u) == gridDim.x - 1) {
      *count = 0;
      asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(gen), "r"(g + 1) : "memory");
    } else {
      for (uint32_t polls = 0;; ++polls) {
        unsigned int now;
        asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(now) : "l"(gen) : "memory");
        if (now != g) break;
        if (polls >= kBarrierPolls) {
          raise_error(error, ERR_WAIT_LIMIT);
          barrier_ok = 0;
          break;
        }
        __nanosleep(64);
      }
    }
  }
  __syncthreads();
  asm volatile("fence.acq_rel.gpu;" ::: "memory");
  return barrier_ok != 0;
}

__device__ __forceinline__ uint64_t apply_terms(uint64_t p, const Term* t, uint32_t begin, uint32_t end) {
  uint64_t c = 0;
  for (uint32_t k = begin; k < end; ++k) c |= ((p >> t[k].rshift) << t[k].lshift) & t[k].mask;
  return c;
}

// splitmix64 finaliser (Steele, Lea, Flood 2014): a bijective 64-bit mixer.
__device__ __host__ __forceinline__ uint64_t mix64(uint64_t x) {
  x ^= x >> 30;
  x *= 0xbf58476d1ce4e5b9ull;
  x ^= x >> 27;
  x *= 0x94d049bb133111ebull;
  x ^= x >> 31;
  return x;
}

// ---------------------------------------------------------------------------
// Lexicographic rank of a permutation of N distinct 4-bit codes 0..N-1.
// rank = sum_i c_i (N-1-i)!, c_i = #{j > i : s_j < s_i} = s_i - #{used codes < s_i}.
// Horner over positions; the first N-12 positions accumulate in `hi` so every
// step stays 32-bit: rank = hi * 12! + lo.  Restates the distinct-symbol case
// of bitmap_rank_component, cuda/permutation_bitmap.cuh:23-49.
template <int N>
__device__ __forceinline__ uint64_t lehmer_rank4(uint64_t w) {
  constexpr int kSplit = N > 12 ? N - 12 : 0;
  const uint32_t lo_word = static_cast<uint32_t>(w), hi_word = static_cast<uint32_t>(w >> 32);
  uint32_t used = 0, hi = 0, lo = 0;
#pragma unroll
  for (int i = 0; i < N - 1; ++i) {
    const uint32_t s = (i < 8 ? (lo_word >> (4 * i)) : (hi_word >> (4 * (i - 8)))) & 15u;
    const uint32_t c = s - __popc(used & ((1u << s) - 1u));
    used |= 1u << s;
    if (i < kSplit) hi = hi * static_cast<uint32_t>(N - i) + c;
    else lo = lo * static_cast<uint32_t>(N - i) + c;
  }
  if (kSplit) return static_cast<uint64_t>(hi) * 479001600ull + lo;
  return lo;
}

// lehmer_rank4<N> split at digit K: *group = the first K digits in mixed radix
// N, N-1, ..., N-K+1 and *inner = the Horner value of the remaining digits, so
// rank = group * (N-K)! + inner.  Needs (N-K)! < 2^32, i.e. N - K <= 12.
template <int N, int K>
__device__ __forceinline__ void lehmer_split4(uint64_t w, uint32_t* group, uint32_t* inner) {
  static_assert(N - K <= 12, "in-group rank must fit 32 bits");
  const uint32_t lo_word = static_cast<uint32_t>(w), hi_word = static_cast<uint32_t>(w >> 32);
  uint32_t used = 0, head = 0, tail = 0;
#pragma unroll
  for (int i = 0; i < N - 1; ++i) {
    const uint32_t s = (i < 8 ? (lo_word >> (4 * i)) : (hi_word >> (4 * (i - 8)))) & 15u;
    const uint32_t c = s - __popc(used & ((1u << s) - 1u));
    used |= 1u << s;
    if (i < K) head = head * static_cast<uint32_t>(N - i) + c;
    else tail = tail * static_cast<uint32_t>(N - i) + c;
  }
  *group = head;
  *inner = tail;
}

// lehmer_split4<N, K> that also returns every Lehmer digit, 4 bits each
// (digit i in bits [4i, 4i+4); the last digit is always 0 and left out).
template <int N, int K>
__device__ __forceinline__ void lehmer_digits_split4(uint64_t w, uint64_t* digits, uint32_t* group, uint32_t* inner) {
  static_assert(N - K <= 12, "in-group rank must fit 32 bits");
  const uint32_t lo_word = static_cast<uint32_t>(w), hi_word = static_cast<uint32_t>(w >> 32);
  uint32_t used = 0, head = 0, tail = 0, dlo = 0, dhi = 0;
#pragma unroll
  for (int i = 0; i < N - 1; ++i) {
    const uint32_t s = (i < 8 ? (lo_word >> (4 * i)) : (hi_word >> (4 * (i - 8)))) & 15u;
    const uint32_t c = s - __popc(used & ((1u << s) - 1u));
    used |= 1u << s;
    if (i < 8) dlo |= c << (4 * i);
    else dhi |= c << (4 * (i - 8));
    if (i < K) head = head * static_cast<uint32_t>(N - i) + c;
    else tail = tail * static_cast<uint32_t>(N - i) + c;
  }
  *digits = (static_cast<uint64_t>(dhi) << 32) | dlo;
  *group = head;
  *inner = tail;
}

// Inverse of lehmer_rank4<N>: factorial-base digits (mixed radix, least
// significant first, all divisors compile-time constants), then the c_i-th
// unused symbol of a sorted nibble list for every position.
template <int N>
__device__ __forceinline__ uint64_t lehmer_unrank4(uint64_t r) {
  constexpr int kSplit = N > 12 ? N - 12 : 0;
  uint32_t digit[N];
  uint32_t hi = kSplit ? static_cast<uint32_t>(r / 479001600ull) : 0u;
  uint32_t lo = kSplit ? static_cast<uint32_t>(r - static_cast<uint64_t>(hi) * 479001600ull) : static_cast<uint32_t>(r);
#pragma unroll
  for (int i = N - 1; i >= kSplit; --i) {
    digit[i] = lo % static_cast<uint32_t>(N - i);
    lo /= static_cast<uint32_t>(N - i);
  }
#pragma unroll
  for (int i = kSplit - 1; i >= 0; --i) {
    digit[i] = hi % static_cast<uint32_t>(N - i);
    hi /= static_cast<uint32_t>(N - i);
  }
  uint64_t avail = 0xfedcba9876543210ull;  // symbols still unused, ascending
  uint64_t out = 0;
#pragma unroll
  for (int i = 0; i < N; ++i) {
    // symbol = nibble c of the list; delete it: the nibbles above c move down
    // one place, the c nibbles below stay (bit-field insert of the low 4c bits).
    const uint32_t sh = 4 * digit[i];
    uint64_t sym, rest;
    asm("bfe.u64 %0, %1, %2, 4;" : "=l"(sym) : "l"(avail), "r"(sh));
    asm("bfi.b64 %0, %1, %2, 0, %3;" : "=l"(rest) : "l"(avail), "l"(avail >> 4), "r"(sh));
    out |= sym << (4 * i);
    avail = rest;
  }
  return out;
}

// Runtime-N variant for tests and rarely used sizes.
__device__ __forceinline__ uint64_t lehmer_rank4_n(uint64_t w, uint32_t n) {
  uint64_t rank = 0;
  uint32_t used = 0;
  for (uint32_t i = 0; i + 1 < n; ++i) {
    const uint32_t s = static_cast<uint32_t>(w >> (4 * i)) & 15u;
    const uint32_t c = s - __popc(used & ((1u << s) - 1u));
    used |= 1u << s;
    rank = rank * (n - i) + c;
  }
  return rank;
}

// Exact lexicographic rank of a multiset permutation (repeated labels), the
// general case of cuda/permutation_bitmap.cuh:23-49 and of
// MultisetDomain::rank, crates/mgbfs-runtime/src/permutation_bitmap.rs:36-45.
// Codes are b-bit (b = 4 or 8), counts[c] = multiplicity of code c, and
// total = n! / prod(counts!).  floor(ways*f/r) is evaluated without overflow as
// (ways/r)*f + ((ways%r)*f)/r.
struct MultisetDomain {
  uint32_t n, bits, distinct, pad;
  unsigned long long total;
  uint32_t counts[16];
};

__device__ __forceinline__ uint64_t scale_floor(uint64_t ways, uint32_t f, uint32_t r) {
  return (ways / r) * f + ((ways % r) * f) / r;
}

__device__ __forceinline__ bool multiset_rank(uint64_t w, const MultisetDomain& d, uint64_t* out) {
  // Byte-lane counts: lane c of (c_lo, c_hi) holds counts[c] (<= 16).
  uint64_t c_lo = 0, c_hi = 0;
  for (uint32_t c = 0; c < d.distinct; ++c) {
    if (c < 8) c_lo |= static_cast<uint64_t>(d.counts[c]) << (8 * c);
    else c_hi |= static_cast<uint64_t>(d.counts[c]) << (8 * (c - 8));
  }
  const uint64_t sym_mask = (1ull << d.bits) - 1;
  uint64_t ways = d.total, rank = 0;
  for (uint32_t e = 0; e < d.n; ++e) {
    const uint32_t s = static_cast<uint32_t>((w >> (d.bits * e)) & sym_mask);
    if (s >= d.distinct) return false;
    const uint32_t cnt = s < 8 ? static_cast<uint32_t>((c_lo >> (8 * s)) & 0xff)
                               : static_cast<uint32_t>((c_hi >> (8 * (s - 8))) & 0xff);
    if (!cnt) return false;
    // less = sum of counts of codes below s (horizontal byte sum of the masked lanes)
    uint64_t below_lo = s >= 8 ? c_lo : (c_lo & ((1ull << (8 * s)) - 1));
    uint64_t below_hi = s <= 8 ? 0 : (c_hi & ((1ull << (8 * (s - 8))) - 1));
    const uint32_t less = static_cast<uint32_t>(((below_lo * 0x0101010101010101ull) >> 56) +
                                                ((below_hi * 0x0101010101010101ull) >> 56));
    const uint32_t remaining = d.n - e;
    rank += scale_floor(ways, less, remaining);
    ways = scale_floor(ways, cnt, remaining);
    if (s < 8) c_lo -= 1ull << (8 * s);
    else c_hi -= 1ull << (8 * (s - 8));
  }
  if (rank >= d.total || ways != 1) return false;
  *out = rank;
  return true;
}

// ---------------------------------------------------------------------------
// Open-addressing set of packed one-word keys with exact key equality.  Slots
// hold the key itself (kEmpty = free); an insert is one CAS on the key, so no
// pending state, row arena or regeneration is needed (the reference's
// accept_candidates, cuda/generic_visited.cu:18-58, CASes a hash-prefix/row
// token and compares states element by element).
// `tag` occupies bits above `key_mask` (the BFS depth), ignored by equality.
__device__ __forceinline__ int hash_insert(unsigned long long* table, uint64_t mask, uint64_t key,
                                           uint64_t key_mask, uint64_t tag, uint32_t probe_limit) {
  uint64_t slot = mix64(key) & mask;
  for (uint32_t probe = 0; probe < probe_limit; ++probe) {
    // Read first: a key that is already present (about half of all tests on
    // inverse-closed graphs) costs a load, not an atomic.
    unsigned long long cur = *reinterpret_cast<volatile unsigned long long*>(&table[slot]);
    if (cur == kEmpty) {
      const unsigned long long prev = atomicCAS(&table[slot], kEmpty, key | tag);
      if (prev == kEmpty) return 1;  // inserted
      cur = prev;
    }
    if ((cur & key_mask) == key) return 0;  // present
    slot = (slot + 1) & mask;
  }
  return -1;  // probe limit
}

__device__ __forceinline__ bool hash_contains(const unsigned long long* table, uint64_t mask, uint64_t key,
                                              uint64_t key_mask) {
  if (!table) return false;
  uint64_t slot = mix64(key) & mask;
  for (uint64_t probe = 0; probe <= mask; ++probe) {
    const unsigned long long cur = __ldg(&table[slot]);
    if (cur == kEmpty) return false;
    if ((cur & key_mask) == key) return true;
    slot = (slot + 1) & mask;
  }
  return false;
}

__device__ __forceinline__ uint32_t lane_id() {
  uint32_t lane;
  asm volatile("mov.u32 %0, %%laneid;" : "=r"(lane));
  return lane;
}

__device__ __forceinline__ uint32_t lanemask_lt() {
  uint32_t mask;
  asm volatile("mov.u32 %0, %%lanemask_lt;" : "=r"(mask));
  return mask;
}

// L2 eviction priority for the bitmap words a layer keeps hitting: an
// evict-last access policy (PTX createpolicy) attached to the atomicOr, so the
// streaming frontier traffic is evicted before the hot bitmap lines.
__device__ __forceinline__ unsigned long long l2_policy_evict_last() {
  unsigned long long policy;
  asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(policy));
  return policy;
}

__device__ __forceinline__ unsigned int atomic_or_hinted32(unsigned int* address, unsigned int bits,
                                                           unsigned long long policy) {
  unsigned int old;
  asm volatile("atom.global.or.L2::cache_hint.b32 %0, [%1], %2, %3;"
               : "=r"(old)
               : "l"(address), "r"(bits), "l"(policy)
               : "memory");
  return old;
}

__device__ __forceinline__ unsigned long long atomic_or_hinted(unsigned long long* address, unsigned long long bits,
                                                               unsigned long long policy) {
  unsigned long long old;
  asm volatile("atom.global.or.L2::cache_hint.b64 %0, [%1], %2, %3;"
               : "=l"(old)
               : "l"(address), "l"(bits), "l"(policy)
               : "memory");
  return old;
}

}  // namespace mgbfs2
