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
  ERR_BAD_REFERENCE = 1u << 7,      // a routed state reached a rank that does not own it
};

constexpr uint32_t kFullMask = 0xffffffffu;

__host__ __device__ constexpr uint64_t factorial_u64(int m) {
  return m <= 1 ? 1ull : static_cast<uint64_t>(m) * factorial_u64(m - 1);
}
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

// A grid barrier waits for the slowest block to finish its share of a layer,
// so its bound is device time, not a poll count: 30 s of %globaltimer, two
// orders of magnitude above the longest layer of the workloads here (the
// largest fused S13 layer takes about 60 ms; a block's wait is at most one
// layer).  The poll cap is a second bound that holds even if the timer were
// to stop.
constexpr unsigned long long kBarrierWaitNs = 30ull * 1000 * 1000 * 1000;
constexpr uint32_t kBarrierPolls = 1u << 30;

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long now;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(now));
  return now;
}

// Grid-wide barrier of a cooperative launch, with a bounded wait.  Thread 0
// of each block arrives on *count; the last to arrive resets it and advances
// *gen with a release store; the others poll *gen with acquire loads until
// kBarrierWaitNs have passed (or kBarrierPolls polls), after which they raise
// ERR_WAIT_LIMIT in *error and return false (the caller then ends the kernel:
// nothing waits forever).  Every thread orders its later loads after the
// barrier.  *count and *gen start at zero for each launch.
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
      const unsigned long long started = global_ns();
      for (uint32_t polls = 0;; ++polls) {
        unsigned int now;
        asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(now) : "l"(gen) : "memory");
        if (now != g) break;
        if (polls >= kBarrierPolls || ((polls & 255u) == 255u && global_ns() - started > kBarrierWaitNs)) {
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

// The rank over byte-lane counts: lane c of (c_lo, c_hi) holds the
// multiplicity of code c (<= 16); codes of multiplicity 0 may appear in the
// alphabet and never in the state.
__device__ __forceinline__ bool multiset_rank_lanes(uint64_t w, uint32_t n, uint32_t bits, uint32_t distinct,
                                                    uint64_t total, uint64_t c_lo, uint64_t c_hi, uint64_t* out) {
  const uint64_t sym_mask = (1ull << bits) - 1;
  uint64_t ways = total, rank = 0;
  for (uint32_t e = 0; e < n; ++e) {
    const uint32_t s = static_cast<uint32_t>((w >> (bits * e)) & sym_mask);
    if (s >= distinct) return false;
    const uint32_t cnt = s < 8 ? static_cast<uint32_t>((c_lo >> (8 * s)) & 0xff)
                               : static_cast<uint32_t>((c_hi >> (8 * (s - 8))) & 0xff);
    if (!cnt) return false;
    // less = sum of counts of codes below s (horizontal byte sum of the masked lanes)
    uint64_t below_lo = s >= 8 ? c_lo : (c_lo & ((1ull << (8 * s)) - 1));
    uint64_t below_hi = s <= 8 ? 0 : (c_hi & ((1ull << (8 * (s - 8))) - 1));
    const uint32_t less = static_cast<uint32_t>(((below_lo * 0x0101010101010101ull) >> 56) +
                                                ((below_hi * 0x0101010101010101ull) >> 56));
    const uint32_t remaining = n - e;
    rank += scale_floor(ways, less, remaining);
    ways = scale_floor(ways, cnt, remaining);
    if (s < 8) c_lo -= 1ull << (8 * s);
    else c_hi -= 1ull << (8 * (s - 8));
  }
  if (rank >= total || ways != 1) return false;
  *out = rank;
  return true;
}

__device__ __forceinline__ bool multiset_rank(uint64_t w, const MultisetDomain& d, uint64_t* out) {
  uint64_t c_lo = 0, c_hi = 0;
  for (uint32_t c = 0; c < d.distinct; ++c) {
    if (c < 8) c_lo |= static_cast<uint64_t>(d.counts[c]) << (8 * c);
    else c_hi |= static_cast<uint64_t>(d.counts[c]) << (8 * (c - 8));
  }
  return multiset_rank_lanes(w, d.n, d.bits, d.distinct, d.total, c_lo, c_hi, out);
}

// Product of multiset domains over position components: the positions that
// the generators connect (i ~ g[i]) form components, each keeping its own
// multiset of labels, so the reachable states lie in the product of the
// components' multiset permutations.  The rank is mixed-radix over the
// components in order of their first position, each digit the multiset rank
// of the component's codes in position order (the contract of
// cuda/permutation_bitmap.cuh:62-83 and PositionOrbitDomain,
// crates/mgbfs-runtime/src/permutation_bitmap.rs:61-143).
constexpr uint32_t kMaxComponents = 16;
// The visited structure of a packed plan.  V_HASHQ: the all-visited set as
// a quotient table of 32-bit slots.  V_PRODUCT: a bitmap over the product of
// the position components' multiset domains.
enum VisitKind : int { V_LEHMER = 0, V_MULTISET = 1, V_HASH = 2, V_HASH3 = 3, V_HASHQ = 4, V_PRODUCT = 5, V_RADIX = 6 };

// Visited kinds kept as a bitmap over a rank domain.
__host__ __device__ constexpr bool bitmap_kind(int v) {
  return v == V_LEHMER || v == V_MULTISET || v == V_PRODUCT || v == V_RADIX;
}

// ---------------------------------------------------------------------------
// Packed modular matrices: a rows x cols state of entries in [0, mod), entry
// j = i * cols + c in bits [bits * j, bits * (j + 1)) of one word, so row i is
// the contiguous field of cols * bits bits at i * cols * bits.  Generator g's
// program (terms [tb, te)) lists, output row by output row, either one copy
// term (the matrix row is a unit vector: the source row moves unchanged) or
// the row's nonzero coefficients reduced mod m; rows with no term are zero.
// Term fields: mask = coefficient, rshift = source row, lshift = output row
// with kMatrixCopy set for a copy.  The host packs a graph only when no
// partial sum can leave int64, so the result equals the reference's
// wrap-then-modulus (graph_definition.py:77-83), and every coefficient being
// reduced keeps the sums non-negative.
// The bitmap rank is the mixed-radix number of the entries, sum e_j * mod^j,
// over the whole canonical entry space (the reference's certified bound,
// workload_geometry.py:21-36).
constexpr uint32_t kMatrixCopy = 1u << 31;
// Template N of the fused, route and count kernels for packed matrices: the
// action is compiled in, so permutation kernels carry none of its code.
constexpr int kMatrixN = -1;
constexpr uint32_t kMatrixMaxCols = 4;

struct MatrixAction {
  uint32_t rows, cols, bits, mod;  // mod = 0: permutation terms instead
  uint32_t recip;                  // floor(2^32 / mod): Barrett reduction of 32-bit sums
  uint32_t pad;
};

// x mod m.  Below 2^32 by Barrett's method (P. Barrett, CRYPTO 1986): with
// R = floor(2^32 / m), q = floor(x * R / 2^32) is floor(x / m) or one less, so
// one conditional subtraction finishes; larger sums take the 64-bit remainder.
__device__ __forceinline__ uint64_t matrix_reduce(uint64_t x, const MatrixAction& a) {
  if (x >> 32) return x % a.mod;
  const uint32_t x32 = static_cast<uint32_t>(x);
  uint32_t r = x32 - __umulhi(x32, a.recip) * a.mod;
  if (r >= a.mod) r -= a.mod;
  return r;
}

__device__ __forceinline__ uint64_t apply_matrix(const MatrixAction& a, uint64_t s, const Term* t, uint32_t tb,
                                                 uint32_t te) {
  const uint32_t row_bits = a.bits * a.cols;
  const uint64_t row_mask = row_bits >= 64 ? ~0ull : ((1ull << row_bits) - 1);
  const uint64_t field = (1ull << a.bits) - 1;
  uint64_t child = 0;
  for (uint32_t j = tb; j < te;) {
    const uint32_t out = t[j].lshift;
    if (out & kMatrixCopy) {
      child |= ((s >> (row_bits * t[j].rshift)) & row_mask) << (row_bits * (out & ~kMatrixCopy));
      ++j;
      continue;
    }
    uint64_t acc[kMatrixMaxCols];
#pragma unroll
    for (uint32_t c = 0; c < kMatrixMaxCols; ++c) acc[c] = 0;
    for (; j < te && t[j].lshift == out; ++j) {
      const uint64_t coef = t[j].mask;
      const uint64_t src = s >> (row_bits * t[j].rshift);
#pragma unroll
      for (uint32_t c = 0; c < kMatrixMaxCols; ++c)
        if (c < a.cols) acc[c] += coef * ((src >> (a.bits * c)) & field);
    }
#pragma unroll
    for (uint32_t c = 0; c < kMatrixMaxCols; ++c)
      if (c < a.cols) child |= matrix_reduce(acc[c], a) << (row_bits * out + a.bits * c);
  }
  return child;
}

__device__ __forceinline__ uint64_t radix_rank(uint64_t s, const MatrixAction& a) {
  const uint64_t field = (1ull << a.bits) - 1;
  const uint32_t n = a.rows * a.cols;
  uint64_t r = 0;
  for (uint32_t j = n; j-- > 0;) r = r * a.mod + ((s >> (a.bits * j)) & field);
  return r;
}

struct ProductDomain {
  uint32_t components, bits, distinct, pad;
  unsigned long long total;
  unsigned long long positions[kMaxComponents];  // 4-bit position indices, the first in the low nibble
  unsigned long long radix[kMaxComponents];      // multiset permutations of each component
  unsigned long long lanes[kMaxComponents][2];   // byte-lane label counts of each component
  uint32_t length[kMaxComponents];
};

__device__ __forceinline__ bool product_rank(uint64_t w, const ProductDomain& d, uint64_t* out) {
  const uint64_t sym_mask = (1ull << d.bits) - 1;
  uint64_t rank = 0;
  for (uint32_t c = 0; c < d.components; ++c) {
    const uint32_t len = d.length[c];
    const uint64_t pos = d.positions[c];
    uint64_t compact = 0;
    for (uint32_t j = 0; j < len; ++j) {
      const uint32_t at = static_cast<uint32_t>(pos >> (4 * j)) & 15u;
      compact |= ((w >> (d.bits * at)) & sym_mask) << (d.bits * j);
    }
    uint64_t digit = 0;
    if (!multiset_rank_lanes(compact, len, d.bits, d.distinct, d.radix[c], d.lanes[c][0], d.lanes[c][1], &digit))
      return false;
    rank = rank * d.radix[c] + digit;
  }
  if (rank >= d.total) return false;
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

// ---------------------------------------------------------------------------
// Quotient set of packed keys in 32-bit slots.  A key of B bits is first
// mixed by a bijection of the B-bit integers (xorshift-multiply rounds, the
// construction of MurmurHash3's 64-bit finaliser restricted to B bits: every
// round is invertible modulo 2^B).  The low s bits of the mixed value x pick
// the home slot of a table of 2^s slots; the slot stores the other B - s bits
// of x together with the probe distance j + 1 in its low D = 32 - (B - s)
// bits (0 = empty).  Slot t then holds the key whose mixed value is
// (stored >> D) << s | (t - j), so equality is exact and a table of 40 M
// 44-bit keys takes 4 bytes per slot instead of 8.  Slots only ever go from
// empty to a key, so a stale read is harmless: an empty read is settled by the
// CAS, and a key read stays that key.
__device__ __host__ __forceinline__ uint64_t mix_bits(uint64_t k, uint32_t bits) {
  const uint64_t m = bits >= 64 ? ~0ull : ((1ull << bits) - 1);
  const uint32_t h = (bits + 1) / 2;
  uint64_t x = k & m;
  x ^= x >> h;
  x = (x * 0xff51afd7ed558ccdull) & m;
  x ^= x >> h;
  x = (x * 0xc4ceb9fe1a85ec53ull) & m;
  x ^= x >> h;
  return x;
}

struct QuotientSlots {
  unsigned int* slots;
  uint64_t mask;        // 2^s - 1
  uint32_t s, bits, d;  // log2 slots, key bits B, distance bits D = 32 - (B - s)
  uint32_t limit;       // probe limit, < 2^D - 1
};

__device__ __forceinline__ unsigned int load_slot(const unsigned int* slot) {
  unsigned int v;
  asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(slot) : "memory");
  return v;
}

// First probe of `key`: the home slot's current value.
__device__ __forceinline__ unsigned int qhash_first(const QuotientSlots& q, uint64_t key) {
  return load_slot(q.slots + (mix_bits(key, q.bits) & q.mask));
}

// Insert `key`, given the home slot's value read before (`v`).  Returns 1 if
// inserted, 0 if present, -1 at the probe limit.
__device__ __forceinline__ int qhash_resolve(const QuotientSlots& q, uint64_t key, unsigned int v) {
  const uint64_t x = mix_bits(key, q.bits);
  const uint64_t home = x & q.mask, rem = x >> q.s;
  for (uint32_t j = 0; j < q.limit; ++j) {
    const unsigned int want = static_cast<unsigned int>((rem << q.d) | (j + 1));
    unsigned int* slot = q.slots + ((home + j) & q.mask);
    if (j) v = load_slot(slot);
    if (v == 0u) {
      const unsigned int prev = atomicCAS(slot, 0u, want);
      if (prev == 0u) return 1;
      v = prev;
    }
    if (v == want) return 0;
  }
  return -1;
}

__device__ __forceinline__ int qhash_insert(const QuotientSlots& q, uint64_t key) {
  return qhash_resolve(q, key, qhash_first(q, key));
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

// Generators from which the grouped layers' claims test before they set
// (claim_bit32): with g generators about (g - 2) / (g - 1) of an inverse-
// closed graph's tests find a visited state, and a work item's children fall
// into a few 454 KB group slices, so the load often hits L1.  Measured on the
// B200: S13 Coxeter (12 generators) 544 -> 414 ms, S13 LRX (3) 145 -> 150 ms.
// The fused and batched layers scatter their claims over the whole bitmap;
// there the load lost (S10 Coxeter 1.15 -> 1.39 ms, S12 planner instances
// 2.41 -> 2.81 s), so they keep the plain atomic.
constexpr uint32_t kTestFirstGens = 5;

// Test, then set: a bit that a plain load sees set is set for good (a run
// only ever sets bits, and a launch starts with no stale L1 lines), so only a
// bit seen clear costs an L2 atomic.  True when this call set it.
__device__ __forceinline__ bool claim_bit32(unsigned int* word, unsigned int bit, unsigned long long policy) {
  if (*word & bit) return false;
  return !(atomic_or_hinted32(word, bit, policy) & bit);
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
