// Fused layer-expansion kernels of the packed (one-word state) path.
//
// One launch expands a whole frontier layer: parent load (128-bit, coalesced)
// -> generator application in registers -> visited test-and-set -> block
// compaction of the winners in shared memory -> one global reservation per
// tile -> coalesced append to the next frontier.  The reference splits the
// same work over accept_candidates (cuda/generic_visited.cu:18-58) for the
// hash and bitmap_route + bitmap_accept[_grouped] (cuda/permutation_bitmap.cu:
// 27-48, 105-205) for the bitmap, with one global atomicAdd per appended row.
#pragma once
#include "device.cuh"
#include "sort_tiles.cuh"

namespace mgbfs2 {


constexpr uint32_t kOutCap = 4096;  // shared-memory winners per block (32 KiB)
// Layers of at most this many (parent, generator) candidates per thread of the
// grid run candidate-parallel in the expand_packed<..., CAND = true> kernels
// (measured: 4 waves beat 1 and 2 on S10 Coxeter and S11 LRX hash).  The
// mode's code is compiled only where the host selects it: present in a kernel
// it slowed the parent path of the Lehmer kernels (S12 LRX 17.2 -> 22.3 ms).
constexpr unsigned long long kCandidateWaves = 4;
// The quotient-hash kernel runs six blocks per SM (its registers allow six)
// with a 16 KB stage, so that 6 x 17 KB stays in the 132 KB shared-memory
// configuration and leaves about 100 KB of L1 (a 32 KB stage pushed it to the
// 228 KB configuration, and the BFS ran 1.3x slower).
constexpr uint32_t kOutCapHashQ = 2048;
constexpr int kHashQBlocksPerSM = 6;
constexpr uint32_t kBlock = 256;
constexpr int kPackedBlocksPerSM = 4;  // resident expand_packed blocks: the 164 KB configuration, 92 KB left as L1

// Device-resident layer loop: the frontier size, which of the two buffers
// holds it, and the loop's stop reason live on the device, so one persistent
// cooperative launch (or, as the fallback, one CUDA graph with a WHILE node)
// runs a whole BFS without host round trips.
struct LoopState {
  unsigned long long count, visited, capacity;
  unsigned long long* buf[2];
  uint32_t parity, depth, max_entries, stop;  // stop: 0 running, 1 exhausted, 2 error, 3 table full of layers
  unsigned long long* layers;  // max_entries layer sizes
  unsigned long long* stamps;  // max_entries globaltimer readings (stamp d = end of layer d)
  uint32_t bar_count, bar_gen; // grid barrier of the persistent form (zero at launch)
  // All-visited hash sized below the state bound (learned plan): the loop
  // pauses (stop 3) before a layer that could take the table past this many
  // states, and the host loop grows it.  0 = the table holds every state.
  unsigned long long table_limit;
  uint32_t gens, pad;
};

struct ExpandParams {
  const unsigned long long* frontier;
  unsigned long long count;
  unsigned long long* next;
  unsigned long long capacity;
  const Term* terms;
  const uint32_t* term_begin;  // gens + 1 entries, followed by inverse[gens]
  uint32_t gens, total_terms;
  // Parent-edge tags (inverse-closed graphs): a frontier word carries
  // (g + 1) << gen_shift for the generator g that produced it; generator
  // inverse[g] applied to it returns to the previous layer and is skipped.
  // gen_shift = 0 disables tagging.
  uint32_t gen_shift;
  uint32_t persistent;  // with `loop`: one cooperative launch runs every layer (grid barriers between)
  Control* control;
  unsigned long long* bitmap;
  MultisetDomain ms;
  unsigned long long* table;  // insert table (all-visited table, or bank of layer d+1)
  unsigned long long table_mask, key_mask, tag;
  uint32_t probe_limit, ppt;
  const unsigned long long* look0;  // three-bank lookups: layer d and layer d-1
  unsigned long long look0_mask;
  const unsigned long long* look1;
  unsigned long long look1_mask;
  LoopState* loop;  // graph mode: count and buffers from here instead of frontier/count/next
  QuotientSlots q;  // V_HASHQ table
  ProductDomain pd;  // V_PRODUCT rank domain
  MatrixAction mat;  // packed modular matrices (mat.mod != 0); V_RADIX rank domain
};

// The child of packed state s under generator g (terms [tb, te) of the
// program): permutation displacement terms, or (N = kMatrixN) a modular
// matrix product.
template <int N>
__device__ __forceinline__ uint64_t apply_action(const ExpandParams& p, uint64_t s, const Term* terms, uint32_t tb,
                                                 uint32_t te) {
  if constexpr (N == kMatrixN) {
    return apply_matrix(p.mat, s, terms, tb, te);
  } else {
    return apply_terms(s, terms, tb, te);
  }
}

// Visited test-and-set of candidate c.  Must be reached by all 32 lanes (the
// warp-aggregated bitmap path uses warp collectives); `valid` masks lanes
// without a candidate.
template <int V, int N, bool WARP>
__device__ __forceinline__ bool claim(const ExpandParams& p, uint64_t c, bool valid) {
  if constexpr (bitmap_kind(V)) {
    uint64_t r = 0;
    bool ok = valid;
    if (valid) {
      if constexpr (V == V_LEHMER) {
        r = lehmer_rank4<N>(c);
      } else if constexpr (V == V_RADIX) {
        r = radix_rank(c, p.mat);
      } else if constexpr (V == V_PRODUCT) {
        ok = product_rank(c, p.pd, &r);
        if (!ok) raise_error(&p.control->error, ERR_RANK_RANGE);
      } else {
        ok = multiset_rank(c, p.ms, &r);
        if (!ok) raise_error(&p.control->error, ERR_RANK_RANGE);
      }
    }
    if constexpr (WARP) {
      // Lanes whose ranks share a bitmap word merge their bits into one
      // atomicOr; among lanes with the same rank only the lowest may win.
      const unsigned active = __ballot_sync(kFullMask, ok);
      bool won = false;
      if (ok) {
        const unsigned long long word = r >> 6;
        const unsigned peers = __match_any_sync(active, word);
        const unsigned same = __match_any_sync(peers, static_cast<unsigned long long>(r));
        const unsigned long long bit = 1ull << (r & 63);
        const unsigned lo = __reduce_or_sync(peers, static_cast<unsigned>(bit));
        const unsigned hi = __reduce_or_sync(peers, static_cast<unsigned>(bit >> 32));
        const int leader = __ffs(peers) - 1;
        const int lane = static_cast<int>(lane_id());
        unsigned long long old = 0;
        if (lane == leader) old = atomicOr(&p.bitmap[word], (static_cast<unsigned long long>(hi) << 32) | lo);
        old = __shfl_sync(peers, old, leader);
        won = (lane == __ffs(same) - 1) && !(old & bit);
      }
      return won;
    } else {
      if (!ok) return false;
      const unsigned long long bit = 1ull << (r & 63);
      return !(atomicOr(&p.bitmap[r >> 6], bit) & bit);
    }
  } else if constexpr (V == V_HASH) {
    if (!valid) return false;
    const int rc = hash_insert(p.table, p.table_mask, c, p.key_mask, p.tag, p.probe_limit);
    if (rc < 0) raise_error(&p.control->error, ERR_TABLE_FULL);
    return rc == 1;
  } else if constexpr (V == V_HASHQ) {
    if (!valid) return false;
    const int rc = qhash_insert(p.q, c);
    if (rc < 0) raise_error(&p.control->error, ERR_TABLE_FULL);
    return rc == 1;
  } else {
    if (!valid) return false;
    // Inverse-closed graphs: every neighbour of layer d lies in d-1, d or d+1.
    if (hash_contains(p.look0, p.look0_mask, c, p.key_mask) || hash_contains(p.look1, p.look1_mask, c, p.key_mask))
      return false;
    const int rc = hash_insert(p.table, p.table_mask, c, p.key_mask, 0, p.probe_limit);
    if (rc < 0) raise_error(&p.control->error, ERR_TABLE_FULL);
    return rc == 1;
  }
}

// Append the block's shared-memory winners to the next frontier with one
// global reservation.  Called by all threads of the block.
__device__ __forceinline__ void flush_block(const ExpandParams& p, unsigned long long* next, unsigned long long* out,
                                            uint32_t* out_count, unsigned long long* out_base) {
  __syncthreads();
  const uint32_t n = *out_count;
  if (threadIdx.x == 0 && n) *out_base = atomicAdd(&p.control->next_count, static_cast<unsigned long long>(n));
  __syncthreads();
  const unsigned long long base = *out_base;
  bool overflow = false;
  for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) {
    const unsigned long long pos = base + i;
    if (pos < p.capacity) next[pos] = out[i];
    else overflow = true;
  }
  if (overflow) raise_error(&p.control->error, ERR_FRONTIER_OVERFLOW);
  __syncthreads();
  if (threadIdx.x == 0) *out_count = 0;
  __syncthreads();
}

// Graph mode, after each expansion: record the new layer, stop on an empty
// layer, a device error or a full layer table, else make the new layer the
// frontier.  Returns the stop reason (0 = go on).  layers/stamps hold
// max_entries sizes and globaltimer readings (stamp d = end of layer d).
__device__ __forceinline__ uint32_t loop_step(LoopState* s, Control* c) {
  unsigned long long now;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(now));
  const unsigned long long produced = c->next_count;
  uint32_t stop = 0;
  if (c->error || produced > s->capacity) {
    stop = 2;
  } else if (produced == 0) {
    stop = 1;
  } else {
    const uint32_t d = s->depth + 1;
    s->layers[d] = produced;
    s->stamps[d] = now;
    s->count = produced;
    s->visited += produced;
    s->parity ^= 1u;
    s->depth = d;
    c->next_count = 0;
    if (d + 1 >= s->max_entries) stop = 3;
    if (s->table_limit && s->visited + produced * s->gens > s->table_limit) stop = 3;
  }
  s->stop = stop;
  return stop;
}

template <int V, int N, bool WARP, bool CAND>
__global__ void __launch_bounds__(kBlock, V == V_HASHQ ? kHashQBlocksPerSM : 1) expand_packed(ExpandParams p) {
  constexpr uint32_t out_cap = V == V_HASHQ ? kOutCapHashQ : kOutCap;
  extern __shared__ __align__(16) unsigned char program_smem[];
  __shared__ unsigned long long out[out_cap];
  __shared__ uint32_t out_count;
  __shared__ unsigned long long out_base;
  Term* terms = reinterpret_cast<Term*>(program_smem);
  uint32_t* begin = reinterpret_cast<uint32_t*>(program_smem + p.total_terms * sizeof(Term));
  const uint32_t* inverse = begin + p.gens + 1;
  for (uint32_t i = threadIdx.x; i < p.total_terms; i += blockDim.x) terms[i] = p.terms[i];
  for (uint32_t i = threadIdx.x; i <= 2 * p.gens; i += blockDim.x) begin[i] = p.term_begin[i];
  if (threadIdx.x == 0) out_count = 0;
  __syncthreads();

  for (;;) {
    unsigned long long count = p.count;
    const unsigned long long* frontier = p.frontier;
    unsigned long long* next = p.next;
    if (p.loop) {
      count = p.loop->count;
      const uint32_t parity = p.loop->parity;
      frontier = p.loop->buf[parity];
      next = p.loop->buf[parity ^ 1u];
    }
    const uint32_t lane = lane_id();
    const uint32_t tile = blockDim.x * p.ppt;
    const unsigned long long tiles = (count + tile - 1) / tile;
    // When a whole tile's winners fit the stage (tile x generators), the
    // block flushes once per tile and skips the room check (two barriers)
    // after every generator.
    const bool one_flush = tile * p.gens <= out_cap;
    // A small layer runs one thread per (parent, generator) candidate
    // instead (CAND kernels), so its generators are tested in parallel rather
    // than one after another by each thread: at most kCandidateWaves
    // candidates per thread of the grid (uniform across the grid; counted in
    // 32 bits).
    const bool by_candidate =
        CAND && count * p.gens <= kCandidateWaves * static_cast<unsigned long long>(gridDim.x) * blockDim.x;
    if (by_candidate) {
      const uint32_t candidates = static_cast<uint32_t>(count * p.gens);
      const uint32_t ctiles = (candidates + blockDim.x - 1) / blockDim.x;
      for (uint32_t t = blockIdx.x; t < ctiles; t += gridDim.x) {
        const uint32_t q = t * blockDim.x + threadIdx.x;
        bool v = q < candidates;
        uint64_t c = 0;
        unsigned long long gtag = 0;
        if (v) {
          const uint32_t pi = q / p.gens, g = q - pi * p.gens;
          const uint64_t par = frontier[pi];
          const uint32_t tag = p.gen_shift ? static_cast<uint32_t>(par >> p.gen_shift) : 0u;
          if (tag && inverse[tag - 1] == g) {
            v = false;
          } else {
            c = apply_action<N>(p, par, terms, begin[g], begin[g + 1]);
            gtag = p.gen_shift ? static_cast<unsigned long long>(g + 1) << p.gen_shift : 0ull;
          }
        }
        bool won;
        if constexpr (V == V_HASHQ) {
          won = false;
          if (v) {
            const int rc = qhash_insert(p.q, c);
            if (rc < 0) raise_error(&p.control->error, ERR_TABLE_FULL);
            won = rc == 1;
          }
        } else {
          won = claim<V, N, WARP>(p, c, v);
        }
        const unsigned m = __ballot_sync(kFullMask, won);
        if (m) {
          const int leader = __ffs(m) - 1;
          uint32_t wb = 0;
          if (static_cast<int>(lane) == leader) wb = atomicAdd(&out_count, static_cast<uint32_t>(__popc(m)));
          wb = __shfl_sync(kFullMask, wb, leader);
          if (won) out[wb + __popc(m & lanemask_lt())] = c | gtag;
        }
        flush_block(p, next, out, &out_count, &out_base);
      }
    }
    for (unsigned long long t = by_candidate ? tiles : blockIdx.x; t < tiles; t += gridDim.x) {
      const unsigned long long base = t * tile;
      uint64_t par[4];
      bool val[4];
  #pragma unroll
      for (int j = 0; j < 2; ++j) {
        par[2 * j] = par[2 * j + 1] = 0;
        val[2 * j] = val[2 * j + 1] = false;
        if (p.ppt == 1) {
          // One parent per thread: parent base + tid (the pair loads below
          // would cover two tiles' worth of positions).
          const unsigned long long i0 = base + threadIdx.x;
          if (j == 0 && i0 < count) {
            par[0] = frontier[i0];
            val[0] = true;
          }
        } else if (2 * j < static_cast<int>(p.ppt)) {
          const unsigned long long i0 = base + 2ull * (j * blockDim.x + threadIdx.x);
          if (i0 + 1 < count) {
            const ulonglong2 v = *reinterpret_cast<const ulonglong2*>(frontier + i0);
            par[2 * j] = v.x;
            par[2 * j + 1] = v.y;
            val[2 * j] = val[2 * j + 1] = true;
          } else if (i0 < count) {
            par[2 * j] = frontier[i0];
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
      for (uint32_t g = 0; g < p.gens; ++g) {
        const uint32_t tb = begin[g], te = begin[g + 1];
        const unsigned long long gtag = p.gen_shift ? static_cast<unsigned long long>(g + 1) << p.gen_shift : 0ull;
        if constexpr (V == V_HASHQ) {
          // The home-slot reads of all this thread's children of generator g
          // are issued before any is resolved, so up to four table misses
          // are in flight per thread instead of one.
          uint64_t ch[4];
          unsigned int first[4];
          bool live[4];
  #pragma unroll
          for (int k = 0; k < 4; ++k) {
            live[k] = k < static_cast<int>(p.ppt) && val[k] && g != skip[k];
            ch[k] = live[k] ? apply_action<N>(p, par[k], terms, tb, te) : 0;
            first[k] = live[k] ? qhash_first(p.q, ch[k]) : 0u;
          }
  #pragma unroll
          for (int k = 0; k < 4; ++k) {
            if (k >= static_cast<int>(p.ppt)) break;
            bool won = false;
            if (live[k]) {
              const int rc = qhash_resolve(p.q, ch[k], first[k]);
              if (rc < 0) raise_error(&p.control->error, ERR_TABLE_FULL);
              won = rc == 1;
            }
            const unsigned m = __ballot_sync(kFullMask, won);
            if (m) {
              const int leader = __ffs(m) - 1;
              uint32_t wb = 0;
              if (static_cast<int>(lane) == leader) wb = atomicAdd(&out_count, static_cast<uint32_t>(__popc(m)));
              wb = __shfl_sync(kFullMask, wb, leader);
              if (won) out[wb + __popc(m & lanemask_lt())] = ch[k] | gtag;
            }
          }
        } else {
  #pragma unroll
          for (int k = 0; k < 4; ++k) {
            if (k >= static_cast<int>(p.ppt)) break;
            const bool v = val[k] && g != skip[k];
            const uint64_t c = v ? apply_action<N>(p, par[k], terms, tb, te) : 0;
            const bool won = claim<V, N, WARP>(p, c, v);
            const unsigned m = __ballot_sync(kFullMask, won);
            if (m) {
              const int leader = __ffs(m) - 1;
              uint32_t wb = 0;
              if (static_cast<int>(lane) == leader) wb = atomicAdd(&out_count, static_cast<uint32_t>(__popc(m)));
              wb = __shfl_sync(kFullMask, wb, leader);
              if (won) out[wb + __popc(m & lanemask_lt())] = c | gtag;
            }
          }
        }
        if (g + 1 < p.gens && !one_flush) {
          __syncthreads();
          const uint32_t pending = out_count;
          __syncthreads();
          if (pending + tile > out_cap) flush_block(p, next, out, &out_count, &out_base);
        }
      }
      flush_block(p, next, out, &out_count, &out_base);
    }
    // Persistent form: the layer is done when every block is; block 0 records
    // it and makes it the frontier, and all blocks go on unless the loop stops.
    if (!p.persistent) return;
    LoopState* ls = p.loop;
    if (!grid_barrier(&ls->bar_count, &ls->bar_gen, &p.control->error)) return;
    if (blockIdx.x == 0 && threadIdx.x == 0) loop_step(ls, p.control);
    if (!grid_barrier(&ls->bar_count, &ls->bar_gen, &p.control->error)) return;
    if (*reinterpret_cast<volatile uint32_t*>(&ls->stop)) return;
  }
}

// Sort-unique layer expansion (dedup = sort).  A tile of parents writes all
// its children (tagged) into shared memory, a block radix sort on the state
// bits brings equal children together, unique keeps the first of each run,
// and only the distinct children are tested against the visited set; the
// winners are compacted in place and appended with one reservation per tile.
// Restates, per tile and fused with generation and the claim, the
// reference's batch strategy of sorting and uniquing candidates before the
// visited test (cuda/permutation_bitmap_batch.cu:148,
// cuda/segmented_hash_batch.cu:174).
template <int V, int N>
__global__ void __launch_bounds__(kSortThreads) expand_sorted(ExpandParams p) {
  extern __shared__ __align__(16) unsigned char program_smem[];
  __shared__ SortScratch s;
  __shared__ uint8_t won_flag[kSortTile];
  __shared__ unsigned long long out_base;
  Term* terms = reinterpret_cast<Term*>(program_smem);
  uint32_t* begin = reinterpret_cast<uint32_t*>(program_smem + p.total_terms * sizeof(Term));
  const uint32_t* inverse = begin + p.gens + 1;
  for (uint32_t i = threadIdx.x; i < p.total_terms; i += blockDim.x) terms[i] = p.terms[i];
  for (uint32_t i = threadIdx.x; i <= 2 * p.gens; i += blockDim.x) begin[i] = p.term_begin[i];
  __syncthreads();

  const uint32_t per_tile = kSortTile / p.gens;  // parents per tile
  const unsigned long long state_mask = p.gen_shift ? (1ull << p.gen_shift) - 1ull : p.key_mask;
  const uint32_t key_bits = state_mask == ~0ull ? 64u : 64u - __clzll(static_cast<long long>(state_mask));
  for (;;) {
  // The frontier, its size and the output: from the parameters, or (device
  // loop) from the loop state of the layer in progress.
  unsigned long long count = p.count;
  const unsigned long long* frontier = p.frontier;
  unsigned long long* next = p.next;
  if (p.loop) {
    count = p.loop->count;
    const uint32_t parity = p.loop->parity;
    frontier = p.loop->buf[parity];
    next = p.loop->buf[parity ^ 1u];
  }
  const unsigned long long tiles = (count + per_tile - 1) / per_tile;
  for (unsigned long long t = blockIdx.x; t < tiles; t += gridDim.x) {
    const unsigned long long base = t * per_tile;
    for (uint32_t i = threadIdx.x; i < kSortTile; i += kSortThreads) s.keys[i] = kEmpty;
    __syncthreads();
    // Generation: child of local parent j by generator g goes to slot g * per_tile + j.
    for (uint32_t j = threadIdx.x; j < per_tile; j += kSortThreads) {
      const unsigned long long idx = base + j;
      if (idx >= count) break;
      const uint64_t par = frontier[idx];
      const uint32_t tag = p.gen_shift ? static_cast<uint32_t>(par >> p.gen_shift) : 0u;
      const uint32_t skip = tag ? inverse[tag - 1] : 0xffffffffu;
      for (uint32_t g = 0; g < p.gens; ++g) {
        if (g == skip) continue;
        const uint64_t c = apply_action<N>(p, par, terms, begin[g], begin[g + 1]);
        s.keys[g * per_tile + j] = c | (p.gen_shift ? static_cast<unsigned long long>(g + 1) << p.gen_shift : 0ull);
      }
    }
    __syncthreads();
    block_radix_sort(s, key_bits);
    const uint32_t distinct = block_unique(s, state_mask);
    // Visited claim of the distinct children (coalesced shared-memory reads).
    for (uint32_t i = threadIdx.x; i < kSortTile; i += kSortThreads) {
      const bool valid = i < distinct;
      const unsigned long long key = valid ? s.keys[i] : 0ull;
      won_flag[i] = claim<V, N, false>(p, key & state_mask, valid) ? 1 : 0;
    }
    __syncthreads();
    const uint32_t winners = block_compact(s, [&](uint32_t i, unsigned long long) { return won_flag[i] != 0; });
    if (threadIdx.x == 0 && winners)
      out_base = atomicAdd(&p.control->next_count, static_cast<unsigned long long>(winners));
    __syncthreads();
    bool overflow = false;
    for (uint32_t i = threadIdx.x; i < winners; i += kSortThreads) {
      const unsigned long long pos = out_base + i;
      if (pos < p.capacity) next[pos] = s.keys[i];
      else overflow = true;
    }
    if (overflow) raise_error(&p.control->error, ERR_FRONTIER_OVERFLOW);
    __syncthreads();
  }
  // Persistent form, as in expand_packed: block 0 records the layer between
  // two grid barriers and every block goes on unless the loop stops.
  if (!p.persistent) return;
  LoopState* ls = p.loop;
  if (!grid_barrier(&ls->bar_count, &ls->bar_gen, &p.control->error)) return;
  if (blockIdx.x == 0 && threadIdx.x == 0) loop_step(ls, p.control);
  if (!grid_barrier(&ls->bar_count, &ls->bar_gen, &p.control->error)) return;
  if (*reinterpret_cast<volatile uint32_t*>(&ls->stop)) return;
  }
}

// The step as its own launch in the graph form: the WHILE node repeats while
// `stop` is 0.
static __global__ void loop_finalize(LoopState* s, Control* c, cudaGraphConditionalHandle handle) {
  cudaGraphSetConditional(handle, loop_step(s, c) ? 0u : 1u);
}

static __global__ void loop_start(unsigned long long* stamps) {
  unsigned long long now;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(now));
  stamps[0] = now;
}

// Marks the start state visited (and, for the hash paths, inserts it).
static __global__ void seed_packed(ExpandParams p, unsigned long long start, int kind, uint32_t n) {
  if (threadIdx.x || blockIdx.x) return;
  uint64_t r = 0;
  if (kind == V_LEHMER) {
    r = lehmer_rank4_n(start, n);
    atomicOr(&p.bitmap[r >> 6], 1ull << (r & 63));
  } else if (kind == V_MULTISET) {
    if (multiset_rank(start, p.ms, &r)) atomicOr(&p.bitmap[r >> 6], 1ull << (r & 63));
    else raise_error(&p.control->error, ERR_RANK_RANGE);
  } else if (kind == V_PRODUCT) {
    if (product_rank(start, p.pd, &r)) atomicOr(&p.bitmap[r >> 6], 1ull << (r & 63));
    else raise_error(&p.control->error, ERR_RANK_RANGE);
  } else if (kind == V_RADIX) {
    r = radix_rank(start, p.mat);
    atomicOr(&p.bitmap[r >> 6], 1ull << (r & 63));
  } else if (kind == V_HASHQ) {
    if (qhash_insert(p.q, start) < 0) raise_error(&p.control->error, ERR_TABLE_FULL);
  } else {
    if (hash_insert(p.table, p.table_mask, start, p.key_mask, p.tag, p.probe_limit) < 0)
      raise_error(&p.control->error, ERR_TABLE_FULL);
  }
}

// Re-inserts every key of an old all-visited table into a larger one.
static __global__ void rehash_table(const unsigned long long* old_table, unsigned long long old_slots,
                             unsigned long long* table, unsigned long long mask, unsigned long long key_mask,
                             unsigned int* error) {
  for (unsigned long long i = blockIdx.x * static_cast<unsigned long long>(blockDim.x) + threadIdx.x; i < old_slots;
       i += static_cast<unsigned long long>(gridDim.x) * blockDim.x) {
    const unsigned long long v = old_table[i];
    if (v == kEmpty) continue;
    // Keep the tag bits: insert the full word, compare on the key bits.
    uint64_t slot = mix64(v & key_mask) & mask;
    bool placed = false;
    for (unsigned long long probe = 0; probe <= mask; ++probe) {
      if (atomicCAS(&table[slot], kEmpty, v) == kEmpty) {
        placed = true;
        break;
      }
      slot = (slot + 1) & mask;
    }
    if (!placed) atomicOr(error, ERR_TABLE_FULL);
  }
}

// Re-inserts every key of a quotient table into a larger one: the mixed
// value of the key in slot t is (stored >> D) << s | (t - distance).
static __global__ void rehash_qtable(QuotientSlots from, QuotientSlots to, unsigned int* error) {
  const uint64_t slots = from.mask + 1;
  for (unsigned long long t = blockIdx.x * static_cast<unsigned long long>(blockDim.x) + threadIdx.x; t < slots;
       t += static_cast<unsigned long long>(gridDim.x) * blockDim.x) {
    const unsigned int v = from.slots[t];
    if (v == 0u) continue;
    const uint64_t dist = (v & ((from.d >= 32 ? 0u : (1u << from.d)) - 1u)) - 1u;
    const uint64_t x = ((static_cast<uint64_t>(v) >> from.d) << from.s) | ((t - dist) & from.mask);
    const uint64_t home = x & to.mask, rem = x >> to.s;
    bool placed = false;
    for (uint32_t j = 0; j < to.limit; ++j) {
      const unsigned int want = static_cast<unsigned int>((rem << to.d) | (j + 1));
      if (atomicCAS(to.slots + ((home + j) & to.mask), 0u, want) == 0u) {
        placed = true;
        break;
      }
    }
    if (!placed) atomicOr(error, ERR_TABLE_FULL);
  }
}

}  // namespace mgbfs2
