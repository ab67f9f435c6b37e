// Batched sweep: many independent BFS instances (different degrees and
// generator sets, very uneven sizes) advance together, one layer of all of
// them per step, inside ONE CUDA-graph launch per wave:
//
//     WHILE (any instance active) { batch_expand ; batch_finalize }
//
// The loop condition is set on the device by batch_finalize
// (cudaGraphSetConditional), so a wave costs one graph launch and one host
// synchronisation, whatever its depth.  (The reference runs instances one
// after another, multigpubfs/generic_session.py:139; its device-driven graph
// loop precedent is cuda/generic_sorted_carry_graph.cuh:62-84.)
//
// Layout: every instance owns a Lehmer bitmap of n!/64 words and a segment of
// `cap` words in each of the two frontier buffers.  The current frontier is
// cut into tiles of kBatchTile entries that never straddle two instances; a
// block maps a tile index to (instance, local tile) through an exclusive
// prefix of the per-instance tile counts, so the degree, the generator
// program and the segment are uniform over the block (the rank is unrolled
// for that degree).  Winners are staged in shared memory and appended to the
// instance's segment with one reservation per block flush.
//
// Segments sized by a prediction (the learned planner) can overflow.  A winner
// that finds no room in the segment clears its bitmap bit again, so after the
// layer the bitmap holds exactly the visited states plus the winners that were
// stored.  The finalize step then gives the instance a larger next segment
// from a spare pool region of the wave (the exact winner count of the failed
// attempt bounds the layer), the stored winners are moved there by all blocks,
// and the instance expands the same layer again while the others go on: the
// overflow costs one layer, and the table is the same.  Only when the pool is
// exhausted is the instance retired and rerun from depth 0 with its orbit
// bound in a later wave.
#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include "../../include/mgbfs2.h"
#include "engine.h"

#define MG_CHECK_BATCH(expr)                          \
  do {                                                \
    cudaError_t _e = (expr);                          \
    if (_e != cudaSuccess) return cuda_status(_e);    \
  } while (0)

namespace mgbfs2 {
namespace {

constexpr uint32_t kBatchBlock = 256;
constexpr int kBatchBlocksPerSM = 4;   // default resident batch_expand blocks per SM
// Layer loop of a wave (mgbfs2_batch_options.host_loop): persistent, host (1) or graph.
constexpr uint32_t kLoopPersistent = 0, kLoopGraph = 2;
constexpr uint32_t kBatchPpt = 4;                         // most frontier entries per thread per tile
constexpr uint32_t kBatchTile = kBatchBlock * kBatchPpt;  // most entries per tile (one instance per tile)
// A wave's tile is kBatchBlock * ppt entries, ppt in {1, 2, 4} (the tuned
// shape; 4 by default).
constexpr uint32_t kBatchOut = 4096;                      // winners staged in shared memory per block
constexpr uint32_t kMaxBatchGens = 16;
constexpr uint32_t kMaxBatchTerms = kMaxBatchGens * 15;   // <= n distinct displacements per generator
enum : uint32_t { INST_ACTIVE = 0, INST_DONE = 1, INST_OVERFLOW = 2, INST_IDLE = 3 };

struct BatchInst {
  uint32_t n, gens, term_off, inv_off;  // term_off: first of gens + 1 offsets in tbegin
  uint32_t gen_shift, status;           // parent-edge tag position (0 = none)
  uint32_t sel_off, bytes;              // byte-permute selectors (6 per generator) when bytes != 0
  unsigned long long bitmap_off;        // first bitmap word
  // Frontier segments: offset and capacity in buf[0] and in buf[1]; the
  // current layer is in buf[par], the next one is written to buf[par ^ 1].
  unsigned long long seg_off[2], seg_cap[2];
  uint32_t par, depth;                  // this instance's buffer parity and its current depth
};

// A move of the stored winners of an overflowed layer into the instance's new
// segment (entries of buf[buf]).
struct BatchReloc {
  unsigned long long src, dst, count;
  uint32_t buf, pad;
};

struct BatchCtl {
  unsigned long long total;  // entries in the current frontier
  unsigned long long tiles;      // tiles of the current frontier (tile_prefix[count])
  unsigned long long next_tile;  // work counter of batch_expand, reset by every finalize
  unsigned long long pool_base, pool_cap, pool_used;  // spare segment region (entries, same in both buffers)
  uint32_t step, max_depth, error, reloc_count;       // step: layer steps taken by the wave
  uint32_t redo_layers, max_steps;                    // max_steps: entries of the stamp array - 1
  uint32_t ppt, pad;                                  // frontier entries per thread of a tile
  uint32_t bar_count, bar_gen;   // grid barrier of the persistent wave kernel (zero at the wave's start)
};

struct BatchParams {
  BatchInst* inst;
  uint32_t count, pad;
  const Term* terms;
  const uint32_t* tbegin;   // absolute term offsets
  const uint32_t* inverse;  // absolute generator index -> inverse generator index (within the instance)
  const uint32_t* sel;      // byte-permute selectors, 6 per generator of a byte-path instance
  unsigned long long* bitmap;
  unsigned long long* buf[2];
  unsigned long long* tile_prefix;  // count + 1 entries: exclusive prefix of per-instance tile counts
  unsigned long long* cur_count;    // per instance: entries in the current frontier
  unsigned long long* next_count;   // per instance: winners appended to the next frontier
  unsigned long long* layers;       // count x max_depth
  uint32_t* layer_step;             // count x max_depth: the wave's step that produced each layer
  unsigned long long* stamps;       // max_steps + 1: globaltimer at the seed (0) and after step t (t + 1)
  BatchReloc* reloc;                // count entries: moves queued by the last finalize
  BatchCtl* ctl;
};

// Per-block state: the instance of the current tile, its generator program,
// and the staged winners.
struct BatchSmem {
  unsigned long long out[kBatchOut];
  Term terms[kMaxBatchTerms];
  uint32_t sel[kMaxBatchGens * 6];
  uint32_t begin[kMaxBatchGens + 1];
  uint32_t inverse[kMaxBatchGens];
  const unsigned long long* front;  // the instance's current segment
  unsigned long long* next;         // the instance's next segment
  unsigned long long bitmap_off, seg_cap, count, tile, local_tile, out_base;
  uint32_t inst, found, n, gens, shift, out_count, bytes, ppt;
};

__device__ __forceinline__ uint32_t find_instance(const unsigned long long* prefix, uint32_t count,
                                                  unsigned long long idx) {
  uint32_t lo = 0, hi = count;
  while (hi - lo > 1) {
    const uint32_t mid = (lo + hi) >> 1;
    if (prefix[mid] <= idx) lo = mid;
    else hi = mid;
  }
  return lo;
}

// The pointers a tile needs, passed by value (a reference to the kernel
// parameter block would copy it to local memory).
struct TileArgs {
  unsigned long long* bitmap;
  unsigned long long* next_count;
};

// Appends the block's staged winners to the current instance's next segment
// with one reservation.  A winner whose position is at or past the segment's
// capacity is not written and clears its bitmap bit again (with an atomic of
// the claim's width), so that a redo of the layer finds it unvisited;
// batch_finalize sees the count above capacity and redoes the layer in a
// larger segment.  Called by all threads of the block.
__device__ __forceinline__ void batch_flush(const TileArgs a, BatchSmem& s) {
  __syncthreads();
  const uint32_t n = s.out_count;
  if (threadIdx.x == 0 && n) s.out_base = atomicAdd(&a.next_count[s.inst], static_cast<unsigned long long>(n));
  __syncthreads();
  const unsigned long long base = s.out_base, cap = s.seg_cap;
  unsigned long long* seg = s.next;
  for (uint32_t k = threadIdx.x; k < n; k += blockDim.x) {
    if (base + k < cap) {
      seg[base + k] = s.out[k];
    } else {
      const uint64_t w = s.out[k] & ((1ull << (4 * s.n)) - 1ull);
      const uint64_t r = lehmer_rank4_n(w, s.n);
      if (s.bytes)
        atomicAnd(reinterpret_cast<unsigned int*>(a.bitmap + s.bitmap_off) + (r >> 5), ~(1u << (r & 31)));
      else
        atomicAnd(a.bitmap + s.bitmap_off + (r >> 6), ~(1ull << (r & 63)));
    }
  }
  __syncthreads();
  if (threadIdx.x == 0) s.out_count = 0;
  __syncthreads();
}

// Byte-lane form of a packed state of at most 12 symbols: symbol i in byte
// i % 4 of register i / 4 (nibble -> byte spreading, 4 ops per register).
__device__ __forceinline__ void spread_bytes(uint64_t w, uint32_t (&b)[3]) {
#pragma unroll
  for (int j = 0; j < 3; ++j) {
    const uint32_t v = static_cast<uint32_t>(w >> (16 * j)) & 0xffffu;
    const uint32_t y = (v | (v << 8)) & 0x00ff00ffu;
    b[j] = (y | (y << 4)) & 0x0f0f0f0fu;
  }
}

// Inverse of spread_bytes for byte values below 16.
__device__ __forceinline__ uint64_t pack_bytes(const uint32_t (&b)[3]) {
  uint64_t w = 0;
#pragma unroll
  for (int j = 0; j < 3; ++j) {
    const uint32_t y = (b[j] | (b[j] >> 4)) & 0x00ff00ffu;
    w |= static_cast<uint64_t>((y | (y >> 8)) & 0xffffu) << (16 * j);
  }
  return w;
}

// Lehmer rank of N <= 12 distinct byte-lane symbols.
template <int N>
__device__ __forceinline__ uint32_t lehmer_rank_bytes(const uint32_t (&b)[3]) {
  uint32_t used = 0, rank = 0;
#pragma unroll
  for (int i = 0; i < N - 1; ++i) {
    const uint32_t s = (b[i >> 2] >> (8 * (i & 3))) & 0xffu;
    rank = rank * static_cast<uint32_t>(N - i) + (s - __popc(used & ((1u << s) - 1u)));
    used |= 1u << s;
  }
  return rank;
}

// Tile of a byte-path instance (N <= 12, generators with many displacement
// groups): every parent is spread to byte lanes once, and each child is two
// byte permutes per output register (selectors precomputed on the host)
// instead of one shift-mask-or per displacement group; only winners are
// packed back to nibbles.
template <int N>
__device__ __forceinline__ void batch_tile_bytes(const TileArgs a, BatchSmem& s) {
  const uint32_t lane = lane_id();
  const uint32_t ppt = s.ppt, tile = kBatchBlock * ppt;
  const unsigned long long count = s.count, base = s.local_tile * tile;
  const uint32_t gens = s.gens, shift = s.shift;
  const unsigned long long* seg = s.front;
  unsigned int* bitmap = reinterpret_cast<unsigned int*>(a.bitmap + s.bitmap_off);
  uint32_t eb[kBatchPpt][3];
  uint32_t skip[kBatchPpt];
  bool val[kBatchPpt];
#pragma unroll
  for (uint32_t k = 0; k < kBatchPpt; ++k) {
    const unsigned long long idx = base + k * kBatchBlock + threadIdx.x;
    val[k] = k < ppt && idx < count;
    uint64_t w = val[k] ? seg[idx] : 0ull;
    const uint32_t tag = shift ? static_cast<uint32_t>(w >> shift) : 0u;
    skip[k] = tag ? s.inverse[tag - 1] : 0xffffffffu;
    if (shift) w &= (1ull << shift) - 1ull;
    spread_bytes(w, eb[k]);
  }
  for (uint32_t g = 0; g < gens; ++g) {
    const uint32_t* sel = s.sel + 6 * g;
    const uint32_t s0 = sel[0], s1 = sel[1], s2 = sel[2], s3 = sel[3], s4 = sel[4], s5 = sel[5];
    const unsigned long long gtag = shift ? static_cast<unsigned long long>(g + 1) << shift : 0ull;
#pragma unroll
    for (uint32_t k = 0; k < kBatchPpt; ++k) {
      if (k >= ppt) break;  // block-uniform
      const bool live = val[k] && g != skip[k];
      bool won = false;
      uint32_t cb[3];
      cb[0] = __byte_perm(__byte_perm(eb[k][0], eb[k][1], s0), eb[k][2], s1);
      cb[1] = __byte_perm(__byte_perm(eb[k][0], eb[k][1], s2), eb[k][2], s3);
      cb[2] = __byte_perm(__byte_perm(eb[k][0], eb[k][1], s4), eb[k][2], s5);
      if (live) {
        const uint32_t r = lehmer_rank_bytes<N>(cb);
        const uint32_t bit = 1u << (r & 31);
        won = !(atomicOr(&bitmap[r >> 5], bit) & bit);
      }
      const unsigned m = __ballot_sync(kFullMask, won);
      if (m) {
        const int leader = __ffs(m) - 1;
        uint32_t at = 0;
        if (static_cast<int>(lane) == leader) at = atomicAdd(&s.out_count, static_cast<uint32_t>(__popc(m)));
        at = __shfl_sync(kFullMask, at, leader);
        if (won) s.out[at + __popc(m & lanemask_lt())] = pack_bytes(cb) | gtag;
      }
    }
    if (g + 1 < gens) {
      __syncthreads();
      const uint32_t pending = s.out_count;
      __syncthreads();
      if (pending + tile > kBatchOut) batch_flush(a, s);
    }
  }
  batch_flush(a, s);
}

// One tile (ppt * kBatchBlock consecutive entries of one instance's frontier)
// with a compile-time degree, so the Lehmer rank is fully unrolled.
template <int N>
__device__ __forceinline__ void batch_tile(const TileArgs a, BatchSmem& s) {
  if constexpr (N <= 12) {
    if (s.bytes) {
      batch_tile_bytes<N>(a, s);
      return;
    }
  }
  const uint32_t lane = lane_id();
  const uint32_t ppt = s.ppt, tile = kBatchBlock * ppt;
  const unsigned long long count = s.count, base = s.local_tile * tile;
  const uint32_t gens = s.gens, shift = s.shift;
  const unsigned long long* seg = s.front;
  unsigned long long* bitmap = a.bitmap + s.bitmap_off;
  uint64_t par[kBatchPpt];
  uint32_t skip[kBatchPpt];
  bool val[kBatchPpt];
#pragma unroll
  for (uint32_t k = 0; k < kBatchPpt; ++k) {
    const unsigned long long idx = base + k * kBatchBlock + threadIdx.x;
    val[k] = k < ppt && idx < count;
    par[k] = val[k] ? seg[idx] : 0ull;
    const uint32_t tag = shift ? static_cast<uint32_t>(par[k] >> shift) : 0u;
    skip[k] = tag ? s.inverse[tag - 1] : 0xffffffffu;
    if (shift) par[k] &= (1ull << shift) - 1ull;
  }
  for (uint32_t g = 0; g < gens; ++g) {
    const uint32_t tb = s.begin[g], te = s.begin[g + 1];
    const unsigned long long gtag = shift ? static_cast<unsigned long long>(g + 1) << shift : 0ull;
#pragma unroll
    for (uint32_t k = 0; k < kBatchPpt; ++k) {
      if (k >= ppt) break;  // block-uniform
      const bool live = val[k] && g != skip[k];
      bool won = false;
      uint64_t c = 0;
      if (live) {
        c = apply_terms(par[k], s.terms, tb, te);
        const uint64_t r = lehmer_rank4<N>(c);
        const unsigned long long bit = 1ull << (r & 63);
        won = !(atomicOr(&bitmap[r >> 6], bit) & bit);
      }
      const unsigned m = __ballot_sync(kFullMask, won);
      if (m) {
        const int leader = __ffs(m) - 1;
        uint32_t at = 0;
        if (static_cast<int>(lane) == leader) at = atomicAdd(&s.out_count, static_cast<uint32_t>(__popc(m)));
        at = __shfl_sync(kFullMask, at, leader);
        if (won) s.out[at + __popc(m & lanemask_lt())] = c | gtag;
      }
    }
    if (g + 1 < gens) {
      __syncthreads();
      const uint32_t pending = s.out_count;
      __syncthreads();
      if (pending + tile > kBatchOut) batch_flush(a, s);
    }
  }
  batch_flush(a, s);
}

// Persistent expansion of one layer of every active instance.  The frontier
// is cut into per-instance tiles; a block takes the next tile from a device
// counter (so all blocks stay within a window of about one tile each, i.e.
// on one or two instances' bitmaps, which then stay in L2 even when the
// wave's bitmaps together do not fit), finds the tile's instance by binary
// search of the tile prefix, loads that
// instance's generator program into shared memory when it changes, and
// stages its winners for one segment reservation per flush.
__device__ __forceinline__ void expand_layer(const BatchParams& p, BatchSmem& s) {
  const unsigned long long tiles = p.ctl->tiles;
  const TileArgs a{p.bitmap, p.next_count};
  if (threadIdx.x == 0) {
    s.out_count = 0;
    s.inst = 0xffffffffu;
    s.ppt = p.ctl->ppt;
  }
  for (;;) {
    __syncthreads();
    if (threadIdx.x == 0) {
      const unsigned long long t = atomicAdd(&p.ctl->next_tile, 1ull);
      s.tile = t;
      if (t < tiles) {
        const uint32_t i = find_instance(p.tile_prefix, p.count, t);
        s.found = i;
        s.local_tile = t - p.tile_prefix[i];
      }
    }
    __syncthreads();
    if (s.tile >= tiles) break;  // block-uniform
    const uint32_t i = s.found;
    if (i != s.inst) {  // block-uniform: every thread read the same s.found and s.inst
      __syncthreads();
      const BatchInst in = p.inst[i];
      const uint32_t t0 = p.tbegin[in.term_off], t1 = p.tbegin[in.term_off + in.gens];
      for (uint32_t k = threadIdx.x; k < t1 - t0; k += blockDim.x) s.terms[k] = p.terms[t0 + k];
      for (uint32_t k = threadIdx.x; k <= in.gens; k += blockDim.x) s.begin[k] = p.tbegin[in.term_off + k] - t0;
      for (uint32_t k = threadIdx.x; k < in.gens; k += blockDim.x) s.inverse[k] = p.inverse[in.inv_off + k];
      if (in.bytes)
        for (uint32_t k = threadIdx.x; k < 6 * in.gens; k += blockDim.x) s.sel[k] = p.sel[in.sel_off + k];
      if (threadIdx.x == 0) {
        // Select, not index: a runtime index into the parameter block would
        // copy it to local memory.
        const uint32_t cur = in.par, nxt = in.par ^ 1u;
        s.inst = i;
        s.n = in.n;
        s.gens = in.gens;
        s.shift = in.gen_shift;
        s.bytes = in.bytes;
        s.bitmap_off = in.bitmap_off;
        s.front = (cur ? p.buf[1] : p.buf[0]) + (cur ? in.seg_off[1] : in.seg_off[0]);
        s.next = (nxt ? p.buf[1] : p.buf[0]) + (nxt ? in.seg_off[1] : in.seg_off[0]);
        s.seg_cap = nxt ? in.seg_cap[1] : in.seg_cap[0];
        s.count = p.cur_count[i];
      }
      __syncthreads();
    }
    switch (s.n) {
      case 2: batch_tile<2>(a, s); break;
      case 3: batch_tile<3>(a, s); break;
      case 4: batch_tile<4>(a, s); break;
      case 5: batch_tile<5>(a, s); break;
      case 6: batch_tile<6>(a, s); break;
      case 7: batch_tile<7>(a, s); break;
      case 8: batch_tile<8>(a, s); break;
      case 9: batch_tile<9>(a, s); break;
      case 10: batch_tile<10>(a, s); break;
      case 11: batch_tile<11>(a, s); break;
      case 12: batch_tile<12>(a, s); break;
      case 13: batch_tile<13>(a, s); break;
      case 14: batch_tile<14>(a, s); break;
      default: batch_tile<15>(a, s); break;
    }
  }
}

__global__ void __launch_bounds__(kBatchBlock) batch_expand(BatchParams p) {
  __shared__ BatchSmem s;
  expand_layer(p, s);
}


// One block: record the layer, retire finished or overflowed instances, build
// the prefix of the new per-instance tile counts, flip the buffers.  Returns
// the new frontier's tile count (0 ends the wave).
struct FinalizeSmem {
  unsigned long long warp_sums[32];
  unsigned long long carry, entries;
};

__device__ unsigned long long finalize_layer(const BatchParams& p, FinalizeSmem& f) {
  const uint32_t step = p.ctl->step, max_depth = p.ctl->max_depth;
  if (threadIdx.x == 0) {
    f.carry = f.entries = 0;
    p.ctl->reloc_count = 0;  // the moves of the previous step are done
  }
  __syncthreads();
  for (uint32_t base = 0; base < p.count; base += blockDim.x) {
    const uint32_t i = base + threadIdx.x;
    unsigned long long c = 0;
    if (i < p.count) {
      BatchInst& in = p.inst[i];
      const unsigned long long produced = p.next_count[i];
      unsigned long long frontier = 0;  // the instance's frontier entries in the next step
      unsigned long long stored = 0;    // entries already in its next segment at the next step
      if (in.status == INST_ACTIVE) {
        const uint32_t nb = in.par ^ 1u;
        const unsigned long long cap = in.seg_cap[nb];
        if (produced > cap) {
          // Every winner of the failed attempt was counted, so `produced`
          // bounds the layer: a segment of that size cannot overflow again.
          // The first `cap` winners were stored (and keep their bits); they
          // move to the new segment, the rest are found again by the redo.
          const unsigned long long off = atomicAdd(&p.ctl->pool_used, produced);
          if (off + produced <= p.ctl->pool_cap) {
            const uint32_t j = atomicAdd(&p.ctl->reloc_count, 1u);
            p.reloc[j] = BatchReloc{in.seg_off[nb], p.ctl->pool_base + off, cap, nb, 0u};
            in.seg_off[nb] = p.ctl->pool_base + off;
            in.seg_cap[nb] = produced;
            stored = cap;
            frontier = p.cur_count[i];
            atomicAdd(&p.ctl->redo_layers, 1u);
          } else {
            in.status = INST_OVERFLOW;  // pool exhausted: rerun from depth 0 later
          }
        } else if (produced == 0) {
          in.status = INST_DONE;
        } else if (in.depth + 1 >= max_depth) {
          in.status = INST_OVERFLOW;
          atomicOr(&p.ctl->error, ERR_FRONTIER_OVERFLOW);
        } else {
          const unsigned long long row = static_cast<unsigned long long>(i) * max_depth + in.depth + 1;
          p.layers[row] = produced;
          p.layer_step[row] = step;
          in.depth += 1;
          in.par = nb;
          frontier = produced;
        }
      }
      p.next_count[i] = stored;
      p.cur_count[i] = frontier;
      const unsigned long long tile = kBatchBlock * p.ctl->ppt;
      c = (frontier + tile - 1) / tile;
      if (frontier) atomicAdd(&f.entries, frontier);
    }
    // Block-wide exclusive scan of c.
    unsigned long long incl = c;
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const unsigned long long up = __shfl_up_sync(kFullMask, incl, o);
      if (lane >= static_cast<uint32_t>(o)) incl += up;
    }
    if (lane == 31) f.warp_sums[warp] = incl;
    __syncthreads();
    if (warp == 0) {
      unsigned long long v = lane < blockDim.x / 32 ? f.warp_sums[lane] : 0ull, x = v;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const unsigned long long up = __shfl_up_sync(kFullMask, x, o);
        if (lane >= static_cast<uint32_t>(o)) x += up;
      }
      if (lane < blockDim.x / 32) f.warp_sums[lane] = x - v;
    }
    __syncthreads();
    if (i < p.count) p.tile_prefix[i] = f.carry + f.warp_sums[warp] + incl - c;
    __syncthreads();
    if (threadIdx.x == blockDim.x - 1) f.carry += f.warp_sums[warp] + incl;
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    unsigned long long now;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(now));
    if (step + 1 <= p.ctl->max_steps) p.stamps[step + 1] = now;
    p.tile_prefix[p.count] = f.carry;
    p.ctl->tiles = f.carry;
    p.ctl->next_tile = 0;
    p.ctl->total = f.entries;
    p.ctl->step = step + 1;
  }
  __syncthreads();
  return f.carry;
}

// The moves queued by the last finalize, by every thread of the grid.
__device__ __forceinline__ void relocate_segments(const BatchParams& p, uint32_t moves) {
  const unsigned long long stride = static_cast<unsigned long long>(gridDim.x) * blockDim.x;
  for (uint32_t j = 0; j < moves; ++j) {
    const BatchReloc r = p.reloc[j];
    unsigned long long* b = r.buf ? p.buf[1] : p.buf[0];
    for (unsigned long long k = blockIdx.x * static_cast<unsigned long long>(blockDim.x) + threadIdx.x; k < r.count;
         k += stride)
      b[r.dst + k] = b[r.src + k];
  }
}

// The moves as their own launch (graph and host loops), after batch_finalize.
__global__ void __launch_bounds__(kBatchBlock) batch_relocate(BatchParams p) {
  const uint32_t moves = *reinterpret_cast<volatile uint32_t*>(&p.ctl->reloc_count);
  relocate_segments(p, moves);
}

// The finalize step as its own one-block launch (graph and host loops); in
// the graph loop it also sets the WHILE node's condition.
__global__ void __launch_bounds__(1024) batch_finalize(BatchParams p, cudaGraphConditionalHandle handle,
                                                       int use_handle) {
  __shared__ FinalizeSmem f;
  const unsigned long long tiles = finalize_layer(p, f);
  if (use_handle && threadIdx.x == 0) cudaGraphSetConditional(handle, tiles > 0 ? 1u : 0u);
}

// A whole wave in one cooperative launch: every block expands its tiles of
// the layer, a grid barrier, block 0 finalizes, a second barrier, and all
// blocks go on while the new frontier has tiles.  Two barriers per layer
// replace two kernel launches per layer.
// Four blocks per SM (as many as its shared memory and registers allow):
// the bound lets the compiler keep 64 registers, 1 % faster than 48 on S12.
__global__ void __launch_bounds__(kBatchBlock, kBatchBlocksPerSM) batch_wave(BatchParams p) {
  __shared__ BatchSmem s;
  __shared__ FinalizeSmem f;
  __shared__ int more;
  __shared__ uint32_t moves;
  for (;;) {
    expand_layer(p, s);
    if (!grid_barrier(&p.ctl->bar_count, &p.ctl->bar_gen, &p.ctl->error)) return;
    if (blockIdx.x == 0) finalize_layer(p, f);
    if (!grid_barrier(&p.ctl->bar_count, &p.ctl->bar_gen, &p.ctl->error)) return;
    if (threadIdx.x == 0) {
      more = *reinterpret_cast<volatile unsigned long long*>(&p.ctl->tiles) > 0;
      moves = *reinterpret_cast<volatile uint32_t*>(&p.ctl->reloc_count);
    }
    __syncthreads();
    // A layer redo moves stored winners first; only then may the redo claim.
    // `moves` is the same in every block (read after the barrier that follows
    // the finalize), so all blocks take this barrier or none.
    if (moves) {
      relocate_segments(p, moves);
      if (!grid_barrier(&p.ctl->bar_count, &p.ctl->bar_gen, &p.ctl->error)) return;
    }
    if (!more) return;
  }
}

__global__ void batch_seed(BatchParams p) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < p.count; i += gridDim.x * blockDim.x) {
    const BatchInst in = p.inst[i];
    // Identity-coded start: code c at position c.  Its rank is 0.
    unsigned long long start = 0;
    for (uint32_t e = 0; e < in.n; ++e) start |= static_cast<unsigned long long>(e) << (4 * e);
    p.buf[0][in.seg_off[0]] = start;
    p.bitmap[in.bitmap_off] |= 1ull;
    p.tile_prefix[i] = i;  // one entry, one tile per instance
    p.cur_count[i] = 1;
    p.layers[static_cast<unsigned long long>(i) * p.ctl->max_depth] = 1;
    p.next_count[i] = 0;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    unsigned long long now;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(now));
    p.stamps[0] = now;
    p.tile_prefix[p.count] = p.count;
    p.ctl->tiles = p.count;
    p.ctl->next_tile = 0;
    p.ctl->total = p.count;
    p.ctl->step = 0;
    p.ctl->error = 0;
    p.ctl->reloc_count = 0;
    p.ctl->redo_layers = 0;
    p.ctl->pool_used = 0;
  }
}

uint64_t factorial(uint32_t n) {
  uint64_t f = 1;
  for (uint32_t i = 2; i <= n; ++i) f *= i;
  return f;
}

}  // namespace

// Host side of one batch.
struct Batch {
  struct Instance {
    uint32_t n = 0, gens = 0;
    std::vector<Term> terms;
    std::vector<uint32_t> begin;   // gens + 1 relative offsets
    std::vector<uint32_t> inverse; // gens entries
    std::vector<uint32_t> sel;     // byte-permute selectors (6 per generator); empty = displacement terms
    bool inverse_closed = false;
    uint64_t orbit = 0;            // n!
    std::vector<uint64_t> layers;
    std::vector<double> layer_seconds;  // per layer d >= 1: its wave's expansion of layer d - 1
    uint32_t status = INST_IDLE;
    uint32_t runs = 0;
  };
  int device = 0;
  cudaStream_t stream = nullptr;
  int sm_count = 148;
  std::vector<Instance> inst;
  DeviceBuffer arena;
  mgbfs2_batch_status last{};
};

static int validate_instance(const mgbfs2_graph_desc& d, Batch::Instance* out, std::string* why) {
  if (d.kind != 0 || !d.permutations || !d.start) { *why = "BATCH_REQUIRES_PERMUTATION_ACTION"; return MGBFS2_UNSUPPORTED; }
  const uint32_t n = d.elements;
  if (n < 2 || n > 15) { *why = "BATCH_DEGREE"; return MGBFS2_UNSUPPORTED; }
  if (!d.generators || d.generators > kMaxBatchGens) { *why = "BATCH_GENERATORS"; return MGBFS2_UNSUPPORTED; }
  // Distinct labels: the instance is coded by sorted label order.
  std::vector<int64_t> labels(d.start, d.start + n);
  std::vector<int64_t> sorted = labels;
  std::sort(sorted.begin(), sorted.end());
  if (std::adjacent_find(sorted.begin(), sorted.end()) != sorted.end()) {
    *why = "BATCH_REQUIRES_DISTINCT_LABELS";
    return MGBFS2_UNSUPPORTED;
  }
  // With distinct labels the layer table does not depend on the start: a
  // state x (as codes) evolves by x -> x o g, and x = c o y maps the BFS from
  // the start's coding c bijectively, layer by layer, onto the BFS of y from
  // the identity.  Every instance therefore runs from the identity coding.
  Batch::Instance in;
  in.n = n;
  in.gens = d.generators;
  in.orbit = factorial(n);
  in.begin.assign(1, 0);
  // A generator of at most 15 points is one 60-bit word (4 bits per image), so
  // finding a generator's inverse among them is a word comparison.
  std::vector<uint64_t> words(in.gens);
  for (uint32_t k = 0; k < in.gens; ++k) {
    const uint32_t* g = d.permutations + static_cast<size_t>(k) * n;
    uint32_t seen = 0;
    uint64_t w = 0;
    for (uint32_t i = 0; i < n; ++i) {
      const uint32_t v = g[i];
      if (v >= n || (seen >> v) & 1u) { *why = "GRAPH_PERMUTATION_GENERATOR"; return MGBFS2_INVALID_ARGUMENT; }
      seen |= 1u << v;
      w |= static_cast<uint64_t>(v) << (4 * i);
    }
    words[k] = w;
    // One term per displacement g[i] - i, in ascending displacement order.
    uint64_t masks[2 * 15 + 1] = {};
    for (uint32_t i = 0; i < n; ++i) masks[static_cast<int>(g[i]) - static_cast<int>(i) + 15] |= 15ull << (4 * i);
    for (int disp = -15; disp <= 15; ++disp) {
      if (!masks[disp + 15]) continue;
      const int shift = disp * 4;
      in.terms.push_back(Term{masks[disp + 15], shift > 0 ? static_cast<uint32_t>(shift) : 0u,
                              shift < 0 ? static_cast<uint32_t>(-shift) : 0u});
    }
    in.begin.push_back(static_cast<uint32_t>(in.terms.size()));
  }
  // Byte path for degree <= 12 when the generators average more than three
  // displacement groups: child register j (symbols 4j..4j+3) is
  // perm(perm(parent0, parent1, s1), parent2, s2) over the byte lanes, with
  // source symbol g[q] (or a zero lane past the degree) for every output symbol q.
  if (n <= 12 && in.terms.size() > 3ull * in.gens) {
    for (uint32_t k = 0; k < in.gens; ++k) {
      const uint32_t* g = d.permutations + static_cast<size_t>(k) * n;
      for (uint32_t j = 0; j < 3; ++j) {
        uint32_t s1 = 0, s2 = 0;
        for (uint32_t t = 0; t < 4; ++t) {
          const uint32_t q = 4 * j + t;
          const uint32_t src = q < n ? g[q] : (n < 12 ? n : 0);
          s1 |= (src < 8 ? src : 0u) << (4 * t);
          s2 |= (src < 8 ? t : 4 + (src - 8)) << (4 * t);
        }
        in.sel.push_back(s1);
        in.sel.push_back(s2);
      }
    }
  }
  in.inverse_closed = true;
  in.inverse.assign(in.gens, 0xffffffffu);
  for (uint32_t k = 0; k < in.gens; ++k) {
    uint64_t inv = 0;
    for (uint32_t i = 0; i < n; ++i)
      inv |= static_cast<uint64_t>(i) << (4 * d.permutations[static_cast<size_t>(k) * n + i]);
    // The first generator equal to the inverse, as the index lookup did.
    uint32_t h = 0;
    while (h < in.gens && words[h] != inv) ++h;
    if (h == in.gens) in.inverse_closed = false;
    else in.inverse[k] = h;
  }
  if (!in.inverse_closed) std::fill(in.inverse.begin(), in.inverse.end(), 0xffffffffu);
  *out = in;
  return MGBFS2_OK;
}

static int batch_create(const mgbfs2_graph_desc* graphs, uint32_t count, int device, Batch** out, char* error,
                        size_t cap) {
  auto fail = [&](int rc, const std::string& why) {
    if (error && cap) std::snprintf(error, cap, "%s", why.c_str());
    return rc;
  };
  if (!graphs || !count || !out) return fail(MGBFS2_INVALID_ARGUMENT, "BATCH_ARGUMENT");
  auto b = new Batch();
  b->device = device;
  b->inst.resize(count);
  for (uint32_t i = 0; i < count; ++i) {
    std::string why;
    const int rc = validate_instance(graphs[i], &b->inst[i], &why);
    if (rc) {
      delete b;
      return fail(rc, "instance " + std::to_string(i) + ": " + why);
    }
  }
  int rc = cuda_status(cudaSetDevice(device));
  if (!rc) rc = cuda_status(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking));
  if (rc) {
    delete b;
    return fail(rc, "CUDA_SETUP");
  }
  b->arena.stream = b->stream;
  retain_pool_memory(device);
  cudaDeviceGetAttribute(&b->sm_count, cudaDevAttrMultiProcessorCount, device);
  *out = b;
  return MGBFS2_OK;
}

// Runs one wave (the instances in `ids`, with segment capacities `caps`, and
// `pool` spare entries in each frontier buffer for layer redos).
static int run_wave(Batch* b, const std::vector<uint32_t>& ids, const std::vector<uint64_t>& caps, uint64_t pool,
                    uint32_t max_depth, uint32_t blocks_per_sm, uint32_t tile_ppt, uint32_t loop, mgbfs2_batch_status* st,
                    double* kernel_seconds) {
  TraceRange range("batch.wave");
  const uint32_t W = static_cast<uint32_t>(ids.size());
  std::vector<BatchInst> host(W);
  std::vector<Term> terms;
  std::vector<uint32_t> tbegin, inverse, sels;
  uint64_t bitmap_words = 0, seg = 0;
  for (uint32_t k = 0; k < W; ++k) {
    const auto& in = b->inst[ids[k]];
    BatchInst& h = host[k];
    h.n = in.n;
    h.gens = in.gens;
    h.term_off = static_cast<uint32_t>(tbegin.size());
    for (uint32_t x : in.begin) tbegin.push_back(static_cast<uint32_t>(terms.size()) + x);
    terms.insert(terms.end(), in.terms.begin(), in.terms.end());
    h.inv_off = static_cast<uint32_t>(inverse.size());
    inverse.insert(inverse.end(), in.inverse.begin(), in.inverse.end());
    h.gen_shift = in.inverse_closed ? 4 * in.n : 0;
    h.bytes = in.sel.empty() ? 0u : 1u;
    h.sel_off = static_cast<uint32_t>(sels.size());
    sels.insert(sels.end(), in.sel.begin(), in.sel.end());
    h.status = INST_ACTIVE;
    h.bitmap_off = bitmap_words;
    bitmap_words += (in.orbit + 63) / 64;
    h.seg_off[0] = h.seg_off[1] = seg;
    h.seg_cap[0] = h.seg_cap[1] = caps[k];
    h.par = 0;
    h.depth = 0;
    seg += caps[k] + 1;  // +1 keeps every segment non-empty
  }
  // Every layer is redone at most once (a redo's segment holds the failed
  // attempt's exact winner count), so a wave takes at most 2 * max_depth steps.
  const uint32_t max_steps = 2 * max_depth;
  // Arena: instance table | terms | tbegin | inverse | tile prefix | counts | next counts | layers | ctl |
  // bitmaps | buf0 | buf1
  auto al = [](size_t x) { return (x + 255) / 256 * 256; };
  size_t off = 0;
  const size_t o_inst = off; off = al(off + W * sizeof(BatchInst));
  const size_t o_terms = off; off = al(off + terms.size() * sizeof(Term) + 16);
  const size_t o_tbegin = off; off = al(off + tbegin.size() * 4 + 4);
  const size_t o_inv = off; off = al(off + inverse.size() * 4 + 4);
  const size_t o_sel = off; off = al(off + sels.size() * 4 + 4);
  const size_t o_prefix = off; off = al(off + (W + 1) * 8);
  const size_t o_cur = off; off = al(off + W * 8);
  const size_t o_next = off; off = al(off + W * 8);
  const size_t o_layers = off; off = al(off + static_cast<size_t>(W) * max_depth * 8);
  const size_t o_step = off; off = al(off + static_cast<size_t>(W) * max_depth * 4);
  const size_t o_stamps = off; off = al(off + (static_cast<size_t>(max_steps) + 1) * 8);
  const size_t o_reloc = off; off = al(off + W * sizeof(BatchReloc));
  const size_t o_ctl = off; off = al(off + sizeof(BatchCtl));
  const size_t o_bitmap = off; off = al(off + bitmap_words * 8);
  const size_t o_buf0 = off; off = al(off + (seg + pool) * 8);
  const size_t o_buf1 = off; off = al(off + (seg + pool) * 8);
  // Exact size: waves are planned against the memory budget, so no headroom.
  int rc = b->arena.ensure(off, true);
  if (rc) return rc;
  char* base = static_cast<char*>(b->arena.ptr);
  BatchCtl ctl{};
  ctl.max_depth = max_depth;
  ctl.max_steps = max_steps;
  ctl.pool_base = seg;
  ctl.pool_cap = pool;
  ctl.ppt = tile_ppt;
  MG_CHECK_BATCH(cudaMemcpyAsync(base + o_inst, host.data(), W * sizeof(BatchInst), cudaMemcpyHostToDevice, b->stream));
  if (!terms.empty())
    MG_CHECK_BATCH(cudaMemcpyAsync(base + o_terms, terms.data(), terms.size() * sizeof(Term), cudaMemcpyHostToDevice, b->stream));
  MG_CHECK_BATCH(cudaMemcpyAsync(base + o_tbegin, tbegin.data(), tbegin.size() * 4, cudaMemcpyHostToDevice, b->stream));
  if (!inverse.empty())
    MG_CHECK_BATCH(cudaMemcpyAsync(base + o_inv, inverse.data(), inverse.size() * 4, cudaMemcpyHostToDevice, b->stream));
  if (!sels.empty())
    MG_CHECK_BATCH(cudaMemcpyAsync(base + o_sel, sels.data(), sels.size() * 4, cudaMemcpyHostToDevice, b->stream));
  MG_CHECK_BATCH(cudaMemcpyAsync(base + o_ctl, &ctl, sizeof(ctl), cudaMemcpyHostToDevice, b->stream));
  MG_CHECK_BATCH(cudaMemsetAsync(base + o_layers, 0, static_cast<size_t>(W) * max_depth * 8, b->stream));
  MG_CHECK_BATCH(cudaMemsetAsync(base + o_bitmap, 0, bitmap_words * 8, b->stream));
  BatchParams p{};
  p.inst = reinterpret_cast<BatchInst*>(base + o_inst);
  p.count = W;
  p.terms = reinterpret_cast<const Term*>(base + o_terms);
  p.tbegin = reinterpret_cast<const uint32_t*>(base + o_tbegin);
  p.inverse = reinterpret_cast<const uint32_t*>(base + o_inv);
  p.sel = reinterpret_cast<const uint32_t*>(base + o_sel);
  p.bitmap = reinterpret_cast<unsigned long long*>(base + o_bitmap);
  p.buf[0] = reinterpret_cast<unsigned long long*>(base + o_buf0);
  p.buf[1] = reinterpret_cast<unsigned long long*>(base + o_buf1);
  p.tile_prefix = reinterpret_cast<unsigned long long*>(base + o_prefix);
  p.cur_count = reinterpret_cast<unsigned long long*>(base + o_cur);
  p.next_count = reinterpret_cast<unsigned long long*>(base + o_next);
  p.layers = reinterpret_cast<unsigned long long*>(base + o_layers);
  p.layer_step = reinterpret_cast<uint32_t*>(base + o_step);
  p.stamps = reinterpret_cast<unsigned long long*>(base + o_stamps);
  p.reloc = reinterpret_cast<BatchReloc*>(base + o_reloc);
  p.ctl = reinterpret_cast<BatchCtl*>(base + o_ctl);
  batch_seed<<<std::max<uint32_t>(1, (W + 255) / 256), 256, 0, b->stream>>>(p);
  ++st->kernel_launches;
  // The carveout is sized for the tuned resident blocks of batch_expand (0 =
  // the default) and the rest left as L1.
  const int want = blocks_per_sm ? static_cast<int>(blocks_per_sm) : kBatchBlocksPerSM;
  const int per_sm = size_carveout(reinterpret_cast<const void*>(batch_expand), 0, want, kBatchBlock);
  const uint32_t grid = static_cast<uint32_t>(per_sm * b->sm_count);
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaEventRecord(e0, b->stream);
  uint32_t layers_run = 0;
  if (loop == kLoopPersistent) {
    // One cooperative launch; its grid must be co-resident, so it is sized by
    // the occupancy of batch_wave itself under the carveout set above.
    int wave_sm = size_carveout(reinterpret_cast<const void*>(batch_wave), 0, want, kBatchBlock);
    int resident = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&resident, batch_wave, kBatchBlock, 0) != cudaSuccess) {
      cudaGetLastError();
      resident = 1;
    }
    wave_sm = std::max(1, std::min(wave_sm, resident));
    void* args[] = {&p};
    cudaError_t e = cudaErrorCooperativeLaunchTooLarge;
    for (; wave_sm >= 1 && e == cudaErrorCooperativeLaunchTooLarge; --wave_sm) {
      e = cudaLaunchCooperativeKernel(reinterpret_cast<const void*>(batch_wave), dim3(wave_sm * b->sm_count),
                                      dim3(kBatchBlock), args, 0, b->stream);
      if (e == cudaErrorCooperativeLaunchTooLarge) cudaGetLastError();
    }
    MG_CHECK_BATCH(e);
    ++st->kernel_launches;
    MG_CHECK_BATCH(cudaStreamSynchronize(b->stream));
  } else if (loop == kLoopGraph) {
    cudaGraph_t graph;
    MG_CHECK_BATCH(cudaGraphCreate(&graph, 0));
    cudaGraphConditionalHandle handle;
    MG_CHECK_BATCH(cudaGraphConditionalHandleCreate(&handle, graph, 1, cudaGraphCondAssignDefault));
    cudaGraphNodeParams cp = {};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = handle;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    cudaGraphNode_t node;
    MG_CHECK_BATCH(cudaGraphAddNode(&node, graph, nullptr, 0, &cp));
    cudaGraph_t body = cp.conditional.phGraph_out[0];
    cudaStream_t cap_stream;
    MG_CHECK_BATCH(cudaStreamCreateWithFlags(&cap_stream, cudaStreamNonBlocking));
    MG_CHECK_BATCH(cudaStreamBeginCaptureToGraph(cap_stream, body, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed));
    batch_expand<<<grid, kBatchBlock, 0, cap_stream>>>(p);
    batch_finalize<<<1, 1024, 0, cap_stream>>>(p, handle, 1);
    batch_relocate<<<grid, kBatchBlock, 0, cap_stream>>>(p);
    MG_CHECK_BATCH(cudaStreamEndCapture(cap_stream, &body));
    cudaGraphExec_t exec;
    MG_CHECK_BATCH(cudaGraphInstantiate(&exec, graph, 0));
    MG_CHECK_BATCH(cudaGraphLaunch(exec, b->stream));
    ++st->graph_launches;
    MG_CHECK_BATCH(cudaStreamSynchronize(b->stream));
    cudaGraphExecDestroy(exec);
    cudaGraphDestroy(graph);
    cudaStreamDestroy(cap_stream);
  } else {
    for (;;) {
      batch_expand<<<grid, kBatchBlock, 0, b->stream>>>(p);
      batch_finalize<<<1, 1024, 0, b->stream>>>(p, cudaGraphConditionalHandle{}, 0);
      batch_relocate<<<grid, kBatchBlock, 0, b->stream>>>(p);
      st->kernel_launches += 3;
      BatchCtl h{};
      MG_CHECK_BATCH(cudaMemcpyAsync(&h, p.ctl, sizeof(h), cudaMemcpyDeviceToHost, b->stream));
      MG_CHECK_BATCH(cudaStreamSynchronize(b->stream));
      ++layers_run;
      if (!h.total) break;
    }
  }
  cudaEventRecord(e1, b->stream);
  cudaEventSynchronize(e1);
  float ms = 0;
  cudaEventElapsedTime(&ms, e0, e1);
  *kernel_seconds += ms * 1e-3;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  // Results.  The instance records come first: their deepest layer bounds
  // the columns of the layer and step tables that are read back (a strided
  // copy of depth + 1 columns instead of max_depth).
  std::vector<BatchInst> done(W);
  BatchCtl hc{};
  MG_CHECK_BATCH(cudaMemcpyAsync(done.data(), p.inst, W * sizeof(BatchInst), cudaMemcpyDeviceToHost, b->stream));
  MG_CHECK_BATCH(cudaMemcpyAsync(&hc, p.ctl, sizeof(hc), cudaMemcpyDeviceToHost, b->stream));
  std::vector<unsigned long long> stamps(static_cast<size_t>(max_steps) + 1, 0);
  MG_CHECK_BATCH(cudaMemcpyAsync(stamps.data(), p.stamps, stamps.size() * 8, cudaMemcpyDeviceToHost, b->stream));
  MG_CHECK_BATCH(cudaStreamSynchronize(b->stream));
  uint32_t cols = 1;
  for (uint32_t k = 0; k < W; ++k) cols = std::max(cols, std::min(done[k].depth + 1, max_depth));
  std::vector<unsigned long long> layers(static_cast<size_t>(W) * cols);
  std::vector<uint32_t> steps(static_cast<size_t>(W) * cols);
  MG_CHECK_BATCH(cudaMemcpy2DAsync(layers.data(), cols * 8ull, p.layers, max_depth * 8ull, cols * 8ull, W,
                                   cudaMemcpyDeviceToHost, b->stream));
  MG_CHECK_BATCH(cudaMemcpy2DAsync(steps.data(), cols * 4ull, p.layer_step, max_depth * 4ull, cols * 4ull, W,
                                   cudaMemcpyDeviceToHost, b->stream));
  MG_CHECK_BATCH(cudaStreamSynchronize(b->stream));
  if (loop == kLoopGraph) st->kernel_launches += 3 * hc.step;
  st->layer_steps += hc.step;
  st->redo_layers += hc.redo_layers;
  for (uint32_t k = 0; k < W; ++k) {
    auto& in = b->inst[ids[k]];
    in.status = done[k].status;
    in.runs++;
    in.layers.clear();
    in.layer_seconds.clear();
    if (in.status == INST_DONE) {
      for (uint32_t d = 0; d < cols && layers[static_cast<size_t>(k) * cols + d]; ++d) {
        in.layers.push_back(layers[static_cast<size_t>(k) * cols + d]);
        // Layer d >= 1 came from the wave's step t (shared by the wave's
        // instances, stamped at its end); depth 0 is the seed.
        double dt = 0.0;
        if (d) {
          const uint32_t t = steps[static_cast<size_t>(k) * cols + d];
          if (t < max_steps && stamps[t + 1] > stamps[t]) dt = (stamps[t + 1] - stamps[t]) * 1e-9;
        }
        in.layer_seconds.push_back(dt);
      }
    }
  }
  if (hc.error) st->fatal |= hc.error;
  return MGBFS2_OK;
}

}  // namespace mgbfs2

using mgbfs2::Batch;

struct mgbfs2_batch {
  Batch* impl;
};

extern "C" {

int mgbfs2_batch_create(const mgbfs2_graph_desc* graphs, uint32_t count, int device, mgbfs2_batch** out, char* error,
                        size_t error_capacity) {
  if (!out) return MGBFS2_INVALID_ARGUMENT;
  *out = nullptr;
  Batch* b = nullptr;
  const int rc = mgbfs2::batch_create(graphs, count, device, &b, error, error_capacity);
  if (rc) return rc;
  *out = new mgbfs2_batch{b};
  return MGBFS2_OK;
}

int mgbfs2_batch_run(mgbfs2_batch* batch, const mgbfs2_batch_options* options, mgbfs2_batch_status* status) {
  using namespace mgbfs2;
  if (!batch) return MGBFS2_INVALID_ARGUMENT;
  Batch* b = batch->impl;
  mgbfs2_batch_options o{};
  if (options) o = *options;
  const uint32_t max_depth = o.max_depth ? o.max_depth : 1024;
  const uint32_t blocks_per_sm = o.blocks_per_sm;
  const uint32_t loop = o.host_loop;
  if (loop > kLoopGraph) return MGBFS2_INVALID_ARGUMENT;
  const uint32_t tile = o.tile_entries ? o.tile_entries : kBatchTile;
  if (tile != kBatchBlock && tile != 2 * kBatchBlock && tile != 4 * kBatchBlock) return MGBFS2_INVALID_ARGUMENT;
  const uint32_t tile_ppt = tile / kBatchBlock;
  MG_CHECK_BATCH(cudaSetDevice(b->device));
  size_t free_bytes = 0;
  if (int frc = device_free_bytes(b->device, &free_bytes)) return frc;
  free_bytes += pool_idle_bytes(b->device) + device_cache_bytes(b->device) + b->arena.bytes;
  const uint64_t reserve = o.reserve_bytes ? o.reserve_bytes : (2ull << 30);
  uint64_t budget = o.memory_bytes ? o.memory_bytes : (free_bytes > reserve ? free_bytes - reserve : 0);
  mgbfs2_batch_status st{};
  const auto started = std::chrono::steady_clock::now();
  double kernel_seconds = 0.0;
  const uint32_t I = static_cast<uint32_t>(b->inst.size());
  // Capacities: the plain planner reserves each instance's orbit bound; a
  // caller-provided prediction (the learned planner) reserves less, and an
  // instance that overflows it is rerun with the plain bound.
  std::vector<uint64_t> cap(I);
  for (uint32_t i = 0; i < I; ++i) {
    cap[i] = b->inst[i].orbit;
    if (o.predicted_capacity && o.predicted_capacity[i] > 0)
      cap[i] = std::min<uint64_t>(cap[i], o.predicted_capacity[i]);
    b->inst[i].status = INST_IDLE;
    b->inst[i].runs = 0;
    b->inst[i].layers.clear();
  }
  std::vector<uint32_t> pending(I);
  for (uint32_t i = 0; i < I; ++i) pending[i] = i;
  int rc = MGBFS2_OK;
  while (!pending.empty() && !rc) {
    // Fill a wave up to the memory budget (bitmap + two segments + tables).
    // Waves whose capacities are predictions keep an eighth of the budget as
    // the redo pool: an instance whose layer outgrows its segment moves to a
    // larger one from there and redoes that layer only.
    std::vector<uint32_t> wave;
    std::vector<uint64_t> caps;
    uint64_t used = 1 << 20, short_by = 0, orbits = 0;
    bool predicted = false;
    for (uint32_t i : pending) predicted = predicted || cap[i] < b->inst[i].orbit;
    const uint64_t fill = predicted ? budget - budget / 8 : budget;
    std::vector<uint32_t> later;
    for (uint32_t i : pending) {
      const uint64_t need = (b->inst[i].orbit + 63) / 64 * 8 + 2 * (cap[i] + 1) * 8 + 12ull * max_depth + 160;
      if (wave.empty() || used + need <= fill) {
        wave.push_back(i);
        caps.push_back(cap[i]);
        used += need;
        short_by += b->inst[i].orbit - cap[i];
        orbits += b->inst[i].orbit;
      } else {
        later.push_back(i);
      }
    }
    // Pool entries (both buffers): what is left of the budget, at most twice
    // the wave's orbits.  An instance redoes each layer at most once, with a
    // segment of that layer's winner count (a state won again after a winner
    // released its bit counts again), so its redo segments rarely sum to more
    // than twice its orbit; a pool that runs out falls back to the rerun.
    const uint64_t pool = predicted && short_by && budget > used ? std::min((budget - used) / 16, 2 * orbits) : 0;
    rc = run_wave(b, wave, caps, pool, max_depth, blocks_per_sm, tile_ppt, loop, &st, &kernel_seconds);
    ++st.waves;
    for (uint32_t i : wave) {
      if (b->inst[i].status == INST_OVERFLOW) {
        if (cap[i] >= b->inst[i].orbit) {
          rc = MGBFS2_CAPACITY;  // cannot happen with the orbit bound; keeps the loop finite
          break;
        }
        cap[i] = b->inst[i].orbit;  // exact rerun with the plain bound
        ++st.redo_instances;
        later.push_back(i);
      }
    }
    pending.swap(later);
  }
  for (uint32_t i = 0; i < I; ++i) {
    for (uint64_t s : b->inst[i].layers) st.states += s;
    st.successors += [&] {
      uint64_t e = 0;
      for (uint64_t s : b->inst[i].layers) e += s * b->inst[i].gens;
      return e;
    }();
    if (b->inst[i].status == INST_DONE) ++st.complete_instances;
  }
  st.instances = I;
  st.seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - started).count();
  st.device_seconds = kernel_seconds;
  b->last = st;
  if (status) *status = st;
  return rc;
}

int mgbfs2_batch_layer_table(const mgbfs2_batch* batch, uint32_t instance, uint64_t* sizes, size_t capacity,
                             size_t* count) {
  if (!batch || !count || instance >= batch->impl->inst.size()) return MGBFS2_INVALID_ARGUMENT;
  const auto& layers = batch->impl->inst[instance].layers;
  *count = layers.size();
  for (size_t d = 0; d < layers.size() && d < capacity; ++d)
    if (sizes) sizes[d] = layers[d];
  return MGBFS2_OK;
}

int mgbfs2_batch_layer_tables(const mgbfs2_batch* batch, uint64_t* tables, uint64_t capacity, uint64_t* offsets) {
  if (!batch || !offsets) return MGBFS2_INVALID_ARGUMENT;
  const auto& inst = batch->impl->inst;
  uint64_t run = 0;
  for (size_t i = 0; i < inst.size(); ++i) {
    offsets[i] = run;
    run += inst[i].layers.size();
  }
  offsets[inst.size()] = run;
  if (!tables) return MGBFS2_OK;
  if (capacity < run) return MGBFS2_CAPACITY;
  for (size_t i = 0; i < inst.size(); ++i)
    std::copy(inst[i].layers.begin(), inst[i].layers.end(), tables + offsets[i]);
  return MGBFS2_OK;
}

int mgbfs2_batch_layer_seconds(const mgbfs2_batch* batch, uint32_t instance, double* seconds, size_t capacity,
                               size_t* count) {
  if (!batch || !count || instance >= batch->impl->inst.size()) return MGBFS2_INVALID_ARGUMENT;
  const auto& t = batch->impl->inst[instance].layer_seconds;
  *count = t.size();
  for (size_t d = 0; d < t.size() && d < capacity; ++d)
    if (seconds) seconds[d] = t[d];
  return MGBFS2_OK;
}

void mgbfs2_batch_destroy(mgbfs2_batch* batch) {
  if (!batch) return;
  Batch* b = batch->impl;
  cudaSetDevice(b->device);
  // Nothing of the batch is in flight after this: the arena goes to the
  // device cache, where the next batch or graph handle takes it.
  if (b->stream) cudaStreamSynchronize(b->stream);
  b->arena.release_to_cache(b->device);
  if (b->stream) cudaStreamDestroy(b->stream);
  delete b;
  delete batch;
}

}  // extern "C"
