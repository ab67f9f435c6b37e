// Wide-key path: states of K uint64 words (int64 matrices, or permutations
// whose codes do not fit one packed word).  All visited states are retained
// as rows of a device arena; a layer is a contiguous row range, so appending a
// new state IS the next-frontier append.  The visited set is an
// open-addressing table of 64-bit tokens
//     bit 63 pending | bits 40..62 fingerprint | bits 0..39 arena row
// and equality is always decided on the full key (word-by-word compare with
// the arena row).  Children are never materialised before the probe: every
// word is regenerated from the parent on demand.
//
// Reference counterpart: accept_candidates, cuda/generic_visited.cu:18-58
// (31-bit hash prefix + row token, pending bit, exact element compare), the
// retained arena of crates/mgbfs-runtime/src/generic_native.rs:31-57, and the
// matrix action of cuda/generic_graph.cu:7-36 / graph_definition.py:77-83.
#include <algorithm>
#include <chrono>
#include <cstring>

#include "engine.h"

namespace mgbfs2 {

namespace {

constexpr unsigned long long kPending = 1ull << 63;
constexpr unsigned long long kRowMask = (1ull << 40) - 1;
constexpr unsigned long long kFailedRow = kRowMask - 1;
// Row field of a pending claim.  It must not be kRowMask: with an all-ones
// fingerprint that claim would equal kEmpty, a second thread would take the
// still "empty" slot for the same key, and the state would be stored twice.
constexpr unsigned long long kClaimRow = kRowMask - 2;
constexpr uint32_t kFpShift = 40;
constexpr unsigned long long kFpMask = (1ull << 23) - 1;
static_assert((kPending | (kFpMask << kFpShift) | kClaimRow) != kEmpty, "a pending claim must never read as empty");
constexpr uint32_t kWaitLimit = 1u << 22;
constexpr uint32_t kWideBlock = 256;

struct WideParams {
  unsigned long long* arena;
  unsigned long long parent_begin, parent_count;
  unsigned long long* arena_count;
  unsigned long long arena_capacity;
  uint32_t K, kind, elements, rows, cols, gens, bits, pad;
  const uint32_t* perms;
  const int64_t* mats;
  const uint32_t* mods;
  unsigned long long* table;
  unsigned long long mask;
  unsigned int* error;
};

__device__ __forceinline__ uint64_t child_word(const WideParams& p, const unsigned long long* parent, uint32_t g,
                                               uint32_t j) {
  if (p.kind == 1) {
    const uint32_t i = j / p.cols, c = j % p.cols;
    const int64_t* m = p.mats + static_cast<size_t>(g) * p.rows * p.rows + static_cast<size_t>(i) * p.rows;
    uint64_t total = 0;  // int64 multiply-add wraps exactly as uint64
    for (uint32_t k = 0; k < p.rows; ++k)
      total += static_cast<uint64_t>(m[k]) * parent[static_cast<size_t>(k) * p.cols + c];
    int64_t v = static_cast<int64_t>(total);
    const uint32_t mod = p.mods[g];
    if (mod) {
      v %= static_cast<int64_t>(mod);
      if (v < 0) v += mod;
    }
    return static_cast<uint64_t>(v);
  }
  const uint32_t* perm = p.perms + static_cast<size_t>(g) * p.elements;
  if (p.bits == 64) return parent[perm[j]];
  const uint32_t per = 64 / p.bits;
  const uint64_t sym = (1ull << p.bits) - 1;
  uint64_t w = 0;
  for (uint32_t s = 0; s < per; ++s) {
    const uint32_t i = j * per + s;
    if (i >= p.elements) break;
    const uint32_t src = perm[i];
    w |= ((parent[src / per] >> ((src % per) * p.bits)) & sym) << (s * p.bits);
  }
  return w;
}

__device__ __forceinline__ uint64_t fold_hash(uint64_t h, uint64_t w, uint32_t j) {
  return mix64(h ^ mix64(w + 0x9e3779b97f4a7c15ull * (j + 1)));
}

__global__ void __launch_bounds__(kWideBlock) wide_expand(WideParams p) {
  const unsigned long long total = p.parent_count * p.gens;
  for (unsigned long long idx = blockIdx.x * static_cast<unsigned long long>(blockDim.x) + threadIdx.x; idx < total;
       idx += static_cast<unsigned long long>(gridDim.x) * blockDim.x) {
    const unsigned long long par = p.parent_begin + idx / p.gens;
    const uint32_t g = static_cast<uint32_t>(idx % p.gens);
    const unsigned long long* parent = p.arena + par * p.K;
    uint64_t h = 0x19f856a2ull;
    for (uint32_t j = 0; j < p.K; ++j) h = fold_hash(h, child_word(p, parent, g, j), j);
    const unsigned long long fp = (h >> 41) & kFpMask;
    unsigned long long slot = h & p.mask;
    for (unsigned long long probe = 0; probe <= p.mask; ++probe, slot = (slot + 1) & p.mask) {
      unsigned long long cur = *reinterpret_cast<volatile unsigned long long*>(&p.table[slot]);
      if (cur == kEmpty) {
        const unsigned long long claim = kPending | (fp << kFpShift) | kClaimRow;
        const unsigned long long prev = atomicCAS(&p.table[slot], kEmpty, claim);
        if (prev == kEmpty) {
          const unsigned long long row = atomicAdd(p.arena_count, 1ull);
          if (row >= p.arena_capacity) {
            atomicOr(p.error, ERR_ARENA_OVERFLOW);
            atomicExch(&p.table[slot], (fp << kFpShift) | kFailedRow);
            break;
          }
          for (uint32_t j = 0; j < p.K; ++j) p.arena[row * p.K + j] = child_word(p, parent, g, j);
          __threadfence();
          atomicExch(&p.table[slot], (fp << kFpShift) | row);
          break;
        }
        cur = prev;
      }
      if (((cur >> kFpShift) & kFpMask) != fp) continue;
      uint32_t spins = 0;
      while (cur & kPending) {
        if (++spins > kWaitLimit) {
          atomicOr(p.error, ERR_WAIT_LIMIT);
          break;
        }
        __nanosleep(64);
        cur = *reinterpret_cast<volatile unsigned long long*>(&p.table[slot]);
      }
      if (cur & kPending) break;  // gave up; the layer is reported as failed
      const unsigned long long row = cur & kRowMask;
      if (row == kFailedRow) continue;
      __threadfence();
      bool equal = true;
      for (uint32_t j = 0; j < p.K && equal; ++j)
        equal = child_word(p, parent, g, j) == __ldcg(&p.arena[row * p.K + j]);
      if (equal) break;
    }
  }
}

// Rebuilds the token table from the arena rows [0, rows).
__global__ void wide_rehash(const unsigned long long* arena, unsigned long long rows, uint32_t K,
                            unsigned long long* table, unsigned long long mask, unsigned int* error) {
  for (unsigned long long r = blockIdx.x * static_cast<unsigned long long>(blockDim.x) + threadIdx.x; r < rows;
       r += static_cast<unsigned long long>(gridDim.x) * blockDim.x) {
    uint64_t h = 0x19f856a2ull;
    for (uint32_t j = 0; j < K; ++j) h = fold_hash(h, arena[r * K + j], j);
    const unsigned long long token = (((h >> 41) & kFpMask) << kFpShift) | r;
    unsigned long long slot = h & mask;
    bool placed = false;
    for (unsigned long long probe = 0; probe <= mask; ++probe, slot = (slot + 1) & mask)
      if (atomicCAS(&table[slot], kEmpty, token) == kEmpty) {
        placed = true;
        break;
      }
    if (!placed) atomicOr(error, ERR_TABLE_FULL);
  }
}

uint64_t next_pow2_u64(uint64_t x) {
  uint64_t p = 1;
  while (p < x) p <<= 1;
  return p;
}

}  // namespace

struct WideState {
  DeviceBuffer arena, table, perms, mats, mods, counters;
  uint64_t arena_rows = 0, slots = 0;
  uint32_t K = 0, bits = 64;
  std::vector<uint64_t> start_words;
  uint64_t last_begin = 0, last_count = 0, prev_begin = 0, prev_count = 0;
  bool have_prev = false;
};

uint32_t Graph::wide_key_words() const {
  if (kind == 1) return elements;
  uint32_t b = 8;
  while (b < 64 && (1ull << b) < distinct) b *= 2;
  return static_cast<uint32_t>((static_cast<uint64_t>(elements) * b + 63) / 64);
}

int Graph::wide_plan(mgbfs2_plan_info* p, uint64_t budget) {
  if (p->visited != MGBFS2_VISITED_HASH && p->visited != MGBFS2_VISITED_HASH3) return MGBFS2_UNSUPPORTED;
  // Retained rows make the all-visited table exact for directed and
  // inverse-closed graphs alike.
  p->visited = MGBFS2_VISITED_HASH;
  p->history_layers = 1;
  p->dedup = MGBFS2_DEDUP_ATOMIC;
  if (!wide) {
    wide = new WideState();
    for (DeviceBuffer* b : {&wide->arena, &wide->table, &wide->perms, &wide->mats, &wide->mods, &wide->counters})
      b->stream = stream;
  }
  WideState& w = *wide;
  w.K = wide_key_words();
  w.bits = 64;
  if (kind == 0) {
    w.bits = 8;
    while (w.bits < 64 && (1ull << w.bits) < distinct) w.bits *= 2;
  }
  p->key_words = w.K;
  p->bits_per_symbol = w.bits;
  const uint64_t row_bytes = 8ull * w.K;
  const uint64_t per_state = row_bytes + 16;  // arena row + table slots at load <= 1/2
  uint64_t cap = state_bound ? state_bound : UINT64_MAX;
  cap = std::min<uint64_t>(cap, budget / per_state);
  cap = std::min<uint64_t>(cap, kClaimRow);  // rows stay below kClaimRow and kFailedRow
  if (!cap) return MGBFS2_OUT_OF_MEMORY;
  p->capacity = std::min(p->capacity, cap);
  p->table_slots = std::max<uint64_t>(1024, next_pow2_u64(2 * std::min<uint64_t>(cap, 1ull << 20)));
  p->device_bytes = 0;
  // Start row packed with the same word layout the kernel produces.
  w.start_words.assign(w.K, 0);
  if (kind == 1) {
    for (uint32_t i = 0; i < elements; ++i) w.start_words[i] = static_cast<uint64_t>(start[i]);
  } else {
    const uint32_t per = 64 / w.bits;
    for (uint32_t i = 0; i < elements; ++i)
      w.start_words[i / per] |= (w.bits == 64 ? static_cast<uint64_t>(codes[i])
                                              : static_cast<uint64_t>(codes[i]) << ((i % per) * w.bits));
  }
  int rc = MGBFS2_OK;
  if (kind == 0) {
    if ((rc = w.perms.ensure(perms.size() * 4 + 4))) return rc;
    if (cudaMemcpyAsync(w.perms.ptr, perms.data(), perms.size() * 4, cudaMemcpyHostToDevice, stream) != cudaSuccess)
      return MGBFS2_CUDA_BASE;
  } else {
    if ((rc = w.mats.ensure(matrices.size() * 8 + 8)) || (rc = w.mods.ensure(moduli.size() * 4 + 4))) return rc;
    if (cudaMemcpyAsync(w.mats.ptr, matrices.data(), matrices.size() * 8, cudaMemcpyHostToDevice, stream) !=
            cudaSuccess ||
        cudaMemcpyAsync(w.mods.ptr, moduli.data(), moduli.size() * 4, cudaMemcpyHostToDevice, stream) != cudaSuccess)
      return MGBFS2_CUDA_BASE;
  }
  if ((rc = w.counters.ensure(16))) return rc;
  return cuda_status(cudaStreamSynchronize(stream));
}

int Graph::wide_run(const mgbfs2_run_limits* limits, mgbfs2_layer_callback cb, void* user, mgbfs2_status* status) {
  using Clock = std::chrono::steady_clock;
  WideState& w = *wide;
  mgbfs2_status st{};
  layer_sizes.assign(1, 1);
  layer_seconds.clear();
  launches = 0;
  const auto started = Clock::now();
  int rc = MGBFS2_OK;
  // counters: [0] arena rows used (u64), [8] error (u32)
  unsigned long long* d_rows = static_cast<unsigned long long*>(w.counters.ptr);
  unsigned int* d_error = reinterpret_cast<unsigned int*>(static_cast<char*>(w.counters.ptr) + 8);
  w.slots = plan.table_slots;
  if ((rc = w.table.ensure(w.slots * 8))) return rc;
  w.arena_rows = std::max<uint64_t>(1024, std::min<uint64_t>(plan.capacity, 1ull << 16));
  if ((rc = w.arena.ensure(w.arena_rows * w.K * 8))) return rc;
  if (cudaMemsetAsync(w.table.ptr, 0xff, w.slots * 8, stream) != cudaSuccess) return MGBFS2_CUDA_BASE;
  if (cudaMemcpyAsync(w.arena.ptr, w.start_words.data(), w.K * 8, cudaMemcpyHostToDevice, stream) != cudaSuccess)
    return MGBFS2_CUDA_BASE;
  const unsigned long long one = 1;
  if (cudaMemsetAsync(w.counters.ptr, 0, 16, stream) != cudaSuccess) return MGBFS2_CUDA_BASE;
  // Seed the start row's token through the rehash kernel (rows [0, 1)).
  wide_rehash<<<1, 32, 0, stream>>>(static_cast<const unsigned long long*>(w.arena.ptr), 1, w.K,
                                    static_cast<unsigned long long*>(w.table.ptr), w.slots - 1, d_error);
  ++launches;
  if (cudaMemcpyAsync(d_rows, &one, 8, cudaMemcpyHostToDevice, stream) != cudaSuccess) return MGBFS2_CUDA_BASE;
  uint64_t begin = 0, count = 1, visited = 1;
  uint32_t depth = 0;
  w.have_prev = false;
  w.prev_begin = w.prev_count = 0;
  st.reason = MGBFS2_REASON_FRONTIER_EXHAUSTED;
  uint64_t peak = 0;
  for (;;) {
    const double elapsed = std::chrono::duration<double>(Clock::now() - started).count();
    if (limits && limits->cancel && *limits->cancel) { st.reason = MGBFS2_REASON_CANCELLED; break; }
    if (limits && limits->max_seconds > 0 && elapsed >= limits->max_seconds) { st.reason = MGBFS2_REASON_DEADLINE; break; }
    if (limits && limits->max_layers && layer_sizes.size() >= limits->max_layers) {
      st.reason = MGBFS2_REASON_LAYER_LIMIT;
      break;
    }
    const auto layer_start = Clock::now();
    const uint64_t bound = std::min<uint64_t>(next_bound(depth, count, visited), plan.capacity);
    // Arena growth keeps every retained row (device-to-device copy).
    if (visited + bound > w.arena_rows) {
      const uint64_t rows = std::max<uint64_t>(visited + bound, 2 * w.arena_rows);
      DeviceBuffer grown;
      grown.stream = stream;
      if ((rc = grown.ensure(rows * w.K * 8))) break;
      if (cudaMemcpyAsync(grown.ptr, w.arena.ptr, visited * w.K * 8, cudaMemcpyDeviceToDevice, stream) != cudaSuccess) {
        grown.free();
        rc = MGBFS2_CUDA_BASE;
        break;
      }
      if (cudaStreamSynchronize(stream) != cudaSuccess) { grown.free(); rc = MGBFS2_CUDA_BASE; break; }
      w.arena.free();
      w.arena = grown;
      w.arena_rows = rows;
    }
    // Keep the token table at most half full after the layer.
    if (2 * (visited + bound) > w.slots) {
      const uint64_t slots = next_pow2_u64(2 * (visited + bound));
      if ((rc = w.table.ensure(slots * 8))) break;
      w.slots = slots;
      if (cudaMemsetAsync(w.table.ptr, 0xff, slots * 8, stream) != cudaSuccess) { rc = MGBFS2_CUDA_BASE; break; }
      const uint32_t blocks = static_cast<uint32_t>(std::min<uint64_t>((visited + 255) / 256, 65535));
      wide_rehash<<<blocks, 256, 0, stream>>>(static_cast<const unsigned long long*>(w.arena.ptr), visited, w.K,
                                              static_cast<unsigned long long*>(w.table.ptr), slots - 1, d_error);
      ++launches;
    }
    WideParams p{};
    p.arena = static_cast<unsigned long long*>(w.arena.ptr);
    p.parent_begin = begin;
    p.parent_count = count;
    p.arena_count = d_rows;
    p.arena_capacity = std::min<uint64_t>(w.arena_rows, visited + bound);
    p.K = w.K;
    p.kind = kind;
    p.elements = elements;
    p.rows = rows;
    p.cols = cols;
    p.gens = gens;
    p.bits = w.bits;
    p.perms = static_cast<const uint32_t*>(w.perms.ptr);
    p.mats = static_cast<const int64_t*>(w.mats.ptr);
    p.mods = static_cast<const uint32_t*>(w.mods.ptr);
    p.table = static_cast<unsigned long long*>(w.table.ptr);
    p.mask = w.slots - 1;
    p.error = d_error;
    const uint64_t work = count * gens;
    const uint32_t blocks = grid_for(reinterpret_cast<const void*>(wide_expand), 0, (work + kWideBlock - 1) / kWideBlock);
    wide_expand<<<blocks, kWideBlock, 0, stream>>>(p);
    ++launches;
    if (cudaGetLastError() != cudaSuccess) { rc = MGBFS2_CUDA_BASE; break; }
    unsigned long long host[2] = {0, 0};
    if (cudaMemcpyAsync(host, w.counters.ptr, 16, cudaMemcpyDeviceToHost, stream) != cudaSuccess ||
        cudaStreamSynchronize(stream) != cudaSuccess) {
      rc = MGBFS2_CUDA_BASE;
      break;
    }
    st.successors += work;
    peak = std::max<uint64_t>(peak, w.arena.bytes + w.table.bytes);
    const unsigned int err = static_cast<unsigned int>(host[1] & 0xffffffffu);
    if (err) {
      st.reason = MGBFS2_REASON_RESOURCE;
      st.fatal = err;
      break;
    }
    const uint64_t produced = host[0] - visited;
    if (produced == 0) {
      st.complete = 1;
      break;
    }
    const double secs = std::chrono::duration<double>(Clock::now() - layer_start).count();
    layer_sizes.push_back(produced);
    layer_seconds.push_back(secs);
    w.prev_begin = begin;
    w.prev_count = count;
    w.have_prev = true;
    begin = visited;
    count = produced;
    visited += produced;
    ++depth;
    if (cb && cb(user, depth, count, secs)) {
      st.reason = MGBFS2_REASON_CANCELLED;
      break;
    }
  }
  w.last_begin = begin;
  w.last_count = count;
  st.layers = static_cast<uint32_t>(layer_sizes.size());
  for (uint64_t s : layer_sizes) st.states += s;
  st.bfs_seconds = std::chrono::duration<double>(Clock::now() - started).count();
  st.kernel_launches = launches;
  st.peak_device_bytes = peak;
  if (status) *status = st;
  return rc;
}

int Graph::wide_sample(uint32_t which, int64_t* out, size_t cap_rows, size_t* rows) {
  WideState& w = *wide;
  uint64_t begin = w.last_begin, count = w.last_count;
  if (which == 1) {
    if (!w.have_prev || w.prev_count >= 1000) return MGBFS2_OK;
    begin = w.prev_begin;
    count = w.prev_count;
  }
  const uint64_t n = std::min<uint64_t>(count, cap_rows);
  std::vector<uint64_t> raw(n * w.K);
  if (n && (cudaMemcpyAsync(raw.data(), static_cast<uint64_t*>(w.arena.ptr) + begin * w.K, n * w.K * 8,
                            cudaMemcpyDeviceToHost, stream) != cudaSuccess ||
            cudaStreamSynchronize(stream) != cudaSuccess))
    return MGBFS2_CUDA_BASE;
  std::vector<std::vector<int64_t>> decoded(n, std::vector<int64_t>(elements));
  for (uint64_t r = 0; r < n; ++r) {
    const uint64_t* row = raw.data() + r * w.K;
    for (uint32_t i = 0; i < elements; ++i) {
      if (kind == 1) {
        decoded[r][i] = static_cast<int64_t>(row[i]);
      } else if (w.bits == 64) {
        decoded[r][i] = labels[row[i]];
      } else {
        const uint32_t per = 64 / w.bits;
        decoded[r][i] = labels[(row[i / per] >> ((i % per) * w.bits)) & ((1ull << w.bits) - 1)];
      }
    }
  }
  std::sort(decoded.begin(), decoded.end());
  for (uint64_t r = 0; r < n; ++r)
    if (out) std::memcpy(out + r * elements, decoded[r].data(), elements * sizeof(int64_t));
  *rows = n;
  return MGBFS2_OK;
}

void Graph::wide_release() {
  if (!wide) return;
  // Called from release(), after the stream was synchronised.
  for (DeviceBuffer* b : {&wide->arena, &wide->table, &wide->perms, &wide->mats, &wide->mods, &wide->counters})
    b->release_to_cache(device);
  delete wide;
  wide = nullptr;
}

}  // namespace mgbfs2
