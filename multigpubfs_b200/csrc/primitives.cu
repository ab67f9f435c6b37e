// Kernel-level entry points of libmgbfs2: each exposes one hot-path building
// block over caller-owned device buffers, for contract tests and for callers
// that assemble their own pipelines.  None of them allocates.
#include <algorithm>
#include <map>
#include <vector>

#include "../../include/mgbfs2.h"
#include "device.cuh"
#include "engine.h"
#include "sort_tiles.cuh"

namespace mgbfs2 {
namespace {

constexpr uint32_t kPrimBlock = 256;
constexpr uint32_t kMaxPackedGens = 64;
constexpr uint32_t kMaxPackedTerms = 1024;

struct PackedProgramArg {
  Term terms[kMaxPackedTerms];
  uint32_t begin[kMaxPackedGens + 1];
  uint32_t gens;
};

uint32_t blocks_for(uint64_t work) {
  return static_cast<uint32_t>(std::max<uint64_t>(1, std::min<uint64_t>((work + kPrimBlock - 1) / kPrimBlock, 148ull * 16)));
}

__global__ void successors_i64_kernel(uint32_t kind, uint32_t elements, uint32_t rows, uint32_t cols, uint32_t gens,
                                      const int64_t* parents, unsigned long long count, const uint32_t* perms,
                                      const int64_t* mats, const uint32_t* mods, int64_t* children,
                                      unsigned int* error) {
  const unsigned long long total = count * gens * elements;
  for (unsigned long long idx = blockIdx.x * static_cast<unsigned long long>(blockDim.x) + threadIdx.x; idx < total;
       idx += static_cast<unsigned long long>(gridDim.x) * blockDim.x) {
    const uint32_t e = static_cast<uint32_t>(idx % elements);
    const unsigned long long child = idx / elements;
    const unsigned long long p = child / gens;
    const uint32_t g = static_cast<uint32_t>(child % gens);
    const int64_t* parent = parents + p * elements;
    if (kind == 0) {
      const uint32_t src = perms[static_cast<size_t>(g) * elements + e];
      if (src >= elements) {
        if (error) atomicOr(error, ERR_BAD_STATE);
        children[idx] = 0;
        continue;
      }
      children[idx] = parent[src];
    } else {
      const uint32_t i = e / cols, c = e % cols;
      const int64_t* m = mats + static_cast<size_t>(g) * rows * rows + static_cast<size_t>(i) * rows;
      uint64_t sum = 0;
      for (uint32_t k = 0; k < rows; ++k) sum += static_cast<uint64_t>(m[k]) * static_cast<uint64_t>(parent[k * cols + c]);
      int64_t v = static_cast<int64_t>(sum);
      const uint32_t mod = mods[g];
      if (mod) {
        v %= static_cast<int64_t>(mod);
        if (v < 0) v += mod;
      }
      children[idx] = v;
    }
  }
}

__global__ void successors_packed_kernel(PackedProgramArg prog, const unsigned long long* parents,
                                         unsigned long long count, unsigned long long* children) {
  const unsigned long long total = count * prog.gens;
  for (unsigned long long idx = blockIdx.x * static_cast<unsigned long long>(blockDim.x) + threadIdx.x; idx < total;
       idx += static_cast<unsigned long long>(gridDim.x) * blockDim.x) {
    const uint32_t g = static_cast<uint32_t>(idx % prog.gens);
    children[idx] = apply_terms(parents[idx / prog.gens], prog.terms, prog.begin[g], prog.begin[g + 1]);
  }
}

__global__ void rank_kernel(MultisetDomain d, int lehmer, const unsigned long long* words, unsigned long long count,
                            unsigned long long* ranks, unsigned int* error) {
  for (unsigned long long i = blockIdx.x * static_cast<unsigned long long>(blockDim.x) + threadIdx.x; i < count;
       i += static_cast<unsigned long long>(gridDim.x) * blockDim.x) {
    uint64_t r = 0;
    bool ok;
    if (lehmer) {
      // Check the word is a permutation of 0..n-1 before the fast rank.
      uint32_t seen = 0;
      ok = true;
      for (uint32_t e = 0; e < d.n; ++e) {
        const uint32_t s = static_cast<uint32_t>(words[i] >> (4 * e)) & 15u;
        ok = ok && s < d.n && !(seen & (1u << s));
        seen |= 1u << s;
      }
      ok = ok && (d.n == 16 || (words[i] >> (4 * d.n)) == 0);
      if (ok) r = lehmer_rank4_n(words[i], d.n);
    } else {
      ok = multiset_rank(words[i], d, &r);
    }
    ranks[i] = ok ? r : ~0ull;
    if (!ok && error) atomicOr(error, ERR_RANK_RANGE);
  }
}

__global__ void product_rank_kernel(ProductDomain d, const unsigned long long* words, unsigned long long count,
                                    unsigned long long* ranks, unsigned int* error) {
  for (unsigned long long i = blockIdx.x * static_cast<unsigned long long>(blockDim.x) + threadIdx.x; i < count;
       i += static_cast<unsigned long long>(gridDim.x) * blockDim.x) {
    uint64_t r = 0;
    const bool ok = product_rank(words[i], d, &r);
    ranks[i] = ok ? r : ~0ull;
    if (!ok && error) atomicOr(error, ERR_RANK_RANGE);
  }
}

__global__ void bitmap_claim_kernel(const unsigned long long* ranks, unsigned long long count,
                                    unsigned long long* bitmap, unsigned long long domain, uint8_t* won, int warp,
                                    unsigned int* error) {
  const unsigned long long stride = static_cast<unsigned long long>(gridDim.x) * blockDim.x;
  const unsigned long long first = blockIdx.x * static_cast<unsigned long long>(blockDim.x) + threadIdx.x;
  // Uniform trip count per warp so the warp collectives see all 32 lanes.
  const unsigned long long warp_base = first - lane_id();
  for (unsigned long long base = warp_base; base < count; base += stride) {
    const unsigned long long i = base + lane_id();
    const bool valid = i < count;
    const uint64_t r = valid ? ranks[i] : 0;
    const bool ok = valid && r < domain;
    if (valid && !ok && error) atomicOr(error, ERR_RANK_RANGE);
    bool w = false;
    if (warp) {
      const unsigned active = __ballot_sync(kFullMask, ok);
      if (ok) {
        const unsigned long long word = r >> 6;
        const unsigned peers = __match_any_sync(active, word);
        const unsigned same = __match_any_sync(peers, static_cast<unsigned long long>(r));
        const unsigned long long bit = 1ull << (r & 63);
        const unsigned lo = __reduce_or_sync(peers, static_cast<unsigned>(bit));
        const unsigned hi = __reduce_or_sync(peers, static_cast<unsigned>(bit >> 32));
        const int leader = __ffs(peers) - 1;
        unsigned long long old = 0;
        if (static_cast<int>(lane_id()) == leader)
          old = atomicOr(&bitmap[word], (static_cast<unsigned long long>(hi) << 32) | lo);
        old = __shfl_sync(peers, old, leader);
        w = (static_cast<int>(lane_id()) == __ffs(same) - 1) && !(old & bit);
      }
    } else if (ok) {
      const unsigned long long bit = 1ull << (r & 63);
      w = !(atomicOr(&bitmap[r >> 6], bit) & bit);
    }
    if (valid) won[i] = w ? 1 : 0;
  }
}

__global__ void hash_insert_kernel(const unsigned long long* keys, unsigned long long count, unsigned long long* table,
                                   unsigned long long mask, uint8_t* inserted, unsigned int* error) {
  for (unsigned long long i = blockIdx.x * static_cast<unsigned long long>(blockDim.x) + threadIdx.x; i < count;
       i += static_cast<unsigned long long>(gridDim.x) * blockDim.x) {
    const unsigned long long k = keys[i];
    int rc = 0;
    if (k == kEmpty) {
      if (error) atomicOr(error, ERR_BAD_STATE);
    } else {
      rc = hash_insert(table, mask, k, ~0ull, 0, static_cast<uint32_t>(std::min<unsigned long long>(mask + 1, 1ull << 30)));
      if (rc < 0 && error) atomicOr(error, ERR_TABLE_FULL);
    }
    inserted[i] = rc == 1 ? 1 : 0;
  }
}

// Block-aggregated bucketing: one global reservation per (block, shard).
__global__ void bucket_kernel(const unsigned long long* keys, unsigned long long count, uint32_t shift,
                              uint32_t shards, unsigned long long* buckets, unsigned long long capacity,
                              unsigned long long* counts, unsigned int* error) {
  extern __shared__ unsigned long long shard_base[];  // shards entries, then shards u32 counters
  uint32_t* local = reinterpret_cast<uint32_t*>(shard_base + shards);
  const unsigned long long tile = blockDim.x;
  for (unsigned long long base = blockIdx.x * tile; base < count; base += gridDim.x * tile) {
    for (uint32_t s = threadIdx.x; s < shards; s += blockDim.x) local[s] = 0;
    __syncthreads();
    const unsigned long long i = base + threadIdx.x;
    uint32_t shard = 0, slot = 0;
    unsigned long long k = 0;
    const bool valid = i < count;
    if (valid) {
      k = keys[i];
      const unsigned long long s = k >> shift;
      if (s >= shards) {
        atomicOr(error, ERR_BAD_STATE);
        shard = UINT32_MAX;
      } else {
        shard = static_cast<uint32_t>(s);
        slot = atomicAdd(&local[shard], 1u);
      }
    }
    __syncthreads();
    for (uint32_t s = threadIdx.x; s < shards; s += blockDim.x)
      shard_base[s] = local[s] ? atomicAdd(&counts[s], static_cast<unsigned long long>(local[s])) : 0;
    __syncthreads();
    if (valid && shard != UINT32_MAX) {
      const unsigned long long pos = shard_base[shard] + slot;
      if (pos < capacity) buckets[shard * capacity + pos] = k;
      else atomicOr(error, ERR_BUCKET_OVERFLOW);
    }
    __syncthreads();
  }
}

}  // namespace

int build_packed_arg(uint32_t degree, uint32_t bits, uint32_t gens, const uint32_t* perms, PackedProgramArg* arg) {
  if (!perms || !degree || !gens || gens > kMaxPackedGens || (bits != 4 && bits != 8 && bits != 16 && bits != 32) ||
      static_cast<uint64_t>(degree) * bits > 64)
    return MGBFS2_INVALID_ARGUMENT;
  uint32_t nt = 0;
  arg->gens = gens;
  arg->begin[0] = 0;
  for (uint32_t k = 0; k < gens; ++k) {
    std::map<int, uint64_t> groups;
    std::vector<uint8_t> seen(degree, 0);
    for (uint32_t i = 0; i < degree; ++i) {
      const uint32_t src = perms[static_cast<size_t>(k) * degree + i];
      if (src >= degree || seen[src]) return MGBFS2_INVALID_ARGUMENT;
      seen[src] = 1;
      groups[static_cast<int>(src) - static_cast<int>(i)] |= ((1ull << bits) - 1) << (bits * i);
    }
    for (auto& kv : groups) {
      if (nt >= kMaxPackedTerms) return MGBFS2_INVALID_ARGUMENT;
      const int shift = kv.first * static_cast<int>(bits);
      arg->terms[nt].mask = kv.second;
      arg->terms[nt].rshift = shift > 0 ? shift : 0;
      arg->terms[nt].lshift = shift < 0 ? -shift : 0;
      ++nt;
    }
    arg->begin[k + 1] = nt;
  }
  return MGBFS2_OK;
}

}  // namespace mgbfs2

using namespace mgbfs2;

extern "C" {

int mgbfs2_successors_i64(uint32_t kind, uint32_t elements, uint32_t rows, uint32_t cols, uint32_t generators,
                          const int64_t* parents, uint64_t count, const uint32_t* permutations,
                          const int64_t* matrices, const uint32_t* moduli, int64_t* children, uint32_t* error,
                          void* stream) {
  if (kind > 1 || !elements || !generators || (count && (!parents || !children))) return MGBFS2_INVALID_ARGUMENT;
  if (kind == 0 && (!permutations || rows != elements || cols != 1)) return MGBFS2_INVALID_ARGUMENT;
  if (kind == 1 && (!matrices || !moduli || !rows || !cols || static_cast<uint64_t>(rows) * cols != elements))
    return MGBFS2_INVALID_ARGUMENT;
  if (!count) return MGBFS2_OK;
  const uint64_t work = count * generators * elements;
  successors_i64_kernel<<<blocks_for(work), kPrimBlock, 0, static_cast<cudaStream_t>(stream)>>>(
      kind, elements, rows, cols, generators, parents, count, permutations, matrices, moduli, children, error);
  return cuda_status(cudaGetLastError());
}

int mgbfs2_successors_packed(uint32_t degree, uint32_t bits, uint32_t generators, const uint32_t* permutations_host,
                             const uint64_t* parents, uint64_t count, uint64_t* children, void* stream) {
  static thread_local PackedProgramArg arg;
  int rc = build_packed_arg(degree, bits, generators, permutations_host, &arg);
  if (rc) return rc;
  if (!count) return MGBFS2_OK;
  if (!parents || !children) return MGBFS2_INVALID_ARGUMENT;
  successors_packed_kernel<<<blocks_for(count * generators), kPrimBlock, 0, static_cast<cudaStream_t>(stream)>>>(
      arg, reinterpret_cast<const unsigned long long*>(parents), count, reinterpret_cast<unsigned long long*>(children));
  return cuda_status(cudaGetLastError());
}

int mgbfs2_rank_packed(uint32_t degree, uint32_t bits, uint32_t distinct, const uint32_t* counts_host,
                       const uint64_t* words, uint64_t count, uint64_t* ranks, uint32_t* error, void* stream) {
  if (!degree || !counts_host || !distinct || distinct > 16 || (bits != 4 && bits != 8) ||
      static_cast<uint64_t>(degree) * bits > 64)
    return MGBFS2_INVALID_ARGUMENT;
  MultisetDomain d{};
  d.n = degree;
  d.bits = bits;
  d.distinct = distinct;
  uint32_t sum = 0;
  for (uint32_t c = 0; c < distinct; ++c) {
    if (!counts_host[c]) return MGBFS2_INVALID_ARGUMENT;
    d.counts[c] = counts_host[c];
    sum += counts_host[c];
  }
  if (sum != degree) return MGBFS2_INVALID_ARGUMENT;
  unsigned __int128 ways = 1;
  uint64_t placed = 0;
  for (uint32_t c = 0; c < distinct; ++c)
    for (uint32_t k = 1; k <= d.counts[c]; ++k) {
      ways = ways * (placed + k) / k;
      if (ways > static_cast<unsigned __int128>(UINT64_MAX)) return MGBFS2_UNSUPPORTED;
      if (k == d.counts[c]) placed += d.counts[c];
    }
  d.total = static_cast<unsigned long long>(ways);
  if (!count) return MGBFS2_OK;
  if (!words || !ranks) return MGBFS2_INVALID_ARGUMENT;
  const int lehmer = distinct == degree && bits == 4;
  rank_kernel<<<blocks_for(count), kPrimBlock, 0, static_cast<cudaStream_t>(stream)>>>(
      d, lehmer, reinterpret_cast<const unsigned long long*>(words), count,
      reinterpret_cast<unsigned long long*>(ranks), error);
  return cuda_status(cudaGetLastError());
}

int mgbfs2_rank_components(uint32_t degree, uint32_t bits, uint32_t distinct, const uint32_t* codes_host,
                           uint32_t generators, const uint32_t* permutations_host, const uint64_t* words,
                           uint64_t count, uint64_t* ranks, uint64_t* domain_size, uint32_t* error, void* stream) {
  if (!degree || !codes_host || !generators || !permutations_host) return MGBFS2_INVALID_ARGUMENT;
  mgbfs2::ProductDomain d{};
  if (!mgbfs2::build_product_domain(degree, bits, distinct, codes_host, generators, permutations_host, &d))
    return MGBFS2_INVALID_ARGUMENT;
  if (domain_size) *domain_size = d.total;
  if (!count) return MGBFS2_OK;
  if (!words || !ranks) return MGBFS2_INVALID_ARGUMENT;
  product_rank_kernel<<<blocks_for(count), kPrimBlock, 0, static_cast<cudaStream_t>(stream)>>>(
      d, reinterpret_cast<const unsigned long long*>(words), count, reinterpret_cast<unsigned long long*>(ranks),
      error);
  return cuda_status(cudaGetLastError());
}

int mgbfs2_bitmap_claim(const uint64_t* ranks, uint64_t count, uint64_t* bitmap, uint64_t domain, uint8_t* won,
                        uint32_t warp, uint32_t* error, void* stream) {
  if (!count) return MGBFS2_OK;
  if (!ranks || !bitmap || !won || !domain) return MGBFS2_INVALID_ARGUMENT;
  bitmap_claim_kernel<<<blocks_for(count), kPrimBlock, 0, static_cast<cudaStream_t>(stream)>>>(
      reinterpret_cast<const unsigned long long*>(ranks), count, reinterpret_cast<unsigned long long*>(bitmap), domain,
      won, warp ? 1 : 0, error);
  return cuda_status(cudaGetLastError());
}

int mgbfs2_hash_insert(const uint64_t* keys, uint64_t count, uint64_t* table, uint64_t slots, uint8_t* inserted,
                       uint32_t* error, void* stream) {
  if (!slots || (slots & (slots - 1))) return MGBFS2_INVALID_ARGUMENT;
  if (!count) return MGBFS2_OK;
  if (!keys || !table || !inserted) return MGBFS2_INVALID_ARGUMENT;
  hash_insert_kernel<<<blocks_for(count), kPrimBlock, 0, static_cast<cudaStream_t>(stream)>>>(
      reinterpret_cast<const unsigned long long*>(keys), count, reinterpret_cast<unsigned long long*>(table), slots - 1,
      inserted, error);
  return cuda_status(cudaGetLastError());
}

int mgbfs2_sort_unique_tiles(const uint64_t* keys, uint64_t count, uint32_t tile, uint32_t key_bits, uint64_t* out,
                             uint32_t* counts, void* stream) {
  if (tile != kSortTile || !key_bits || key_bits > 64) return MGBFS2_INVALID_ARGUMENT;
  if (!count) return MGBFS2_OK;
  if (!keys || !out || !counts) return MGBFS2_INVALID_ARGUMENT;
  const uint64_t tiles = (count + tile - 1) / tile;
  sort_unique_tiles_kernel<<<static_cast<uint32_t>(std::min<uint64_t>(tiles, 148ull * 8)), kSortThreads, 0,
                             static_cast<cudaStream_t>(stream)>>>(
      reinterpret_cast<const unsigned long long*>(keys), count, key_bits, reinterpret_cast<unsigned long long*>(out),
      counts);
  return cuda_status(cudaGetLastError());
}

int mgbfs2_bucket_keys(const uint64_t* keys, uint64_t count, uint32_t shift, uint32_t shards, uint64_t* buckets,
                       uint64_t capacity, unsigned long long* counts, uint32_t* error, void* stream) {
  if (!shards || shards > 4096 || shift > 63 || !error) return MGBFS2_INVALID_ARGUMENT;
  if (!count) return MGBFS2_OK;
  if (!keys || !buckets || !counts) return MGBFS2_INVALID_ARGUMENT;
  const size_t smem = shards * (sizeof(unsigned long long) + sizeof(uint32_t));
  bucket_kernel<<<blocks_for(count), kPrimBlock, smem, static_cast<cudaStream_t>(stream)>>>(
      reinterpret_cast<const unsigned long long*>(keys), count, shift, shards,
      reinterpret_cast<unsigned long long*>(buckets), capacity, counts, error);
  return cuda_status(cudaGetLastError());
}

}  // extern "C"
