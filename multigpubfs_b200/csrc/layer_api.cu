// Kernel-level entry point: one exact BFS layer of a packed permutation
// frontier against a caller-owned Lehmer-rank bitmap, through the bucketed
// route/accept kernels (bucket_kernels.cuh).  Stand-alone and asynchronous:
// bucket sizes come from an exact counting pass and an on-device scan, so no
// host round trip and no overflow redo are needed.  All temporaries live in
// caller-provided scratch.
#include <algorithm>
#include <map>
#include <mutex>
#include <vector>

#include "../../include/mgbfs2.h"
#include "bucket_kernels.cuh"
#include "engine.h"

namespace mgbfs2 {
namespace {

constexpr uint32_t kLayerMaxGens = 64;
constexpr size_t kAlign = 256;

size_t align_up(size_t x) { return (x + kAlign - 1) / kAlign * kAlign; }

// Byte offsets of the scratch regions.
struct LayerLayout {
  size_t control, meta, program, buckets, total;
};

LayerLayout layer_layout(uint64_t entries) {
  LayerLayout l{};
  l.control = 0;
  l.meta = align_up(sizeof(Control));
  l.program = l.meta + align_up((3 * kMaxShards + 1) * sizeof(unsigned long long));
  l.buckets = l.program + align_up(kLayerMaxGens * 16 * sizeof(Term) + (2 * kLayerMaxGens + 1) * sizeof(uint32_t));
  l.total = l.buckets + align_up(entries * sizeof(unsigned long long));
  return l;
}

// Single block: begin = exclusive scan of the counts, cap = counts (exact),
// then the counts and the accept work counter restart at zero.
__global__ void layout_shards(unsigned long long* meta, uint32_t shards) {
  if (threadIdx.x == 0) {
    unsigned long long run = 0;
    for (uint32_t s = 0; s < shards; ++s) {
      const unsigned long long c = meta[2 * kMaxShards + s];
      meta[s] = run;
      meta[kMaxShards + s] = c;
      meta[2 * kMaxShards + s] = 0;
      run += c;
    }
    meta[3 * kMaxShards] = 0;
  }
}

__global__ void publish_layer(const Control* control, unsigned long long* next_count, unsigned int* error) {
  if (threadIdx.x == 0) {
    *next_count = control->next_count;
    if (error && control->error) atomicOr(error, control->error);
  }
}

using CountFn = void (*)(RouteParams);
using RouteFn = void (*)(RouteParams);
using AcceptFn = void (*)(AcceptParams);

struct LayerKernels {
  CountFn count;
  RouteFn route;
  AcceptFn accept;
};

template <int N>
LayerKernels kernels_for(uint32_t prefix) {
  if (prefix == 1) return {count_lehmer<N, 1>, route_lehmer<N, 1>, accept_lehmer<N, 1>};
  return {count_lehmer<N, 2>, route_lehmer<N, 2>, accept_lehmer<N, 2>};
}

bool pick_layer_kernels(uint32_t n, uint32_t prefix, LayerKernels* k) {
  switch (n) {
#define MG_CASE(K)                   \
  case K:                            \
    *k = kernels_for<K>(prefix);     \
    return true;
    MG_CASE(2) MG_CASE(3) MG_CASE(4) MG_CASE(5) MG_CASE(6) MG_CASE(7) MG_CASE(8) MG_CASE(9) MG_CASE(10)
    MG_CASE(11) MG_CASE(12) MG_CASE(13) MG_CASE(14) MG_CASE(15) MG_CASE(16)
#undef MG_CASE
    default:
      return false;
  }
}

uint32_t layer_prefix(uint32_t n) {
  uint64_t f = 1;
  for (uint32_t i = 2; i < n; ++i) f *= i;  // (n-1)!
  return (f / 8 > (8ull << 20) && n * (n - 1) <= kMaxShards) ? 2u : 1u;
}

// Host-side program: displacement terms, term offsets, then the (unused)
// parent-edge table.
bool build_layer_program(uint32_t n, uint32_t gens, const uint32_t* perms, std::vector<Term>* terms,
                         std::vector<uint32_t>* begin) {
  terms->clear();
  begin->assign(1, 0);
  for (uint32_t k = 0; k < gens; ++k) {
    std::map<int, uint64_t> groups;
    std::vector<uint8_t> seen(n, 0);
    for (uint32_t i = 0; i < n; ++i) {
      const uint32_t src = perms[static_cast<size_t>(k) * n + i];
      if (src >= n || seen[src]) return false;
      seen[src] = 1;
      groups[static_cast<int>(src) - static_cast<int>(i)] |= 15ull << (4 * i);
    }
    for (auto& kv : groups) {
      const int shift = kv.first * 4;
      terms->push_back(Term{kv.second, shift > 0 ? static_cast<uint32_t>(shift) : 0u,
                            shift < 0 ? static_cast<uint32_t>(-shift) : 0u});
    }
    begin->push_back(static_cast<uint32_t>(terms->size()));
  }
  begin->insert(begin->end(), gens, 0xffffffffu);
  return true;
}

uint32_t occupancy_grid(const void* fn, size_t smem, int device) {
  int sms = 148, per_sm = 1;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, kBlock, smem) != cudaSuccess || per_sm < 1) {
    cudaGetLastError();
    per_sm = 1;
  }
  return static_cast<uint32_t>(sms * per_sm);
}

// Largest count * generators whose scratch size layer_layout can represent:
// the bucket region is 8 bytes per successor.
constexpr uint64_t kMaxLayerSuccessors = (UINT64_MAX / 2) / sizeof(unsigned long long);

// The route kernels read two parents at a time as one 16-byte load.
bool frontier_aligned(const uint64_t* frontier) { return reinterpret_cast<uintptr_t>(frontier) % 16 == 0; }

bool layer_arguments_ok(uint32_t degree, uint32_t generators, const uint32_t* permutations_host,
                        const uint64_t* frontier, uint64_t count, const uint64_t* bitmap, const uint64_t* next,
                        const uint64_t* next_count) {
  return degree >= 2 && degree <= 16 && generators && generators <= kLayerMaxGens && permutations_host && bitmap &&
         next_count && (!count || (frontier && next && frontier_aligned(frontier)));
}

// The generator program of one layer call, as the kernels read it from scratch.
struct LayerProgram {
  std::vector<Term> terms;
  std::vector<uint32_t> begin;
  uint32_t prefix = 1;
  LayerKernels kernels{};
  size_t bytes() const { return terms.size() * sizeof(Term) + begin.size() * sizeof(uint32_t); }
};

int prepare_layer_program(uint32_t degree, uint32_t generators, const uint32_t* permutations_host,
                          LayerProgram* prog) {
  if (!build_layer_program(degree, generators, permutations_host, &prog->terms, &prog->begin))
    return MGBFS2_INVALID_ARGUMENT;
  prog->prefix = layer_prefix(degree);
  if (!pick_layer_kernels(degree, prog->prefix, &prog->kernels)) return MGBFS2_UNSUPPORTED;
  return MGBFS2_OK;
}

// Enqueues count -> layout -> route -> accept -> publish on `stream`, with the
// generator program already in scratch at l.program and the control block and
// shard metadata already zeroed.  Both layer entry points end here.
int enqueue_layer(const LayerProgram& prog, uint32_t degree, uint32_t generators, const uint64_t* frontier,
                  uint64_t count, uint64_t* bitmap, uint64_t* next, uint64_t next_capacity, uint64_t* next_count,
                  uint32_t* error, unsigned char* scratch, const LayerLayout& l, int device, cudaStream_t stream) {
  TraceRange range("layer_api.expand");
  Control* control = reinterpret_cast<Control*>(scratch + l.control);
  unsigned long long* meta = reinterpret_cast<unsigned long long*>(scratch + l.meta);
  Term* program = reinterpret_cast<Term*>(scratch + l.program);
  uint64_t fact = 1;
  for (uint32_t i = degree - prog.prefix + 1; i <= degree; ++i) fact *= i;
  RouteParams rp{};
  rp.frontier = reinterpret_cast<const unsigned long long*>(frontier);
  rp.count = count;
  rp.terms = program;
  rp.term_begin = reinterpret_cast<const uint32_t*>(program + prog.terms.size());
  rp.gens = generators;
  rp.total_terms = static_cast<uint32_t>(prog.terms.size());
  rp.ppt = generators <= 3 ? 4 : (generators <= 6 ? 2 : 1);
  rp.group = kMaxEntries / rp.ppt;
  rp.gen_shift = 0;
  rp.shards = static_cast<uint32_t>(fact);  // n!/(n-prefix)!
  rp.prefix = prog.prefix;
  rp.buckets = reinterpret_cast<unsigned long long*>(scratch + l.buckets);
  rp.shard_begin = meta;
  rp.shard_cap = meta + kMaxShards;
  rp.shard_count = meta + 2 * kMaxShards;
  rp.control = control;
  const LayerKernels& k = prog.kernels;
  cudaError_t e = cudaSuccess;
  if (count) {
    const size_t count_smem = kMaxShards * sizeof(uint32_t) + prog.bytes();
    k.count<<<occupancy_grid(reinterpret_cast<const void*>(k.count), count_smem, device), kBlock, count_smem,
              stream>>>(rp);
    layout_shards<<<1, 32, 0, stream>>>(meta, rp.shards);
    const size_t route_smem = sizeof(RouteSmem) + prog.bytes();
    if ((e = cudaFuncSetAttribute(reinterpret_cast<const void*>(k.route), cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  static_cast<int>(route_smem))) != cudaSuccess)
      return cuda_status(e);
    k.route<<<occupancy_grid(reinterpret_cast<const void*>(k.route), route_smem, device), kBlock, route_smem,
              stream>>>(rp);
    AcceptParams ap{};
    ap.buckets = rp.buckets;
    ap.shard_begin = meta;
    ap.shard_count = meta + 2 * kMaxShards;
    ap.shards = rp.shards;
    ap.bitmap = reinterpret_cast<unsigned long long*>(bitmap);
    ap.next = reinterpret_cast<unsigned long long*>(next);
    ap.capacity = next_capacity;
    ap.work = meta + 3 * kMaxShards;
    ap.control = control;
    k.accept<<<occupancy_grid(reinterpret_cast<const void*>(k.accept), 0, device), kBlock, 0, stream>>>(ap);
  }
  publish_layer<<<1, 32, 0, stream>>>(control, reinterpret_cast<unsigned long long*>(next_count), error);
  return cuda_status(cudaGetLastError());
}

}  // namespace

// Enqueues the layer expansion into `scratch` (device memory laid out by
// layer_layout): the caller-scratch entry point.
int expand_layer_into(uint32_t degree, uint32_t generators, const uint32_t* permutations_host,
                      const uint64_t* frontier, uint64_t count, uint64_t* bitmap, uint64_t* next,
                      uint64_t next_capacity, uint64_t* next_count, uint32_t* error, unsigned char* scratch,
                      uint64_t scratch_bytes, cudaStream_t stream) {
  if (!scratch || !layer_arguments_ok(degree, generators, permutations_host, frontier, count, bitmap, next, next_count))
    return MGBFS2_INVALID_ARGUMENT;
  if (count > kMaxLayerSuccessors / generators) return MGBFS2_CAPACITY;
  const LayerLayout l = layer_layout(count * generators);
  if (scratch_bytes < l.total) return MGBFS2_CAPACITY;
  LayerProgram prog;
  if (int rc = prepare_layer_program(degree, generators, permutations_host, &prog)) return rc;
  int device = 0;
  cudaError_t e = cudaGetDevice(&device);
  if (e != cudaSuccess) return cuda_status(e);
  Control* control = reinterpret_cast<Control*>(scratch + l.control);
  unsigned long long* meta = reinterpret_cast<unsigned long long*>(scratch + l.meta);
  unsigned char* program = scratch + l.program;
  if ((e = cudaMemsetAsync(control, 0, sizeof(Control), stream)) != cudaSuccess ||
      (e = cudaMemsetAsync(meta, 0, (3 * kMaxShards + 1) * sizeof(unsigned long long), stream)) != cudaSuccess ||
      (e = cudaMemcpyAsync(program, prog.terms.data(), prog.terms.size() * sizeof(Term), cudaMemcpyHostToDevice,
                           stream)) != cudaSuccess ||
      (e = cudaMemcpyAsync(program + prog.terms.size() * sizeof(Term), prog.begin.data(),
                           prog.begin.size() * sizeof(uint32_t), cudaMemcpyHostToDevice, stream)) != cudaSuccess)
    return cuda_status(e);
  return enqueue_layer(prog, degree, generators, frontier, count, bitmap, next, next_capacity, next_count, error,
                       scratch, l, device, stream);
}

uint64_t expand_layer_scratch_bytes(uint64_t count, uint32_t generators) {
  return layer_layout(count * generators).total;
}

// ---------------------------------------------------------------------------
// Owner-partitioned layers: one BFS whose Lehmer bitmap is split over `world`
// ranks (one per GPU).  Prefix block s (the ranks sharing the first `prefix`
// Lehmer digits, (n - prefix)! of them) belongs to rank s mod world, which
// keeps it as its local block s / world: bit = (s / world) * (n - prefix)! +
// the rank within the block.  A layer is route (every child to its owner's
// buckets) -> an all-to-all of the buckets between the ranks (the caller's,
// over NCCL) -> accept (each rank claims what it received in its slice).
namespace {

struct ShardGeometry {
  uint32_t prefix = 0, blocks_per_owner = 0;
  uint64_t blocks = 0, block_bits = 0, slice_bits = 0;
};

int shard_geometry(uint32_t degree, uint32_t world, ShardGeometry* g) {
  if (degree < 2 || degree > 16 || world < 1) return MGBFS2_INVALID_ARGUMENT;
  g->prefix = degree >= 4 ? 2u : 1u;
  g->blocks = 1;
  for (uint32_t i = degree - g->prefix + 1; i <= degree; ++i) g->blocks *= i;
  g->blocks_per_owner = static_cast<uint32_t>((g->blocks + world - 1) / world);
  // Buckets are owner-major, block-minor: world * blocks_per_owner of them,
  // each an 8-bit bucket index in the route kernel.
  if (static_cast<uint64_t>(world) * g->blocks_per_owner > kMaxShards) return MGBFS2_UNSUPPORTED;
  g->block_bits = 1;
  for (uint32_t i = 2; i <= degree - g->prefix; ++i) g->block_bits *= i;
  g->slice_bits = g->blocks_per_owner * g->block_bits;
  return MGBFS2_OK;
}

// Copies the route's exact bucket counts out and raises the caller's error bits.
__global__ void publish_route(const Control* control, const unsigned long long* meta, uint32_t buckets,
                              unsigned long long* bucket_counts, unsigned int* error) {
  for (uint32_t b = threadIdx.x; b < buckets; b += blockDim.x) bucket_counts[b] = meta[2 * kMaxShards + b];
  if (threadIdx.x == 0 && error && control->error) atomicOr(error, control->error);
}

// Receiving side: the incoming words are the sources' segments back to back
// (source rank order); source r's segment holds its local blocks j in order,
// counts[r * blocks + j] words each.  Accept bucket j * world + r (block-major,
// so the resident blocks claim in one local block at a time) gets its range.
__global__ void layout_incoming(const unsigned long long* counts, uint32_t world, uint32_t blocks,
                                unsigned long long* meta) {
  if (threadIdx.x == 0) {
    unsigned long long run = 0;
    for (uint32_t r = 0; r < world; ++r) {
      for (uint32_t j = 0; j < blocks; ++j) {
        const uint32_t b = j * world + r;
        const unsigned long long c = counts[static_cast<size_t>(r) * blocks + j];
        meta[b] = run;
        meta[kMaxShards + b] = c;
        meta[2 * kMaxShards + b] = c;
        run += c;
      }
    }
    meta[3 * kMaxShards] = 0;
  }
}

// Parent-edge tags of the owner-partitioned path: a child carries the number
// (g + 1) of the generator that produced it in the bits above its 4 * degree
// code bits, and route skips, for each parent, the generator equal to the
// inverse of its tag's, whose child is the parent's own parent (visited in an
// earlier layer).  Replaces the term program's trailing "no skip" table and
// returns the tag shift (0 = no tags: no inverse pairs, or no spare bits).
uint32_t tag_parent_edges(uint32_t degree, uint32_t gens, const uint32_t* perms, std::vector<uint32_t>* begin) {
  const uint32_t tag_bits = 32 - __builtin_clz(gens);
  if (4 * degree + tag_bits > 64) return 0;
  std::vector<uint32_t> inverse(gens, 0xffffffffu);
  bool any = false;
  std::vector<uint32_t> inv(degree);
  for (uint32_t k = 0; k < gens; ++k) {
    for (uint32_t i = 0; i < degree; ++i) inv[perms[static_cast<size_t>(k) * degree + i]] = i;
    for (uint32_t h = 0; h < gens && inverse[k] == 0xffffffffu; ++h)
      if (std::equal(inv.begin(), inv.end(), perms + static_cast<size_t>(h) * degree)) inverse[k] = h;
    any = any || inverse[k] != 0xffffffffu;
  }
  if (!any) return 0;
  std::copy(inverse.begin(), inverse.end(), begin->end() - gens);
  return 4 * degree;
}

int stage_program(const LayerProgram& prog, unsigned char* scratch, const LayerLayout& l, cudaStream_t stream) {
  cudaError_t e;
  if ((e = cudaMemsetAsync(scratch + l.control, 0, sizeof(Control), stream)) != cudaSuccess ||
      (e = cudaMemsetAsync(scratch + l.meta, 0, (3 * kMaxShards + 1) * sizeof(unsigned long long), stream)) !=
          cudaSuccess)
    return cuda_status(e);
  if (prog.terms.empty()) return MGBFS2_OK;
  unsigned char* program = scratch + l.program;
  if ((e = cudaMemcpyAsync(program, prog.terms.data(), prog.terms.size() * sizeof(Term), cudaMemcpyHostToDevice,
                           stream)) != cudaSuccess ||
      (e = cudaMemcpyAsync(program + prog.terms.size() * sizeof(Term), prog.begin.data(),
                           prog.begin.size() * sizeof(uint32_t), cudaMemcpyHostToDevice, stream)) != cudaSuccess)
    return cuda_status(e);
  return MGBFS2_OK;
}

}  // namespace

int shard_route(uint32_t degree, uint32_t generators, const uint32_t* permutations_host, const uint64_t* frontier,
                uint64_t count, uint32_t world, uint64_t* out, uint64_t out_capacity, uint64_t* bucket_counts,
                uint32_t* error, unsigned char* scratch, uint64_t scratch_bytes, cudaStream_t stream) {
  TraceRange range("shard.route");
  ShardGeometry g;
  if (int rc = shard_geometry(degree, world, &g)) return rc;
  if (!generators || generators > kLayerMaxGens || !permutations_host || !bucket_counts || !scratch ||
      (count && (!frontier || !out || !frontier_aligned(frontier))))
    return MGBFS2_INVALID_ARGUMENT;
  if (count > kMaxLayerSuccessors / generators) return MGBFS2_CAPACITY;
  if (out_capacity < count * generators) return MGBFS2_CAPACITY;
  const LayerLayout l = layer_layout(0);
  if (scratch_bytes < l.total) return MGBFS2_CAPACITY;
  LayerProgram prog;
  if (!build_layer_program(degree, generators, permutations_host, &prog.terms, &prog.begin))
    return MGBFS2_INVALID_ARGUMENT;
  const uint32_t gen_shift = tag_parent_edges(degree, generators, permutations_host, &prog.begin);
  prog.prefix = g.prefix;
  if (!pick_layer_kernels(degree, g.prefix, &prog.kernels)) return MGBFS2_UNSUPPORTED;
  int device = 0;
  cudaError_t e = cudaGetDevice(&device);
  if (e != cudaSuccess) return cuda_status(e);
  if (int rc = stage_program(prog, scratch, l, stream)) return rc;
  Control* control = reinterpret_cast<Control*>(scratch + l.control);
  unsigned long long* meta = reinterpret_cast<unsigned long long*>(scratch + l.meta);
  Term* program = reinterpret_cast<Term*>(scratch + l.program);
  const uint32_t buckets = world * g.blocks_per_owner;
  if (count) {
    RouteParams rp{};
    rp.frontier = reinterpret_cast<const unsigned long long*>(frontier);
    rp.count = count;
    rp.terms = program;
    rp.term_begin = reinterpret_cast<const uint32_t*>(program + prog.terms.size());
    rp.gens = generators;
    rp.total_terms = static_cast<uint32_t>(prog.terms.size());
    rp.ppt = generators <= 3 ? 4 : (generators <= 6 ? 2 : 1);
    rp.group = kMaxEntries / rp.ppt;
    rp.gen_shift = gen_shift;
    rp.shards = buckets;
    rp.prefix = g.prefix;
    rp.owners = world;
    rp.owner_blocks = g.blocks_per_owner;
    rp.buckets = reinterpret_cast<unsigned long long*>(out);
    rp.shard_begin = meta;
    rp.shard_cap = meta + kMaxShards;
    rp.shard_count = meta + 2 * kMaxShards;
    rp.control = control;
    const LayerKernels& k = prog.kernels;
    const size_t count_smem = kMaxShards * sizeof(uint32_t) + prog.bytes();
    k.count<<<occupancy_grid(reinterpret_cast<const void*>(k.count), count_smem, device), kBlock, count_smem,
              stream>>>(rp);
    layout_shards<<<1, 32, 0, stream>>>(meta, buckets);
    const size_t route_smem = sizeof(RouteSmem) + prog.bytes();
    if ((e = cudaFuncSetAttribute(reinterpret_cast<const void*>(k.route), cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  static_cast<int>(route_smem))) != cudaSuccess)
      return cuda_status(e);
    k.route<<<occupancy_grid(reinterpret_cast<const void*>(k.route), route_smem, device), kBlock, route_smem,
              stream>>>(rp);
  }
  publish_route<<<1, kBlock, 0, stream>>>(control, meta, buckets, reinterpret_cast<unsigned long long*>(bucket_counts),
                                          error);
  return cuda_status(cudaGetLastError());
}

int shard_accept(uint32_t degree, uint32_t world, uint32_t owner, const uint64_t* incoming,
                 const uint64_t* incoming_counts, uint64_t* bitmap_slice, uint64_t* next, uint64_t next_capacity,
                 uint64_t* next_count, uint32_t* error, unsigned char* scratch, uint64_t scratch_bytes,
                 cudaStream_t stream) {
  TraceRange range("shard.accept");
  ShardGeometry g;
  if (int rc = shard_geometry(degree, world, &g)) return rc;
  if (owner >= world || !incoming_counts || !bitmap_slice || !next_count || !scratch || !incoming || !next)
    return MGBFS2_INVALID_ARGUMENT;
  const LayerLayout l = layer_layout(0);
  if (scratch_bytes < l.total) return MGBFS2_CAPACITY;
  LayerKernels k{};
  if (!pick_layer_kernels(degree, g.prefix, &k)) return MGBFS2_UNSUPPORTED;
  int device = 0;
  cudaError_t e = cudaGetDevice(&device);
  if (e != cudaSuccess) return cuda_status(e);
  if (int rc = stage_program(LayerProgram{}, scratch, l, stream)) return rc;
  Control* control = reinterpret_cast<Control*>(scratch + l.control);
  unsigned long long* meta = reinterpret_cast<unsigned long long*>(scratch + l.meta);
  layout_incoming<<<1, 32, 0, stream>>>(reinterpret_cast<const unsigned long long*>(incoming_counts), world,
                                        g.blocks_per_owner, meta);
  AcceptParams ap{};
  ap.buckets = reinterpret_cast<const unsigned long long*>(incoming);
  ap.shard_begin = meta;
  ap.shard_count = meta + 2 * kMaxShards;
  ap.shards = world * g.blocks_per_owner;
  ap.bitmap = reinterpret_cast<unsigned long long*>(bitmap_slice);
  ap.next = reinterpret_cast<unsigned long long*>(next);
  ap.capacity = next_capacity;
  ap.work = meta + 3 * kMaxShards;
  ap.control = control;
  ap.owners = world;
  ap.owner = owner;
  k.accept<<<occupancy_grid(reinterpret_cast<const void*>(k.accept), 0, device), kBlock, 0, stream>>>(ap);
  publish_layer<<<1, 32, 0, stream>>>(control, reinterpret_cast<unsigned long long*>(next_count), error);
  return cuda_status(cudaGetLastError());
}

// ---------------------------------------------------------------------------
// Allocation-free variant for callers that cannot allocate device memory.
//
// Some callers of this library cannot call cudaMalloc (or any allocator) per
// layer: a host framework that reserves all of the GPU's memory in its own
// pool up front and forbids any other allocation (a second allocator would
// fail or fragment that pool), and search loops that must not stall, since
// cudaMalloc may synchronise the device and can fail under memory pressure
// in the middle of a BFS.  For them the layer's scratch lives in one
// file-scope __device__ array of kStaticScratchBytes that every GPU loading
// this library holds until the process exits.  The generator program and the
// zeroed counters are written into it by one staging kernel from its
// parameters, so a call issues only kernel launches: no allocation, no host
// copy.  All calls on a device share the array and it keeps the last call's
// contents (each call re-zeroes what must start at zero); two calls that
// overlap on the GPU -- concurrent streams, or host threads on one device --
// race on it and must be serialised by the caller.
constexpr size_t kStaticScratchBytes = 32ull << 20;
static __device__ __align__(256) unsigned char g_static_scratch[kStaticScratchBytes];

namespace {

constexpr int kStaticMaxDevices = 64;
std::mutex g_static_lock;
unsigned char* g_static_address[kStaticMaxDevices] = {};

// Device address of g_static_scratch on `device` (the current device).  The
// host-side name is only a stand-in for the symbol, never a device address,
// so it is resolved with cudaGetSymbolAddress on the first call per device
// and kept for the process.  The address belongs to the device's primary
// context, the one the CUDA runtime uses: callers on their own driver-API
// contexts, or after cudaDeviceReset, are not supported.
int static_scratch(int device, unsigned char** out) {
  if (device < 0 || device >= kStaticMaxDevices) return MGBFS2_UNSUPPORTED;
  std::lock_guard<std::mutex> hold(g_static_lock);
  if (!g_static_address[device]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_static_scratch);
    if (e != cudaSuccess) return cuda_status(e);
    g_static_address[device] = static_cast<unsigned char*>(p);
  }
  *out = g_static_address[device];
  return MGBFS2_OK;
}

struct StagedProgram {
  Term terms[kLayerMaxGens * 16];
  uint32_t begin[2 * kLayerMaxGens + 1];
  uint32_t total_terms, begin_entries;
};
// Passed by value as a kernel parameter: kernel parameters above 4 KB need
// CUDA 12.1 or newer (limit 32,764 bytes).
static_assert(sizeof(StagedProgram) <= 32764, "StagedProgram exceeds the kernel parameter limit");

// Writes the program into scratch and zeroes the control block and shard
// metadata (counts, capacities, work counter).
__global__ void stage_static_layer(StagedProgram prog, Term* terms, uint32_t* begin, Control* control,
                                   unsigned long long* meta) {
  for (uint32_t i = threadIdx.x; i < prog.total_terms; i += blockDim.x) terms[i] = prog.terms[i];
  for (uint32_t i = threadIdx.x; i < prog.begin_entries; i += blockDim.x) begin[i] = prog.begin[i];
  for (uint32_t i = threadIdx.x; i < 3 * kMaxShards + 1; i += blockDim.x) meta[i] = 0;
  if (threadIdx.x == 0) {
    control->next_count = 0;
    control->aux = 0;
    control->error = 0;
    control->pad = 0;
  }
}

}  // namespace

int expand_layer_static(uint32_t degree, uint32_t generators, const uint32_t* permutations_host,
                        const uint64_t* frontier, uint64_t count, uint64_t* bitmap, uint64_t* next,
                        uint64_t next_capacity, uint64_t* next_count, uint32_t* error, cudaStream_t stream) {
  if (!layer_arguments_ok(degree, generators, permutations_host, frontier, count, bitmap, next, next_count))
    return MGBFS2_INVALID_ARGUMENT;
  // count * generators above the static bucket room (checked without forming
  // a product that could wrap).
  if (count > kMaxLayerSuccessors / generators) return MGBFS2_CAPACITY;
  const LayerLayout l = layer_layout(count * generators);
  if (l.total > kStaticScratchBytes) return MGBFS2_CAPACITY;
  LayerProgram prog;
  if (int rc = prepare_layer_program(degree, generators, permutations_host, &prog)) return rc;
  static thread_local StagedProgram staged;
  std::copy(prog.terms.begin(), prog.terms.end(), staged.terms);
  std::copy(prog.begin.begin(), prog.begin.end(), staged.begin);
  staged.total_terms = static_cast<uint32_t>(prog.terms.size());
  staged.begin_entries = static_cast<uint32_t>(prog.begin.size());
  int device = 0;
  cudaError_t e = cudaGetDevice(&device);
  if (e != cudaSuccess) return cuda_status(e);
  unsigned char* scratch = nullptr;
  if (int rc = static_scratch(device, &scratch)) return rc;
  Term* program = reinterpret_cast<Term*>(scratch + l.program);
  stage_static_layer<<<1, kBlock, 0, stream>>>(staged, program,
                                               reinterpret_cast<uint32_t*>(program + prog.terms.size()),
                                               reinterpret_cast<Control*>(scratch + l.control),
                                               reinterpret_cast<unsigned long long*>(scratch + l.meta));
  return enqueue_layer(prog, degree, generators, frontier, count, bitmap, next, next_capacity, next_count, error,
                       scratch, l, device, stream);
}

}  // namespace mgbfs2

extern "C" {

uint64_t mgbfs2_expand_layer_scratch_bytes(uint32_t degree, uint32_t generators, uint64_t count) {
  (void)degree;
  return mgbfs2::expand_layer_scratch_bytes(count, generators);
}

int mgbfs2_expand_layer_bitmap(uint32_t degree, uint32_t generators, const uint32_t* permutations_host,
                               const uint64_t* frontier, uint64_t count, uint64_t* bitmap, uint64_t* next,
                               uint64_t next_capacity, uint64_t* next_count, uint32_t* error, void* scratch,
                               uint64_t scratch_bytes, void* stream) {
  return mgbfs2::expand_layer_into(degree, generators, permutations_host, frontier, count, bitmap, next,
                                   next_capacity, next_count, error, static_cast<unsigned char*>(scratch),
                                   scratch_bytes, static_cast<cudaStream_t>(stream));
}

}  // extern "C"

extern "C" {

int mgbfs2_shard_geometry(uint32_t degree, uint32_t world, uint32_t* prefix, uint32_t* blocks_per_owner,
                          uint64_t* slice_bits) {
  mgbfs2::ShardGeometry g;
  if (int rc = mgbfs2::shard_geometry(degree, world, &g)) return rc;
  if (prefix) *prefix = g.prefix;
  if (blocks_per_owner) *blocks_per_owner = g.blocks_per_owner;
  if (slice_bits) *slice_bits = g.slice_bits;
  return MGBFS2_OK;
}

uint64_t mgbfs2_shard_scratch_bytes(void) { return mgbfs2::layer_layout(0).total; }

int mgbfs2_shard_route(uint32_t degree, uint32_t generators, const uint32_t* permutations_host,
                       const uint64_t* frontier, uint64_t count, uint32_t world, uint64_t* out, uint64_t out_capacity,
                       uint64_t* bucket_counts, uint32_t* error, void* scratch, uint64_t scratch_bytes, void* stream) {
  return mgbfs2::shard_route(degree, generators, permutations_host, frontier, count, world, out, out_capacity,
                             bucket_counts, error, static_cast<unsigned char*>(scratch), scratch_bytes,
                             static_cast<cudaStream_t>(stream));
}

int mgbfs2_shard_accept(uint32_t degree, uint32_t world, uint32_t owner, const uint64_t* incoming,
                        const uint64_t* incoming_counts, uint64_t* bitmap_slice, uint64_t* next,
                        uint64_t next_capacity, uint64_t* next_count, uint32_t* error, void* scratch,
                        uint64_t scratch_bytes, void* stream) {
  return mgbfs2::shard_accept(degree, world, owner, incoming, incoming_counts, bitmap_slice, next, next_capacity,
                              next_count, error, static_cast<unsigned char*>(scratch), scratch_bytes,
                              static_cast<cudaStream_t>(stream));
}

int mgbfs2_expand_layer_bitmap_static(uint32_t degree, uint32_t generators, const uint32_t* permutations_host,
                                      const uint64_t* frontier, uint64_t count, uint64_t* bitmap, uint64_t* next,
                                      uint64_t next_capacity, uint64_t* next_count, uint32_t* error, void* stream) {
  return mgbfs2::expand_layer_static(degree, generators, permutations_host, frontier, count, bitmap, next,
                                     next_capacity, next_count, error, static_cast<cudaStream_t>(stream));
}

}  // extern "C"
