// Host-side engine state of one graph handle (libmgbfs2 internal header).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <map>
#include <vector>

#include <nvtx3/nvToolsExt.h>

#include "../../include/mgbfs2.h"
#include "device.cuh"

namespace mgbfs2 {

int cuda_status(cudaError_t e);

// Sets fn's shared-memory carveout on the current device to the smallest
// configuration that holds `want` resident blocks of `threads` threads (fewer
// where registers or shared memory allow fewer), leaving the rest as L1.
// smem is the dynamic shared memory per block; returns the resident blocks.
int size_carveout(const void* fn, size_t smem, int want, int threads);

// A device allocation that only grows, ordered on its owner's stream.  No
// destructor: owners call free().
struct DeviceBuffer {
  void* ptr = nullptr;
  size_t bytes = 0;
  cudaStream_t stream = nullptr;
  // Mapped buffers (kMappedMin bytes and up): a reserved virtual range of
  // `span` bytes (0 = a pool allocation) that grows in place, one physical
  // chunk per growth, through the driver's virtual memory calls.
  size_t span = 0;
  int device = 0;                                             // of a mapped buffer
  std::vector<std::pair<unsigned long long, size_t>> chunks;  // physical handle, bytes
  int ensure(size_t want, bool exact = false);  // exact: no geometric headroom
  void free();
  // Hands the buffer to the process-wide device cache instead of the pool.
  // Only when no work in flight on any stream uses it (its owner synchronised).
  void release_to_cache(int device);
};

// Process-wide cache of device buffers given back by destroyed graph handles,
// per device: a new handle's buffers are taken from it (smallest that fits)
// before the stream-ordered pool is asked.  Creating and destroying a handle
// per search then costs no pool allocation at all; allocating multi-GB
// blocks from a pool whose free memory is split over blocks of other sizes
// took 6-12 ms per allocation on a B200.
bool device_cache_take(int device, size_t want, void** ptr, size_t* bytes);
void device_cache_give(int device, void* ptr, size_t bytes);
uint64_t device_cache_bytes(int device);
void device_cache_drain(int device, cudaStream_t stream);
int device_cache_release(int device);

int retain_pool_memory(int device);
// Pinned host buffers from a process-wide cache: creating and freeing page-
// locked memory is slow, and cudaFreeHost synchronises the device, so handles
// take their small pinned mirrors from the cache and give them back.
int pinned_take(size_t bytes, void** out);
void pinned_give(void* ptr);
uint64_t pool_idle_bytes(int device);
// Free device memory (cudaMemGetInfo), reused for up to two seconds per device and
// corrected by the change in this process's pool reservation since; `fresh`
// queries the device now (memory taken by others, e.g. another allocator of
// the process, is seen only then).
int device_free_bytes(int device, size_t* free_bytes, bool fresh = false);

struct WideState;     // int64-key arena path (wide.cu)
struct ExpandParams;  // packed_kernels.cuh

// A named NVTX range for the lifetime of the object: a profiler's timeline
// shows the library's phases (plan, run, each layer by kernel family, batch
// waves, planner training) around the kernels.  NVTX v3 is header-only and
// costs a pointer check when no tool is attached.
struct TraceRange {
  explicit TraceRange(const char* name) { nvtxRangePushA(name); }
  ~TraceRange() { nvtxRangePop(); }
  TraceRange(const TraceRange&) = delete;
  TraceRange& operator=(const TraceRange&) = delete;
};

// The bitmap's product domain over the generators' position components of
// packed codes (engine.cu); false when it cannot be represented.
bool build_product_domain(uint32_t n, uint32_t bits, uint32_t distinct, const uint32_t* codes, uint32_t gens,
                          const uint32_t* perms, ProductDomain* out);

struct Graph {
  // Description.
  int device = 0;
  uint32_t kind = 0, elements = 0, rows = 0, cols = 0, gens = 0;
  std::vector<uint32_t> perms;
  std::vector<int64_t> matrices;
  std::vector<uint32_t> moduli;
  std::vector<int64_t> start;
  uint64_t orbit_bound = 0;

  // Analysis.
  bool packed = false, inverse_closed = false, lehmer = false, rank_ok = false;
  // Modular matrices with one modulus, canonical start entries and no int64
  // overflow in any product: packed into one word of `bits`-bit entries and
  // expanded by the fused kernels (MatrixAction); others take the wide path.
  bool packed_matrix = false;
  MatrixAction matrix_action() const {
    if (!packed_matrix) return MatrixAction{0, 0, 0, 0, 0, 0};
    return MatrixAction{rows, cols, bits, moduli[0], static_cast<uint32_t>((1ull << 32) / moduli[0]), 0};
  }
  uint32_t bits = 4, distinct = 0;
  std::vector<int64_t> labels;     // code -> label
  std::vector<uint32_t> codes;     // start codes
  std::vector<uint32_t> code_counts;
  uint64_t start_word = 0, key_mask = ~0ull;
  uint64_t rank_total = 0, state_bound = 0;
  // Position components of the generators: when they split the positions
  // and their product of multiset domains is smaller than the whole multiset
  // domain, the bitmap ranks over the product (ProductDomain).
  bool product = false;
  ProductDomain product_domain{};
  bool use_product = false;  // plan: rank over the product (not with the Lehmer-only routed / grouped layers)
  uint64_t rank_domain() const { return use_product ? product_domain.total : rank_total; }
  std::vector<uint64_t> coxeter;   // certified layer sizes, empty if not Coxeter
  std::vector<Term> terms;
  std::vector<uint32_t> term_begin;  // gens + 1 term offsets, then inverse[gens]
  uint32_t gen_shift = 0;            // parent-edge tag position, 0 = no tags
  bool parent_skip = false;          // plan: use the tags

  // Plan and device state.
  bool planned = false;
  mgbfs2_plan_info plan{};
  cudaStream_t stream = nullptr;
  cudaEvent_t ev_run[2] = {nullptr, nullptr}, ev_kernel[2] = {nullptr, nullptr};
  int sm_count = 148;
  DeviceBuffer bitmap, front, next, table, bank[3], program, control_buf, scratch;
  uint64_t table_slots = 0, bank_slots[3] = {0, 0, 0};
  // All-visited hash in 32-bit quotient slots (device.cuh QuotientSlots).
  bool hash_quotient = false;
  uint32_t hash_load = 50;  // growth threshold, percent
  uint64_t learned_peak = 0;  // learned plan: predicted largest layer (pre-sizes the frontier buffers)
  uint64_t memory_reserve = 2ull << 30;  // plan: device bytes left free for others
  uint32_t group_chunk = 4096;  // plan shape: parents per grouped work item
  int blocks_per_sm = 0;        // plan shape: resident layer-kernel blocks per SM, 0 = defaults
  uint32_t parents_per_thread = 0;  // plan shape: fused layers' states per thread, 0 = by generators
  uint64_t route_chunk = 0;         // plan shape: parents per routed pass, 0 = by memory
  int want_blocks(int kernel_default) const { return blocks_per_sm ? blocks_per_sm : kernel_default; }
  QuotientSlots quotient_slots(uint64_t slots) const;
  Control* host_control = nullptr;
  WideState* wide = nullptr;

  // Bucketed (owner-routed) bitmap layers: shard s holds the states whose
  // first bucket_prefix Lehmer digits spell s, i.e. one contiguous rank range.
  uint32_t bucket_prefix = 0, bucket_shards = 0;
  uint64_t bucket_margin = 4096, bucket_min_work = 1ull << 22;
  DeviceBuffer buckets, shard_meta;            // uint32 offsets; begin/cap/count per shard
  unsigned long long* host_meta = nullptr;     // pinned: begin, cap, count (3 x kMaxShards), work
  std::vector<uint64_t> shard_history;         // last routed layer's per-shard counts
  uint64_t shard_history_total = 0;
  int bucket_setup(uint64_t work, bool exact);
  int bucket_launch(const void* route, const void* accept, const ExpandParams& p, size_t smem);
  int routed_setup(uint64_t count, uint64_t* cap, uint64_t* chunk);
  int bucket_chunks(const void* route, const void* accept, const ExpandParams& p, size_t smem, uint64_t chunk,
                    uint32_t* redo);
  bool bucket_alloc_exact = false;  // memory-bounded routed layer: buckets grow without headroom
  uint64_t bucket_work = 0;         // successors the current shard buckets were sized for

  // Grouped layers (claim, then route the winners): the frontier is kept in
  // per-group regions (states sharing their first group_prefix symbols) plus a
  // spill region; `front_grouped` says whether `front` currently has that
  // layout, described by front_begin / front_count (groups, then the spill).
  uint32_t group_prefix = 0, groups = 0;
  DeviceBuffer group_meta;
  unsigned long long* host_group = nullptr;  // pinned mirror of group_meta
  bool front_grouped = false;
  std::vector<uint64_t> front_begin, front_count, next_begin, next_cap;
  std::vector<uint32_t> group_order;  // visiting order of the groups (work items follow it)
  bool group_transp = false;          // every generator swaps two adjacent positions: incremental ranks
  DeviceBuffer transp_buf;            // per generator: t, wg(t-1), wg(t), wi(t-1), wi(t)
  int plan_transpositions(bool allowed);
  void plan_group_order();
  int grouped_setup(uint64_t count, uint64_t prev_count, uint64_t cap, void** fn, size_t* smem_total, size_t smem,
                    uint64_t* items, uint32_t* grid);
  // Sets fn's shared-memory carveout to the smallest configuration holding
  // `want` resident blocks (fewer where registers allow fewer); returns them.
  int set_carveout(const void* fn, size_t smem, int want);
  std::map<const void*, int> carveout_blocks;  // resident blocks per SM of kernels given a carveout
  int grouped_finish();   // after the layer: per-region counts of `next` into next_begin/next_cap layout
  int gather_front(uint64_t count);  // grouped `front` -> contiguous

  // Graph mode of the fused path: one CUDA graph whose WHILE node repeats
  // {expand, loop_finalize} with the layer loop state on the device.
  DeviceBuffer loop_buf;
  bool host_loop_only = false;  // plan option MGBFS2_OPTION_HOST_LOOP
  int run_device_loop(const void* fn, ExpandParams* p, size_t smem, uint64_t cap, mgbfs2_status* st,
                      double* kernel_seconds, uint64_t* count, uint64_t* visited, uint32_t* depth, bool* paused);

  // Checkpoint / resume (checkpoint.cu): read_checkpoint restores the visited
  // structure, the deepest layer (in `front`) and the layer table, and the
  // next run() goes on from there.
  bool resume_pending = false;
  std::vector<uint64_t> resume_layers;
  int write_checkpoint(const char* path);
  int read_checkpoint(const char* path);
  int frontier_words(uint64_t* out, size_t capacity, size_t* count);
  int table_probe_mean(double* mean, uint64_t* keys);

  // Results.
  std::vector<uint64_t> layer_sizes;
  std::vector<double> layer_seconds;
  std::vector<uint64_t> small_layer[2];  // the two most recent layers with < 1000 states
  uint32_t small_depth[2] = {UINT32_MAX, UINT32_MAX};
  void keep_small(uint32_t depth, std::vector<uint64_t>&& words);
  uint64_t last_count = 0;
  uint32_t launches = 0;

  static int create(const mgbfs2_graph_desc* d, int device, Graph** out, char* error, size_t cap);
  ~Graph();
  void analyse();
  void build_program();
  void build_matrix_program();
  bool matrix_inverse_closed() const;
  void release();
  int make_plan(const mgbfs2_plan_request* req, mgbfs2_plan_info* out);
  int run(const mgbfs2_run_limits* limits, mgbfs2_layer_callback cb, void* user, mgbfs2_status* status);
  int sample(uint32_t which, int64_t* out, size_t cap_rows, size_t* rows);
  int visit_kind() const;
  uint32_t grid_for(const void* fn, size_t smem, uint64_t work_blocks);
  uint64_t next_bound(uint32_t depth, uint64_t count, uint64_t visited) const;
  std::vector<int64_t> decode(uint64_t w) const;

  // Wide (multi-word int64 key) path, wide.cu.
  uint32_t wide_key_words() const;
  int wide_plan(mgbfs2_plan_info* p, uint64_t budget);
  int wide_run(const mgbfs2_run_limits* limits, mgbfs2_layer_callback cb, void* user, mgbfs2_status* status);
  int wide_sample(uint32_t which, int64_t* out, size_t cap_rows, size_t* rows);
  void wide_release();
};

}  // namespace mgbfs2

// The C-ABI handle (mgbfs2.h) around a Graph.
struct mgbfs2_graph {
  mgbfs2::Graph* impl;
};
