/*
 * libmgbfs2 — C ABI of the B200-native exact BFS engine for implicit Cayley and
 * permutation graphs.
 *
 * Conventions (kept from the reference's C ABI, cuda/mgbfs_cuda.h:10-19):
 *   - every function returns int: 0 = success (or enqueued), a small positive
 *     MGBFS2_* code, or MGBFS2_CUDA_BASE + cudaError_t;
 *   - create functions take (char* error, size_t error_capacity) for a message;
 *   - kernel-level entry points take caller-owned device pointers and a
 *     `void* stream` (cudaStream_t, NULL = legacy default stream) and allocate
 *     nothing; device-side failures land in a sticky uint32 error word
 *     (reference: cuda/generic_visited.h:19);
 *   - a graph handle is single-threaded: one caller at a time.
 *
 * Every entry point cites the reference interface it replaces.  Paths are
 * relative to the TryDotAtwo/MultiGPUBFS tree.
 */
#ifndef MGBFS2_H
#define MGBFS2_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define MGBFS2_API __attribute__((visibility("default")))
#else
#define MGBFS2_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

enum {
  MGBFS2_OK = 0,
  MGBFS2_INVALID_ARGUMENT = 1,
  MGBFS2_UNSUPPORTED = 2,
  MGBFS2_OUT_OF_MEMORY = 3,
  MGBFS2_CAPACITY = 4,
  MGBFS2_DEVICE_STATUS = 5,
  MGBFS2_STATE = 6,
  MGBFS2_NOT_FOUND = 7,
  MGBFS2_CUDA_BASE = 1000
};

/* Graph description: the lossless schema-2 contract of
 * multigpubfs/graph_definition.py:17-69 as plain arrays. */
typedef struct {
  uint32_t kind;                 /* 0 = permutation, 1 = int64 matrix */
  uint32_t elements;             /* state length: degree, or rows * cols */
  uint32_t rows, cols;           /* matrix shape; permutation: rows = degree, cols = 1 */
  uint32_t generators;
  const uint32_t* permutations;  /* generators x elements; child[i] = state[g[i]] */
  const int64_t* matrices;       /* generators x rows x rows, row-major */
  const uint32_t* moduli;        /* generators; 0 = plain int64 wrap, else 2..2^31 */
  const int64_t* start;          /* elements */
  uint64_t orbit_bound;          /* expected_max_unique_states, 0 = none */
} mgbfs2_graph_desc;

enum { MGBFS2_VISITED_AUTO = 0, MGBFS2_VISITED_BITMAP = 1, MGBFS2_VISITED_HASH = 2, MGBFS2_VISITED_HASH3 = 3 };
/* SORT: per-tile radix sort + unique of the children before the visited test.
 * BUCKET: route successors to rank-range shard buckets, then claim per shard.
 * GROUPED: claim first, route only the winners into a frontier grouped by its
 * first N-10 symbols (Lehmer bitmaps of degree 11..14). */
enum { MGBFS2_DEDUP_AUTO = 0, MGBFS2_DEDUP_ATOMIC = 1, MGBFS2_DEDUP_WARP = 2, MGBFS2_DEDUP_SORT = 3,
       MGBFS2_DEDUP_BUCKET = 4, MGBFS2_DEDUP_GROUPED = 5 };
enum { MGBFS2_PLANNER_PLAIN = 0, MGBFS2_PLANNER_LEARNED = 1 };

typedef struct {
  uint32_t visited;        /* MGBFS2_VISITED_* */
  uint32_t dedup;          /* MGBFS2_DEDUP_* */
  uint64_t capacity;       /* max states per frontier, 0 = from the state bound */
  uint64_t reserve_bytes;  /* device bytes never planned, 0 = 2 GiB */
  uint32_t shards;         /* MGBFS2_DEDUP_BUCKET on the bitmap: 0 = states sharing their first k symbols,
                              k the smallest of 1, 2 whose (n-k)!-bit bitmap slice is <= 8 MiB (S13: 156
                              shards); non-zero = k = 2 when degree < shards, else k = 1.  Ignored by
                              the other dedup modes (grouped layers use 1-3-symbol prefix groups). */
  uint32_t block;          /* threads per block, 0 = tuned */
  uint32_t planner;        /* MGBFS2_PLANNER_* */
  uint32_t bucket_margin;  /* extra entries per shard bucket, 0 = 4096; UINT32_MAX = none */
  uint64_t bucket_min_work; /* successors per layer from which layers are bucketed or grouped, 0 = 2^22 */
  uint32_t options;        /* MGBFS2_OPTION_* bits */
  uint32_t hash_load_percent; /* largest fill of the all-visited hash table before it grows, in percent
                                 (10..95, 0 = 50) */
  /* MGBFS2_PLANNER_LEARNED: the predicted number of states the BFS settles and
   * its predicted largest layer (e.g. |G| by Schreier-Sims and the planner
   * network's rollout).  Required with that planner (MGBFS2_INVALID_ARGUMENT
   * without them).  They replace the worst-case state bound when choosing
   * between the bitmap and the hash (auto) and when sizing the hash table,
   * and pre-size the frontier buffers; an under-prediction costs a table
   * growth or a buffer growth, never a different table.  Ignored by the plain
   * planner. */
  uint64_t predicted_states;
  uint64_t predicted_peak;
  /* Shapes (the autotuner's choices): parents per work item of grouped layers
   * (0 = 4096), and resident blocks per SM of the layer-expansion kernels
   * (0 = each kernel's default; capped by what its registers and shared
   * memory allow).  They change speed only. */
  uint32_t group_chunk;
  uint32_t blocks_per_sm;
  uint32_t parents_per_thread; /* fused layers: 1, 2 or 4 frontier states per thread and tile (0 = 1 for
                                  quotient-slot hash layers, else 4 up to 4 generators and 2 above) */
  uint32_t route_chunk;    /* routed (BUCKET) layers: parents routed and accepted per pass, a multiple of
                              1024 (0 = the whole layer, or the largest chunk whose buckets fit the device
                              memory left beside the bitmap and both frontiers, e.g. S14 under LRX) */
} mgbfs2_plan_request;

/* Packed graphs tag every frontier state with the generator that produced it
 * and skip that generator's inverse (the edge back to the previous layer)
 * without a visited test, when there are spare bits above the state and the
 * generators come in inverse pairs (permutations: an inverse-closed set;
 * modular matrices: any generator whose inverse mod m is in the set); this
 * option turns that off. */
#define MGBFS2_OPTION_NO_PARENT_SKIP 1u
/* Plans whose frontier buffers and visited set are sized up front (the fused
 * bitmap or all-visited hash layers, no limits or callback) run the whole BFS
 * on the device: one persistent cooperative launch with bounded grid barriers
 * between layers, or, where the grid cannot be co-resident, one CUDA graph
 * whose WHILE node repeats {expand layer, finalize}.  This option keeps the
 * host-driven layer loop instead (one launch and one readback per layer). */
#define MGBFS2_OPTION_HOST_LOOP 2u
/* Grouped layers over adjacent-transposition generators derive each child's
 * rank from its parent's Lehmer digits (two digits change); this option makes
 * them rank every child from scratch instead. */
#define MGBFS2_OPTION_FULL_RANK 4u
/* The all-visited hash of one-word states keeps each key in a 32-bit slot
 * when its bits allow (the slot index and the slot together hold a bijective
 * mix of the key: exact, half the bytes); this option keeps 64-bit slots
 * holding the key itself instead. */
#define MGBFS2_OPTION_WIDE_SLOTS 8u

typedef struct {
  uint32_t visited, dedup;
  uint32_t packed;          /* 1 = states are one packed uint64 word (permutation codes, or the entries of
                               a modular matrix) */
  uint32_t bits_per_symbol; /* packed symbol or matrix-entry width */
  uint32_t key_words;       /* uint64 words per state */
  uint32_t history_layers;  /* 1 = all visited retained, 3 = three-layer banks */
  uint64_t capacity;        /* frontier capacity bound (states) */
  uint64_t table_slots;     /* hash slots (all-visited table) */
  uint64_t bitmap_bits;     /* rank-domain size of the bitmap: n!, the multinomial, the product of the
                               position components' domains, or m^entries for modular matrices */
  uint64_t device_bytes;    /* fixed device allocation of the plan */
  uint64_t state_bound;     /* certified orbit bound, 0 = unknown */
  uint32_t shards, block;
  uint32_t inverse_closed;
  uint32_t planner;
  uint32_t parent_skip;     /* 1 = parent-edge skip active */
  uint32_t bucket_prefix;   /* bucket shards: states sharing their first k symbols */
  uint32_t table_slot_bytes; /* all-visited hash: 4 = quotient slots, 8 = key slots, 0 = no table */
  uint32_t hash_load_percent; /* the table's growth threshold */
  uint32_t group_chunk;      /* parents per grouped work item */
  uint32_t blocks_per_sm;    /* requested resident blocks per SM, 0 = kernel defaults */
  uint32_t rank_components;  /* bitmap: position components of the rank domain (1 = the whole multiset) */
  uint32_t parents_per_thread; /* fused layers' states per thread and tile */
} mgbfs2_plan_info;

typedef struct {
  double max_seconds;          /* 0 = no deadline */
  uint32_t max_layers;         /* 0 = no limit */
  uint32_t reserved;
  const volatile int32_t* cancel; /* optional; non-zero stops before the next layer */
} mgbfs2_run_limits;

enum { MGBFS2_REASON_FRONTIER_EXHAUSTED = 0, MGBFS2_REASON_DEADLINE = 1, MGBFS2_REASON_CANCELLED = 2,
       MGBFS2_REASON_RESOURCE = 3, MGBFS2_REASON_LAYER_LIMIT = 4 };

typedef struct {
  uint32_t complete;     /* 1 = frontier exhausted */
  uint32_t reason;       /* MGBFS2_REASON_* */
  uint32_t fatal;        /* device ERR_* bits when reason = RESOURCE */
  uint32_t layers;       /* entries in the layer table (depth 0 included) */
  uint64_t states;       /* sum of layer sizes */
  uint64_t successors;   /* edges explored: generators x expanded states */
  double bfs_seconds;
  uint32_t redo_layers;  /* layers recomputed after an exact overflow */
  uint32_t kernel_launches;
  uint64_t peak_device_bytes;
  double device_seconds; /* CUDA-event time of the whole run on the engine stream */
  double kernel_seconds; /* CUDA-event time summed over the layer-expansion kernels */
  uint64_t visited_tests; /* successors generated and tested (edges minus skipped parent edges) */
} mgbfs2_status;

/* Per-layer callback; return non-zero to stop (reason CANCELLED). */
typedef int (*mgbfs2_layer_callback)(void* user, uint32_t depth, uint64_t size, double seconds);

typedef struct mgbfs2_graph mgbfs2_graph;

/* Replaces the `mgbfs graph` engine set-up: GenericNativeBfs::new,
 * crates/mgbfs-runtime/src/generic_native.rs:69-98 (validation of
 * graph_definition.py:46-69 included). */
MGBFS2_API int mgbfs2_graph_create(const mgbfs2_graph_desc* desc, int device, mgbfs2_graph** out, char* error,
                        size_t error_capacity);

/* Replaces the plain planner GenericMemoryPlan::{with_storage, automatic_storage},
 * crates/mgbfs-runtime/src/generic_memory.rs:36-49, and the `graph-info` admission
 * verb, crates/mgbfs-cli/src/main.rs:54-84. */
MGBFS2_API int mgbfs2_plan(mgbfs2_graph* graph, const mgbfs2_plan_request* request, mgbfs2_plan_info* plan);

/* Replaces the layer loop of generic_run::run, crates/mgbfs-runtime/src/generic_run.rs:25-34,
 * with GenericNativeBfs::advance, generic_native.rs:106-126 (one scalar readback per layer). */
MGBFS2_API int mgbfs2_run(mgbfs2_graph* graph, const mgbfs2_run_limits* limits, mgbfs2_layer_callback callback,
               void* user, mgbfs2_status* status);

/* layer_sizes / layer_seconds of report.json, generic_run.rs:39. */
MGBFS2_API int mgbfs2_layer_table(const mgbfs2_graph* graph, uint64_t* sizes, double* seconds, size_t capacity,
                       size_t* count);

/* states.json samples, generic_native.rs:129-144: which = 0 -> the deepest layer
 * ("current", up to capacity_rows rows), which = 1 -> the layer before it when
 * it holds fewer than 1000 states ("previous_small").  Rows are int64 labels,
 * row-major, elements per row. */
MGBFS2_API int mgbfs2_sample(mgbfs2_graph* graph, uint32_t which, int64_t* out, size_t capacity_rows, size_t* rows);

/* Checkpoint of a BFS between layers (after mgbfs2_run returned at a layer
 * limit, deadline or cancel, or complete): the layer table, the visited
 * structure (bitmap or all-visited hash), the deepest layer and the small-layer
 * samples, written to `path`.  Bitmap and all-visited hash plans of one-word
 * states (three-bank histories and wide states: MGBFS2_UNSUPPORTED). */
MGBFS2_API int mgbfs2_checkpoint_write(mgbfs2_graph* graph, const char* path);

/* Loads a checkpoint into a handle planned for the same graph and visited
 * structure (MGBFS2_INVALID_ARGUMENT when the file, generators, coding or
 * structure differ); the next mgbfs2_run goes on from the checkpoint's depth
 * and gives the table of an uninterrupted run.  The reference keeps a layer
 * archive and restarts from its manifest (scripts/bfs_tail_archive.py,
 * crates/mgbfs-runtime/src/archive.rs) without resuming a search. */
MGBFS2_API int mgbfs2_checkpoint_resume(mgbfs2_graph* graph, const char* path);

/* The deepest layer's packed states (parent-edge tags removed): *count
 * receives its size; with out non-NULL and capacity >= *count they are copied
 * to out.  Valid after mgbfs2_run and inside its layer callback (the layer just
 * recorded), so a caller can archive every layer, as the reference's layer
 * archive does (scripts/bfs_tail_archive.py:96-131). */
MGBFS2_API int mgbfs2_frontier_words(mgbfs2_graph* graph, uint64_t* out, size_t capacity, size_t* count);

/* After a run on the all-visited hash: the mean number of slots an insert or
 * a successful lookup of each stored key reads (its distance from its home
 * slot plus one, over every key in the table) and the number of keys.  The
 * measured probes per visited test of the roofline's algorithmic bytes.
 * No reference counterpart. */
MGBFS2_API int mgbfs2_table_probes(mgbfs2_graph* graph, double* mean_probes, uint64_t* keys);

/* Static message for a status code (reference: native_fault.rs error markers). */
MGBFS2_API const char* mgbfs2_status_string(int code);

/* Destroying a handle keeps its device buffers in a per-device cache of the
 * library (buffers from 1 GB stay mapped; the stream-ordered pool keeps freed
 * smaller ones reserved), so the next handle on the device allocates nothing.
 * This returns both to the device: it frees the cached buffers and trims the
 * pool.  Call it with no
 * handle or batch of the device running.  No reference counterpart: the
 * reference runs each graph in a CLI process whose exit frees everything
 * (crates/mgbfs-cli/src/main.rs:191-200). */
MGBFS2_API int mgbfs2_trim_memory(int device);

MGBFS2_API void mgbfs2_destroy(mgbfs2_graph* graph);

/* A named range on a profiler's timeline (NVTX), for callers that mark their
 * own phases around the library's; the library marks its own (plan, run, each
 * layer by kernel family, batch waves).  Replaces mgbfs_trace_range_push/pop,
 * cuda/profile_ranges.cpp:6-24, which are compiled in only with MGBFS_NVTX;
 * NVTX v3 is header-only, so these are always present. */
MGBFS2_API void mgbfs2_trace_range_push(const char* label);
MGBFS2_API void mgbfs2_trace_range_pop(void);

/* ------------------------------------------------------------------------ */
/* Kernel-level entry points (caller-owned device buffers, no allocation).    */

/* All successors of `count` parents: children[(p * generators + g) * elements + e].
 * Parents and children are row-major int64 states.  Replaces
 * mgbfs_generic_generate_i64 (cuda/generic_graph.h, kernel cuda/generic_graph.cu:7-36),
 * whose planes are element-major; the int64 matrix action wraps before `% modulo`
 * exactly as graph_definition.py:77-83. */
MGBFS2_API int mgbfs2_successors_i64(uint32_t kind, uint32_t elements, uint32_t rows, uint32_t cols, uint32_t generators,
                          const int64_t* parents, uint64_t count, const uint32_t* permutations,
                          const int64_t* matrices, const uint32_t* moduli, int64_t* children,
                          uint32_t* error, void* stream);

/* Packed successors of one-word states (4/8/16/32-bit symbols):
 * children[p * generators + g].  Device form of the packed transitions of
 * scripts/cpu_small_bfs.py:21-27 for arbitrary permutation generators. */
MGBFS2_API int mgbfs2_successors_packed(uint32_t degree, uint32_t bits, uint32_t generators, const uint32_t* permutations_host,
                             const uint64_t* parents, uint64_t count, uint64_t* children, void* stream);

/* Exact lexicographic multiset rank of packed states.  counts_host[c] is the
 * multiplicity of symbol code c (distinct codes, sum = degree).  Replaces the
 * device contract bitmap_rank_component, cuda/permutation_bitmap.cuh:23-49.
 * Invalid states get rank UINT64_MAX and set *error bit 4 (rank range). */
MGBFS2_API int mgbfs2_rank_packed(uint32_t degree, uint32_t bits, uint32_t distinct, const uint32_t* counts_host,
                       const uint64_t* words, uint64_t count, uint64_t* ranks, uint32_t* error, void* stream);

/* Rank of packed states in the product of the generators' position
 * components' multiset domains (the bitmap domain of graphs whose generators
 * keep groups of positions apart): codes_host[i] is the code at position i of
 * the start (dense codes < distinct), permutations_host the generators
 * (generators x degree).  *domain_size (optional) receives the product size.
 * Invalid states get rank UINT64_MAX and set *error bit 4.  Replaces
 * bitmap_rank over component descriptors, cuda/permutation_bitmap.cuh:62-83,
 * with the domain of PositionOrbitDomain,
 * crates/mgbfs-runtime/src/permutation_bitmap.rs:61-143. */
MGBFS2_API int mgbfs2_rank_components(uint32_t degree, uint32_t bits, uint32_t distinct, const uint32_t* codes_host,
                                      uint32_t generators, const uint32_t* permutations_host, const uint64_t* words,
                                      uint64_t count, uint64_t* ranks, uint64_t* domain_size, uint32_t* error,
                                      void* stream);

/* Test-and-set claim of ranks in a bitmap of `domain` bits; won[i] = 1 for
 * exactly one occurrence of every rank not set before.  warp = 1 merges bits of
 * a warp that share a word into one atomicOr.  Replaces bitmap_accept /
 * bitmap_accept_grouped, cuda/permutation_bitmap.cu:105-205. */
MGBFS2_API int mgbfs2_bitmap_claim(const uint64_t* ranks, uint64_t count, uint64_t* bitmap, uint64_t domain, uint8_t* won,
                        uint32_t warp, uint32_t* error, void* stream);

/* Exact-key insertion of packed keys into an open-addressing table of `slots`
 * (power of two, initialised to all-ones); inserted[i] = 1 for exactly one
 * occurrence of each key that was absent.  Replaces accept_candidates,
 * cuda/generic_visited.cu:18-58 (single-word keys). */
MGBFS2_API int mgbfs2_hash_insert(const uint64_t* keys, uint64_t count, uint64_t* table, uint64_t slots, uint8_t* inserted,
                       uint32_t* error, void* stream);

/* Tile-local sort-unique: each tile of `tile` keys (<= 4096, power of two) is
 * radix-sorted in shared memory and its distinct keys are written, sorted, to
 * out[tile_index * tile ...]; counts[tile_index] = distinct keys of that tile.
 * Replaces the CUB sort + unique stage of cuda/permutation_bitmap_batch.cu:48-160
 * and cuda/segmented_hash_batch.cu:53-190 (here per tile, in shared memory). */
MGBFS2_API int mgbfs2_sort_unique_tiles(const uint64_t* keys, uint64_t count, uint32_t tile, uint32_t key_bits,
                             uint64_t* out, uint32_t* counts, void* stream);

/* Owner routing inside one GPU: key k goes to shard (k >> shift) (< shards);
 * buckets is shards x capacity; counts[s] = keys routed to s (exact, may exceed
 * capacity, which sets error bit 3).  Replaces route / bitmap_route,
 * cuda/generic_route.cu:7-37 and cuda/permutation_bitmap.cu:27-48. */
MGBFS2_API int mgbfs2_bucket_keys(const uint64_t* keys, uint64_t count, uint32_t shift, uint32_t shards, uint64_t* buckets,
                       uint64_t capacity, unsigned long long* counts, uint32_t* error, void* stream);

/* One exact BFS layer of a packed permutation frontier (4-bit codes, degree
 * 2..16, all codes distinct, <= 64 generators) against a caller-owned
 * Lehmer-rank bitmap of ceil(degree!/64) words, through the bucketed
 * route/accept kernels: successors are routed into rank-range shards of the
 * bitmap (exactly sized by a counting pass) and tested shard by shard.
 * New states are written to next[0 .. next_capacity); *next_count (device)
 * receives their exact number (bit 0 of *error when it exceeds the capacity).
 * All temporaries live in `scratch` (device, >= mgbfs2_expand_layer_scratch_bytes
 * bytes, 256-byte aligned); asynchronous on `stream`; allocates nothing.
 * `frontier` must be 16-byte aligned (MGBFS2_INVALID_ARGUMENT otherwise):
 * parents are read two at a time.
 * Replaces the route + accept pair mgbfs_bitmap_route / mgbfs_bitmap_accept,
 * cuda/permutation_bitmap.cu:27-48 and :105-133. */
MGBFS2_API int mgbfs2_expand_layer_bitmap(uint32_t degree, uint32_t generators, const uint32_t* permutations_host,
                                          const uint64_t* frontier, uint64_t count, uint64_t* bitmap,
                                          uint64_t* next, uint64_t next_capacity, uint64_t* next_count,
                                          uint32_t* error, void* scratch, uint64_t scratch_bytes, void* stream);

/* Scratch bytes mgbfs2_expand_layer_bitmap needs for `count` parents. */
MGBFS2_API uint64_t mgbfs2_expand_layer_scratch_bytes(uint32_t degree, uint32_t generators, uint64_t count);

/* mgbfs2_expand_layer_bitmap for callers that cannot allocate device memory:
 * hosts that reserve the whole GPU in their own pool and forbid any other
 * allocator, and search loops that must not stall or fail in an allocator in
 * the middle of a BFS.  Same inputs, outputs and results, but the scratch is a
 * 32 MiB array inside the library (every GPU that loads the library holds it
 * until the process exits), so the call allocates nothing and copies nothing
 * from the host.  Limit: count * generators <= 4,191,328 successors per call
 * (MGBFS2_CAPACITY above it, before anything is launched).  The first call on a
 * device looks up the array's device address (cudaGetSymbolAddress) with that
 * device current, so make it before any stream capture.  All calls on a device
 * share the array and it keeps the last call's contents (each call clears what
 * must start at zero); calls that overlap on the GPU race on it and must be
 * serialised by the caller.  No counterpart in the reference. */
MGBFS2_API int mgbfs2_expand_layer_bitmap_static(uint32_t degree, uint32_t generators,
                                                 const uint32_t* permutations_host, const uint64_t* frontier,
                                                 uint64_t count, uint64_t* bitmap, uint64_t* next,
                                                 uint64_t next_capacity, uint64_t* next_count, uint32_t* error,
                                                 void* stream);

/* ------------------------------------------------------------------------ */
/* Owner-partitioned layers: one BFS over several ranks (one per GPU).      */
/* Replaces the reference's owner route / exchange / accept split
 * (cuda/permutation_bitmap.cu:27-48 and :105-205 with world/owner arguments,
 * the grouped send/recv of crates/mgbfs-runtime/src/generic_distributed_native.rs:199-285).
 * The partition differs from the reference's rank mod world: prefix block s
 * (the states whose first `prefix` Lehmer digits give s; (degree-prefix)!
 * consecutive ranks) belongs to rank s mod world, which stores it as local
 * block s / world, so a rank's slice is blocks_per_owner * (degree-prefix)!
 * bits and the owner of a child costs `prefix` digit steps, not a full rank.
 * Packed states of `degree` <= 16 distinct 4-bit codes, as in the layer call
 * above.  When the generator set holds inverse pairs and the bits fit
 * (4 * degree + bits of the generator count <= 64), every routed child carries
 * the number g + 1 of its generator in the bits from 4 * degree up, and route
 * skips each parent's edge back to its own parent; the tags travel with the
 * words and are ignored by the claim. */

/* The partition of `degree`-symbol states over `world` ranks: prefix digits,
 * blocks per owner and bits per slice.  MGBFS2_UNSUPPORTED when
 * world * blocks_per_owner exceeds 256 buckets.  Host only. */
MGBFS2_API int mgbfs2_shard_geometry(uint32_t degree, uint32_t world, uint32_t* prefix, uint32_t* blocks_per_owner,
                                     uint64_t* slice_bits);

/* Device scratch bytes each of the two calls below needs (256-byte aligned). */
MGBFS2_API uint64_t mgbfs2_shard_scratch_bytes(void);

/* Sending side of a layer: expands `frontier` and writes every child (packed
 * word) to out[], owner-major and block-minor, sized exactly by a counting pass;
 * out_capacity >= count * generators (MGBFS2_CAPACITY otherwise).
 * bucket_counts (device, world * blocks_per_owner u64) receives the count per
 * (owner, local block): owner w's words are the contiguous run of its
 * blocks_per_owner buckets, ready for an all-to-all with these split sizes.
 * `frontier` must be 16-byte aligned (a chunk of a frontier starts at an even
 * entry).  Asynchronous on `stream`. */
MGBFS2_API int mgbfs2_shard_route(uint32_t degree, uint32_t generators, const uint32_t* permutations_host,
                                  const uint64_t* frontier, uint64_t count, uint32_t world, uint64_t* out,
                                  uint64_t out_capacity, uint64_t* bucket_counts, uint32_t* error, void* scratch,
                                  uint64_t scratch_bytes, void* stream);

/* Receiving side: `incoming` holds the words every source rank sent to
 * `owner`, in source order; incoming_counts (device, world * blocks_per_owner
 * u64, source-major) holds each source's bucket_counts row for this owner.
 * Each word is claimed in this rank's slice (bit = local block *
 * (degree-prefix)! + rank within the block); winners go to next[], *next_count
 * (device) receives their number.  A word whose prefix block this rank does not
 * own is not claimed and raises bit 7 (BAD_REFERENCE) of *error.
 * Asynchronous on `stream`. */
MGBFS2_API int mgbfs2_shard_accept(uint32_t degree, uint32_t world, uint32_t owner, const uint64_t* incoming,
                                   const uint64_t* incoming_counts, uint64_t* bitmap_slice, uint64_t* next,
                                   uint64_t next_capacity, uint64_t* next_count, uint32_t* error, void* scratch,
                                   uint64_t scratch_bytes, void* stream);

/* ------------------------------------------------------------------------ */
/* Batched sweep: many BFS instances, each wave one persistent launch.       */

typedef struct mgbfs2_batch mgbfs2_batch;

typedef struct {
  uint32_t max_depth;       /* layer-table capacity per instance, 0 = 1024 */
  uint32_t blocks_per_sm;   /* batch_expand blocks per SM, 0 = occupancy limit (the tuned shape) */
  uint32_t host_loop;       /* layer loop of a wave: 0 = one persistent cooperative launch (grid barriers
                               between layers), 1 = host-driven (one sync per layer), 2 = CUDA-graph WHILE loop */
  uint32_t tile_entries;    /* frontier entries per work tile: 256, 512 or 1024 (0 = 1024; the tuned shape) */
  uint64_t memory_bytes;    /* device bytes available to the waves, 0 = free memory minus reserve */
  uint64_t reserve_bytes;   /* 0 = 2 GiB */
  const uint64_t* predicted_capacity; /* per instance frontier capacity (learned planner); NULL or 0 = orbit bound */
} mgbfs2_batch_options;

typedef struct {
  uint32_t instances, complete_instances, waves;
  uint32_t redo_instances;  /* instances rerun from depth 0 (their wave's redo pool was exhausted) */
  uint32_t graph_launches, kernel_launches, layer_steps, fatal;
  uint64_t states, successors;
  double seconds;           /* wall time of mgbfs2_batch_run */
  double device_seconds;    /* CUDA-event time of the waves' layer loops */
  uint32_t redo_layers;     /* layers redone in a larger segment after overflowing a predicted capacity */
  uint32_t reserved;
} mgbfs2_batch_status;

/* Instances: permutation graphs of degree 2..15 with distinct labels and at
 * most 16 generators (each gets an exact n!-bit Lehmer bitmap).  No reference
 * counterpart as one launch: the reference runs graphs one after another
 * through its resident worker pool, multigpubfs/generic_session.py:139. */
MGBFS2_API int mgbfs2_batch_create(const mgbfs2_graph_desc* graphs, uint32_t count, int device, mgbfs2_batch** out,
                                   char* error, size_t error_capacity);

/* Runs every instance to completion in waves that fit the memory budget.  By
 * default a wave is ONE persistent cooperative launch that expands every active
 * instance's layer, finalizes it behind a bounded grid barrier and repeats
 * until the device finds no active instance (options->host_loop selects the
 * CUDA-graph WHILE form or a host-driven loop instead).  With predicted
 * capacities an eighth of the budget is kept as a redo pool: a layer that
 * overflows its instance's segment is redone in a larger segment from the pool
 * within the same launch (winners that found no room release their bitmap bit,
 * the stored ones move), so only that layer is repeated.  An instance whose
 * pool is exhausted is rerun from depth 0 with its orbit bound in a later
 * wave.  Tables never depend on the capacities. */
MGBFS2_API int mgbfs2_batch_run(mgbfs2_batch* batch, const mgbfs2_batch_options* options, mgbfs2_batch_status* status);

/* Layer table of one instance after mgbfs2_batch_run. */
MGBFS2_API int mgbfs2_batch_layer_table(const mgbfs2_batch* batch, uint32_t instance, uint64_t* sizes,
                                        size_t capacity, size_t* count);

/* Every instance's layer table in one call: instance i's table is
 * tables[offsets[i] .. offsets[i + 1]) (offsets: count + 1 entries).  With
 * tables NULL (or capacity too small) only the offsets are written, and
 * MGBFS2_CAPACITY is returned when tables is given but too small. */
MGBFS2_API int mgbfs2_batch_layer_tables(const mgbfs2_batch* batch, uint64_t* tables, uint64_t capacity,
                                         uint64_t* offsets);

/* Expansion seconds of each layer of one instance after mgbfs2_batch_run,
 * aligned with its layer table: entry d >= 1 is the device time (globaltimer)
 * of the layer step of its wave that produced layer d, shared by every
 * instance of that wave; entry 0 (the start) is 0.  The per-layer expansion
 * time of the reference's sweep layers.csv (docs/reproduce-pair-sweeps.md:20). */
MGBFS2_API int mgbfs2_batch_layer_seconds(const mgbfs2_batch* batch, uint32_t instance, double* seconds,
                                          size_t capacity, size_t* count);

MGBFS2_API void mgbfs2_batch_destroy(mgbfs2_batch* batch);

/* ------------------------------------------------------------------------ */
/* Planner network (learned planner): inputs -> 64 -> 64 -> 2, ReLU, one flat */
/* fp32 parameter buffer W1[64][in] | b1 | W2[64][64] | b2 | W3[2][64] | b3.  */
/* No reference counterpart (the reference plans with worst-case bounds and   */
/* timed pilots: crates/mgbfs-runtime/src/generic_memory.rs:36-49,            */
/* multigpubfs/autotune.py:276).  All device pointers, rows of `inputs` fp32. */

MGBFS2_API uint32_t mgbfs2_mlp_param_count(uint32_t inputs);
MGBFS2_API int mgbfs2_mlp_forward(uint32_t inputs, const float* params, const float* x, uint64_t batch, float* y,
                                  void* stream);
/* grad += d/dparams of sum_s (w0 (y_s0 - t_s0)^2 + w1 (y_s1 - t_s1)^2) / batch; *loss += that sum. */
MGBFS2_API int mgbfs2_mlp_loss_grad(uint32_t inputs, const float* params, const float* x, const float* target,
                                    float weight0, float weight1, uint64_t batch, float* grad, float* loss,
                                    void* stream);
MGBFS2_API int mgbfs2_mlp_adam(uint32_t count, float* params, const float* grad, float* m, float* v, float lr,
                               float beta1, float beta2, float eps, uint32_t step, void* stream);
MGBFS2_API int mgbfs2_mlp_to_bf16(uint32_t count, const float* params, void* params_bf16, void* stream);
/* bf16 parameters and activations, fp32 accumulation. */
MGBFS2_API int mgbfs2_mlp_infer_bf16(uint32_t inputs, const void* params_bf16, const float* x, uint64_t batch,
                                     float* y, void* stream);

/* Device rollout of the planner network (16 inputs, bf16 parameters as made by
 * mgbfs2_mlp_to_bf16), one thread per instance: from |L_0| = 1, predicts
 * layer after layer from the last four (features normalised by x_mean and
 * x_scale, 16 floats each) until the prediction drops below one half or
 * max_depth layers, and writes each instance's predicted peak layer, total and
 * depth.  statics: count x 8 floats (log orbit, n/16, g/8, inverse-closed, mean
 * and max log generator order, fixed-point fraction, cycle fraction); gens:
 * count floats.  All device pointers.  No reference counterpart. */
MGBFS2_API int mgbfs2_mlp_rollout_bf16(const void* params_bf16, const float* x_mean, const float* x_scale,
                                       const float* statics, const float* gens, uint32_t count, uint32_t max_depth,
                                       double* peak, double* total, uint32_t* depth, void* stream);

/* Order of the group generated by `generators` permutations of {0..n-1}
 * (row-major, g[i] = image of i; n <= 20), by deterministic Schreier-Sims on
 * the host.  With distinct labels it is the exact number of states a BFS
 * settles; the learned planner uses it as the orbit size of its features.  The
 * reference bounds the state space by the multinomial n!/prod(c!) instead
 * (crates/mgbfs-runtime/src/generic_memory.rs:82-108). */
MGBFS2_API int mgbfs2_group_order(const uint32_t* permutations, uint32_t n, uint32_t generators, uint64_t* order);

/* The learned planner's per-graph statics for `count` permutation graphs in
 * one host call, spread over `threads` host threads (0 = all).  Graph i has
 * degree[i] <= 20 points and generators[i] >= 1 permutations; the generators
 * of all graphs are concatenated row-major in `permutations` (graph i's block
 * is generators[i] x degree[i]), the start labels (dense ids < 256) in
 * `labels` (degree[i] each).  Writes statics[8i..8i+7] in the layout
 * mgbfs2_mlp_rollout_bf16 reads (log orbit, n/16, g/8, inverse-closed, mean
 * and max log generator order, fixed-point and cycle fractions) and states[i]:
 * |G| (the exact number of states the BFS settles) when the labels are
 * distinct, else the multinomial n!/prod(c!).  Host only.  No reference
 * counterpart: the reference's planner is the worst-case bound alone. */
MGBFS2_API int mgbfs2_graph_statics(uint32_t count, const uint32_t* degree, const uint32_t* generators,
                                    const uint32_t* permutations, const uint32_t* labels, uint32_t threads,
                                    float* statics, uint64_t* states);

#ifdef __cplusplus
}
#endif

#endif /* MGBFS2_H */
