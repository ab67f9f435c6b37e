// Checkpoint / resume of a single-graph BFS, and the deepest layer's packed
// words for a layer archive.
//
// A checkpoint is taken between layers (after mgbfs2_run returned, e.g. at a
// layer limit or a deadline): the layer table, the visited structure (Lehmer
// or product-domain bitmap, or the all-visited hash table), the deepest layer
// (the frontier the next layer expands) and the small-layer samples.  Resuming
// loads them into a handle planned for the same graph, and the next
// mgbfs2_run goes on from that depth with the same results as an
// uninterrupted run.  The reference archives completed layers to disk
// (scripts/bfs_tail_archive.py, crates/mgbfs-runtime/src/archive.rs) and
// restarts from its manifest without resuming a search; here the search
// itself resumes.
//
// File layout (little-endian): CheckpointHeader, the layer table (u64 each),
// the two small-layer samples (u64 words), the visited structure (raw device
// bytes), the frontier (u64 words).
#include <cstdio>
#include <cstring>
#include <vector>

#include "../../include/mgbfs2.h"
#include "engine.h"

#define MG_CHECK(expr)                             \
  do {                                             \
    cudaError_t _e = (expr);                       \
    if (_e != cudaSuccess) return cuda_status(_e); \
  } while (0)

namespace mgbfs2 {
namespace {

constexpr char kMagic[8] = {'M', 'G', 'B', 'F', 'S', '2', 'C', 'K'};
constexpr uint32_t kVersion = 1;
constexpr size_t kStage = 64ull << 20;  // pinned staging chunk

struct CheckpointHeader {
  char magic[8];
  uint32_t version, visit_kind;
  uint32_t elements, gens, bits, slot_bytes;
  unsigned long long key_mask, start_word, program_digest;
  unsigned long long layers, frontier, visited_bytes, table_slots;
  unsigned long long small_count[2];
  uint32_t small_depth[2];
};

// FNV-1a over the packed generator program: a checkpoint only resumes on a
// handle with the same generators and coding.
uint64_t program_digest(const Graph& g) {
  uint64_t h = 0xcbf29ce484222325ull;
  auto mix = [&](const void* p, size_t n) {
    const unsigned char* b = static_cast<const unsigned char*>(p);
    for (size_t i = 0; i < n; ++i) h = (h ^ b[i]) * 0x100000001b3ull;
  };
  mix(g.perms.data(), g.perms.size() * sizeof(uint32_t));
  mix(g.codes.data(), g.codes.size() * sizeof(uint32_t));
  mix(g.matrices.data(), g.matrices.size() * sizeof(int64_t));
  mix(g.moduli.data(), g.moduli.size() * sizeof(uint32_t));
  mix(&g.bits, sizeof(g.bits));
  return h;
}

bool checkpointable(int visit) {
  return bitmap_kind(visit) || visit == V_HASH || visit == V_HASHQ;
}

// Device bytes <-> file through a pinned staging buffer.
int device_to_file(std::FILE* f, const void* dev, size_t bytes, cudaStream_t stream, void* stage) {
  const char* src = static_cast<const char*>(dev);
  for (size_t done = 0; done < bytes;) {
    const size_t n = std::min(kStage, bytes - done);
    cudaError_t e = cudaMemcpyAsync(stage, src + done, n, cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    if (e != cudaSuccess) return cuda_status(e);
    if (std::fwrite(stage, 1, n, f) != n) return MGBFS2_STATE;
    done += n;
  }
  return MGBFS2_OK;
}

int file_to_device(std::FILE* f, void* dev, size_t bytes, cudaStream_t stream, void* stage) {
  char* dst = static_cast<char*>(dev);
  for (size_t done = 0; done < bytes;) {
    const size_t n = std::min(kStage, bytes - done);
    if (std::fread(stage, 1, n, f) != n) return MGBFS2_INVALID_ARGUMENT;
    cudaError_t e = cudaMemcpyAsync(dst + done, stage, n, cudaMemcpyHostToDevice, stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    if (e != cudaSuccess) return cuda_status(e);
    done += n;
  }
  return MGBFS2_OK;
}

struct File {
  std::FILE* f = nullptr;
  ~File() {
    if (f) std::fclose(f);
  }
};

struct Pinned {
  void* p = nullptr;
  ~Pinned() {
    if (p) pinned_give(p);
  }
};

}  // namespace

int Graph::write_checkpoint(const char* path) {
  if (!path) return MGBFS2_INVALID_ARGUMENT;
  if (!planned || !packed || layer_sizes.empty()) return MGBFS2_STATE;
  const int visit = visit_kind();
  if (!checkpointable(visit)) return MGBFS2_UNSUPPORTED;
  MG_CHECK(cudaSetDevice(device));
  MG_CHECK(cudaStreamSynchronize(stream));
  if (front_grouped) {
    if (int rc = gather_front(last_count)) return rc;
  }
  CheckpointHeader h{};
  std::memcpy(h.magic, kMagic, sizeof(kMagic));
  h.version = kVersion;
  h.visit_kind = static_cast<uint32_t>(visit);
  h.elements = elements;
  h.gens = gens;
  h.bits = bits;
  h.key_mask = key_mask;
  h.start_word = start_word;
  h.program_digest = program_digest(*this);
  h.layers = layer_sizes.size();
  h.frontier = last_count;
  const bool hashed = visit == V_HASH || visit == V_HASHQ;
  h.slot_bytes = hashed ? (visit == V_HASHQ ? 4u : 8u) : 0u;
  h.table_slots = hashed ? table_slots : 0;
  h.visited_bytes = hashed ? table_slots * h.slot_bytes : ((rank_domain() + 63) / 64) * 8;
  const void* visited_ptr = hashed ? table.ptr : bitmap.ptr;
  for (int i = 0; i < 2; ++i) {
    h.small_count[i] = small_layer[i].size();
    h.small_depth[i] = small_depth[i];
  }
  if (!visited_ptr || (h.frontier && (!front.ptr || front.bytes < h.frontier * 8))) return MGBFS2_STATE;
  File file;
  file.f = std::fopen(path, "wb");
  if (!file.f) return MGBFS2_INVALID_ARGUMENT;
  Pinned stage;
  if (int rc = pinned_take(kStage, &stage.p)) return rc;
  if (std::fwrite(&h, sizeof(h), 1, file.f) != 1 ||
      std::fwrite(layer_sizes.data(), 8, layer_sizes.size(), file.f) != layer_sizes.size())
    return MGBFS2_STATE;
  for (int i = 0; i < 2; ++i)
    if (std::fwrite(small_layer[i].data(), 8, small_layer[i].size(), file.f) != small_layer[i].size())
      return MGBFS2_STATE;
  if (int rc = device_to_file(file.f, visited_ptr, h.visited_bytes, stream, stage.p)) return rc;
  if (int rc = device_to_file(file.f, front.ptr, h.frontier * 8, stream, stage.p)) return rc;
  return std::fflush(file.f) == 0 ? MGBFS2_OK : MGBFS2_STATE;
}

int Graph::read_checkpoint(const char* path) {
  if (!path) return MGBFS2_INVALID_ARGUMENT;
  if (!planned || !packed) return MGBFS2_STATE;
  const int visit = visit_kind();
  if (!checkpointable(visit)) return MGBFS2_UNSUPPORTED;
  MG_CHECK(cudaSetDevice(device));
  File file;
  file.f = std::fopen(path, "rb");
  if (!file.f) return MGBFS2_NOT_FOUND;
  CheckpointHeader h{};
  if (std::fread(&h, sizeof(h), 1, file.f) != 1 || std::memcmp(h.magic, kMagic, sizeof(kMagic)) != 0 ||
      h.version != kVersion)
    return MGBFS2_INVALID_ARGUMENT;
  // The same graph, coding and visited structure as this plan.
  const bool hashed = visit == V_HASH || visit == V_HASHQ;
  if (h.visit_kind != static_cast<uint32_t>(visit) || h.elements != elements || h.gens != gens || h.bits != bits ||
      h.key_mask != key_mask || h.start_word != start_word || h.program_digest != program_digest(*this) ||
      !h.layers || h.layers > (1u << 24) || h.small_count[0] > 1000 || h.small_count[1] > 1000)
    return MGBFS2_INVALID_ARGUMENT;
  if (hashed) {
    if (h.slot_bytes != (visit == V_HASHQ ? 4u : 8u) || !h.table_slots || (h.table_slots & (h.table_slots - 1)) ||
        h.visited_bytes != h.table_slots * h.slot_bytes)
      return MGBFS2_INVALID_ARGUMENT;
  } else if (h.visited_bytes != ((rank_domain() + 63) / 64) * 8) {
    return MGBFS2_INVALID_ARGUMENT;
  }
  std::vector<uint64_t> layers(h.layers);
  if (std::fread(layers.data(), 8, layers.size(), file.f) != layers.size()) return MGBFS2_INVALID_ARGUMENT;
  if (layers[0] != 1 || layers.back() != h.frontier) return MGBFS2_INVALID_ARGUMENT;
  std::vector<uint64_t> small[2];
  for (int i = 0; i < 2; ++i) {
    small[i].resize(h.small_count[i]);
    if (std::fread(small[i].data(), 8, small[i].size(), file.f) != small[i].size()) return MGBFS2_INVALID_ARGUMENT;
  }
  int rc = MGBFS2_OK;
  void* visited_ptr = nullptr;
  if (hashed) {
    if ((rc = table.ensure(h.visited_bytes))) return rc;
    table_slots = h.table_slots;
    visited_ptr = table.ptr;
  } else {
    if ((rc = bitmap.ensure(h.visited_bytes))) return rc;
    visited_ptr = bitmap.ptr;
  }
  if ((rc = front.ensure((h.frontier + 2) * 8))) return rc;
  Pinned stage;
  if ((rc = pinned_take(kStage, &stage.p))) return rc;
  if ((rc = file_to_device(file.f, visited_ptr, h.visited_bytes, stream, stage.p))) return rc;
  if ((rc = file_to_device(file.f, front.ptr, h.frontier * 8, stream, stage.p))) return rc;
  if (std::fgetc(file.f) != EOF) return MGBFS2_INVALID_ARGUMENT;  // trailing bytes: not this format
  front_grouped = false;
  resume_layers = std::move(layers);
  for (int i = 0; i < 2; ++i) {
    small_layer[i] = std::move(small[i]);
    small_depth[i] = h.small_depth[i];
  }
  last_count = h.frontier;
  resume_pending = true;
  return MGBFS2_OK;
}

// The deepest layer's packed words, tags removed, in frontier order; also
// valid inside a layer callback (the layer just recorded).  A grouped frontier
// is read region by region.
int Graph::frontier_words(uint64_t* out, size_t capacity, size_t* count) {
  if (!count) return MGBFS2_INVALID_ARGUMENT;
  if (!planned || !packed || layer_sizes.empty()) return MGBFS2_STATE;
  MG_CHECK(cudaSetDevice(device));
  const uint64_t n = layer_sizes.size() == 1 ? 1 : layer_sizes.back();
  *count = n;
  if (!out || capacity < n) return out ? MGBFS2_CAPACITY : MGBFS2_OK;
  MG_CHECK(cudaStreamSynchronize(stream));
  const uint64_t mask = gen_shift ? (1ull << gen_shift) - 1ull : ~0ull;
  if (front_grouped) {
    uint64_t at = 0;
    for (size_t r = 0; r < front_begin.size() && r < front_count.size(); ++r) {
      if (!front_count[r]) continue;
      MG_CHECK(cudaMemcpyAsync(out + at, static_cast<const uint64_t*>(front.ptr) + front_begin[r],
                               front_count[r] * 8, cudaMemcpyDeviceToHost, stream));
      at += front_count[r];
    }
    if (at != n) return MGBFS2_STATE;
  } else {
    MG_CHECK(cudaMemcpyAsync(out, front.ptr, n * 8, cudaMemcpyDeviceToHost, stream));
  }
  MG_CHECK(cudaStreamSynchronize(stream));
  for (uint64_t i = 0; i < n; ++i) out[i] &= mask;
  return MGBFS2_OK;
}

}  // namespace mgbfs2

extern "C" {

int mgbfs2_checkpoint_write(mgbfs2_graph* graph, const char* path) {
  if (!graph) return MGBFS2_INVALID_ARGUMENT;
  return graph->impl->write_checkpoint(path);
}

int mgbfs2_checkpoint_resume(mgbfs2_graph* graph, const char* path) {
  if (!graph) return MGBFS2_INVALID_ARGUMENT;
  return graph->impl->read_checkpoint(path);
}

int mgbfs2_frontier_words(mgbfs2_graph* graph, uint64_t* out, size_t capacity, size_t* count) {
  if (!graph) return MGBFS2_INVALID_ARGUMENT;
  return graph->impl->frontier_words(out, capacity, count);
}

}  // extern "C"
