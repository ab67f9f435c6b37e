// Host engine of libmgbfs2: graph validation and packing, the plain planner,
// the level-synchronous layer loop and the graph-level C ABI.
//
// Reference counterparts (TryDotAtwo/MultiGPUBFS):
//   graph validation      multigpubfs/graph_definition.py:46-69
//   state-space bound     crates/mgbfs-runtime/src/generic_memory.rs:82-108
//   Coxeter certificate   multigpubfs/workload_geometry.py:2-19
//   layer loop            crates/mgbfs-runtime/src/generic_run.rs:25-34,
//                         crates/mgbfs-runtime/src/generic_native.rs:106-126
//   three-layer banks     crates/mgbfs-runtime/src/generic_distributed_native.rs:166-179,
//                         cuda/generic_rolling.cuh:3-47
#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <thread>
#include <string>
#include <vector>

#include <cuda.h>

#include "../../include/mgbfs2.h"
#include "bucket_kernels.cuh"
#include "engine.h"
#include "grouped_kernels.cuh"
#include "packed_kernels.cuh"

namespace mgbfs2 {

int cuda_status(cudaError_t e) { return e == cudaSuccess ? MGBFS2_OK : MGBFS2_CUDA_BASE + static_cast<int>(e); }

#define MG_CHECK(expr)                         \
  do {                                         \
    cudaError_t _e = (expr);                   \
    if (_e != cudaSuccess) return cuda_status(_e); \
  } while (0)

namespace {

using Clock = std::chrono::steady_clock;

constexpr uint64_t kRouteChunkAlign = 1024;  // parents: route chunks start 8 KB apart

void set_message(char* error, size_t capacity, const std::string& text) {
  if (!error || !capacity) return;
  std::snprintf(error, capacity, "%s", text.c_str());
}

// Grouped layers' prefix length K for degree n: N - 10 (10!-bit, 454 KB
// groups, whose working set of target groups stays in L2) within 1..4, the
// largest K <= 4 with at most kMaxGroups = 14!/10! groups above that (K = 3
// for degrees 15 and 16).
uint32_t group_prefix_for(uint32_t n) {
  uint32_t K = n > 10 ? std::min<uint32_t>(4, n - 10) : 1;
  const auto groups = [n](uint32_t k) {
    uint64_t g = 1;
    for (uint32_t i = 0; i < k; ++i) g *= n - i;
    return g;
  };
  while (K > 1 && groups(K) > kMaxGroups) --K;
  return K;
}

uint64_t next_pow2(uint64_t x) {
  uint64_t p = 1;
  while (p < x) p <<= 1;
  return p;
}

// n! / prod(c!) with saturation at UINT64_MAX.
uint64_t multinomial(const std::vector<uint32_t>& counts) {
  unsigned __int128 ways = 1;
  uint64_t placed = 0;
  for (uint32_t c : counts) {
    for (uint32_t k = 1; k <= c; ++k) {
      ways = ways * (placed + k) / k;
      if (ways > static_cast<unsigned __int128>(UINT64_MAX)) return UINT64_MAX;
    }
    placed += c;
  }
  return static_cast<uint64_t>(ways);
}

uint64_t sat_mul(uint64_t a, uint64_t b) {
  unsigned __int128 r = static_cast<unsigned __int128>(a) * b;
  return r > UINT64_MAX ? UINT64_MAX : static_cast<uint64_t>(r);
}

}  // namespace

// ---------------------------------------------------------------------------
// Graph construction and validation.

int Graph::create(const mgbfs2_graph_desc* d, int dev, Graph** out, char* error, size_t cap) {
  if (!d || !out) {
    set_message(error, cap, "GRAPH_ARGUMENT");
    return MGBFS2_INVALID_ARGUMENT;
  }
  *out = nullptr;
  auto fail = [&](const char* msg) {
    set_message(error, cap, msg);
    return MGBFS2_INVALID_ARGUMENT;
  };
  if (d->kind > 1) return fail("GRAPH_ACTION_KIND");
  if (!d->generators || !d->start || d->elements == 0) return fail("GRAPH_GENERATORS");
  auto g = new Graph();
  g->device = dev;
  g->kind = d->kind;
  g->elements = d->elements;
  g->gens = d->generators;
  g->start.assign(d->start, d->start + d->elements);
  g->orbit_bound = d->orbit_bound;
  if (d->kind == 0) {
    if (!d->permutations) { delete g; return fail("GRAPH_PERMUTATION_GENERATOR"); }
    g->rows = d->elements;
    g->cols = 1;
    g->perms.assign(d->permutations, d->permutations + static_cast<size_t>(d->generators) * d->elements);
    std::vector<uint8_t> seen(d->elements);
    for (uint32_t k = 0; k < d->generators; ++k) {
      std::fill(seen.begin(), seen.end(), 0);
      for (uint32_t i = 0; i < d->elements; ++i) {
        const uint32_t v = g->perms[static_cast<size_t>(k) * d->elements + i];
        if (v >= d->elements || seen[v]) { delete g; return fail("GRAPH_PERMUTATION_GENERATOR"); }
        seen[v] = 1;
      }
    }
  } else {
    if (!d->matrices || !d->moduli || d->rows == 0 || d->cols == 0 ||
        static_cast<uint64_t>(d->rows) * d->cols != d->elements) {
      delete g;
      return fail("GRAPH_MATRIX_SHAPE");
    }
    g->rows = d->rows;
    g->cols = d->cols;
    g->matrices.assign(d->matrices, d->matrices + static_cast<size_t>(d->generators) * d->rows * d->rows);
    g->moduli.assign(d->moduli, d->moduli + d->generators);
    for (uint32_t m : g->moduli)
      if (m != 0 && (m < 2 || m > (1u << 31))) { delete g; return fail("GRAPH_MATRIX_MODULUS"); }
  }
  int rc = cuda_status(cudaSetDevice(dev));
  if (rc) { set_message(error, cap, "CUDA_SET_DEVICE"); delete g; return rc; }
  rc = cuda_status(cudaStreamCreateWithFlags(&g->stream, cudaStreamNonBlocking));
  if (rc) { set_message(error, cap, "CUDA_STREAM"); delete g; return rc; }
  for (DeviceBuffer* b : {&g->bitmap, &g->front, &g->next, &g->table, &g->bank[0], &g->bank[1], &g->bank[2],
                          &g->program, &g->control_buf, &g->scratch, &g->buckets, &g->shard_meta, &g->group_meta,
                          &g->loop_buf, &g->transp_buf})
    b->stream = g->stream;
  retain_pool_memory(dev);
  for (cudaEvent_t* e : {&g->ev_run[0], &g->ev_run[1], &g->ev_kernel[0], &g->ev_kernel[1]}) {
    rc = cuda_status(cudaEventCreate(e));
    if (rc) { set_message(error, cap, "CUDA_EVENT"); delete g; return rc; }
  }
  int sms = 0;
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) == cudaSuccess && sms > 0) g->sm_count = sms;
  g->analyse();
  *out = g;
  return MGBFS2_OK;
}

// The product of the position components' multiset domains
// (permutation_bitmap.rs:61-143): components are the classes of i ~ g[i] over
// all generators, ordered by their first position, with their positions
// ascending.  False when a component's domain or the product overflows, or
// there are more than kMaxComponents components.
bool build_product_domain(uint32_t n, uint32_t bits, uint32_t distinct, const uint32_t* codes, uint32_t gens,
                          const uint32_t* perms, ProductDomain* out) {
  if (!n || n > 16 || (bits != 4 && bits != 8) || !distinct || distinct > 16 || n * bits > 64) return false;
  std::vector<uint32_t> parent(n);
  for (uint32_t i = 0; i < n; ++i) parent[i] = i;
  auto root = [&](uint32_t x) {
    while (parent[x] != x) x = parent[x] = parent[parent[x]];
    return x;
  };
  for (uint32_t k = 0; k < gens; ++k)
    for (uint32_t i = 0; i < n; ++i) {
      const uint32_t v = perms[static_cast<size_t>(k) * n + i];
      if (v >= n) return false;
      parent[root(i)] = root(v);
    }
  std::map<uint32_t, std::vector<uint32_t>> members;  // first position -> positions
  std::map<uint32_t, uint32_t> first;                  // root -> first position
  for (uint32_t i = 0; i < n; ++i) {
    const uint32_t r = root(i);
    if (!first.count(r)) first[r] = i;
    members[first[r]].push_back(i);
  }
  if (members.size() > kMaxComponents) return false;
  ProductDomain d{};
  d.bits = bits;
  d.distinct = distinct;
  d.total = 1;
  for (auto& kv : members) {
    const uint32_t c = d.components++;
    std::vector<uint32_t> counts(distinct, 0);
    for (uint32_t j = 0; j < kv.second.size(); ++j) {
      d.positions[c] |= static_cast<unsigned long long>(kv.second[j]) << (4 * j);
      if (codes[kv.second[j]] >= distinct) return false;
      counts[codes[kv.second[j]]]++;
    }
    d.length[c] = static_cast<uint32_t>(kv.second.size());
    std::vector<uint32_t> present;
    for (uint32_t code = 0; code < distinct; ++code) {
      if (counts[code]) present.push_back(counts[code]);
      if (code < 8) d.lanes[c][0] |= static_cast<unsigned long long>(counts[code]) << (8 * code);
      else d.lanes[c][1] |= static_cast<unsigned long long>(counts[code]) << (8 * (code - 8));
    }
    d.radix[c] = multinomial(present);
    if (d.radix[c] == UINT64_MAX) return false;
    d.total = sat_mul(d.total, d.radix[c]);
    if (d.total == UINT64_MAX) return false;
  }
  *out = d;
  return true;
}

// Packing, inverse closure, rank domain, state bound and Coxeter certificate.
void Graph::analyse() {
  const uint32_t n = elements;
  inverse_closed = false;
  if (kind == 0) {
    // Dense codes: i-th smallest distinct label -> i.
    labels = start;
    std::sort(labels.begin(), labels.end());
    labels.erase(std::unique(labels.begin(), labels.end()), labels.end());
    distinct = static_cast<uint32_t>(labels.size());
    codes.resize(n);
    for (uint32_t i = 0; i < n; ++i)
      codes[i] = static_cast<uint32_t>(std::lower_bound(labels.begin(), labels.end(), start[i]) - labels.begin());
    bits = 4;
    while (bits < 32 && (1ull << bits) < distinct) bits *= 2;
    packed = static_cast<uint64_t>(n) * bits <= 64;
    if (packed) {
      start_word = 0;
      for (uint32_t i = 0; i < n; ++i) start_word |= static_cast<uint64_t>(codes[i]) << (bits * i);
      key_mask = (n * bits == 64) ? ~0ull : ((1ull << (n * bits)) - 1);
    }
    code_counts.assign(distinct, 0);
    for (uint32_t c : codes) code_counts[c]++;
    // Inverse closure (graph_definition.py:84-92).
    std::map<std::vector<uint32_t>, int> available;
    for (uint32_t k = 0; k < gens; ++k)
      available[std::vector<uint32_t>(perms.begin() + static_cast<size_t>(k) * n,
                                      perms.begin() + static_cast<size_t>(k + 1) * n)] = 1;
    inverse_closed = true;
    for (uint32_t k = 0; k < gens && inverse_closed; ++k) {
      std::vector<uint32_t> inv(n);
      for (uint32_t i = 0; i < n; ++i) inv[perms[static_cast<size_t>(k) * n + i]] = i;
      if (!available.count(inv)) inverse_closed = false;
    }
    // Rank domain of the bitmap: the multiset permutations of the start.
    rank_total = multinomial(code_counts);
    lehmer = packed && bits == 4 && distinct == n && n <= 16;
    rank_ok = packed && (bits == 4 || bits == 8) && distinct <= 16 && rank_total != UINT64_MAX;
    // State bound: positions in one cycle component of the generators keep
    // their labels; the product of per-component multinomials bounds the
    // orbit (generic_memory.rs:82-108).
    std::vector<uint32_t> parent(n);
    for (uint32_t i = 0; i < n; ++i) parent[i] = i;
    auto root = [&](uint32_t x) {
      while (parent[x] != x) x = parent[x] = parent[parent[x]];
      return x;
    };
    for (uint32_t k = 0; k < gens; ++k)
      for (uint32_t i = 0; i < n; ++i) {
        const uint32_t a = root(i), b = root(perms[static_cast<size_t>(k) * n + i]);
        parent[a] = b;
      }
    std::map<uint32_t, std::map<uint32_t, uint32_t>> comp;
    for (uint32_t i = 0; i < n; ++i) comp[root(i)][codes[i]]++;
    state_bound = 1;
    for (auto& c : comp) {
      std::vector<uint32_t> counts;
      for (auto& kv : c.second) counts.push_back(kv.second);
      state_bound = sat_mul(state_bound, multinomial(counts));
    }
    // The product domain, when the components split the positions and it is
    // smaller than the whole multiset domain.
    product = false;
    if (packed && (bits == 4 || bits == 8) && distinct <= 16 && comp.size() > 1 && n <= 16 && state_bound < rank_total)
      product = build_product_domain(n, bits, distinct, codes.data(), gens, perms.data(), &product_domain) &&
                product_domain.components > 1;
    if (orbit_bound) state_bound = std::min(state_bound, orbit_bound);
    // Coxeter certificate: generators = all adjacent transpositions, distinct
    // labels -> layer k holds the permutations with k inversions.
    coxeter.clear();
    if (distinct == n && gens == n - 1 && n >= 2 && n <= 32) {
      std::vector<std::vector<uint32_t>> expected;
      for (uint32_t i = 0; i + 1 < n; ++i) {
        std::vector<uint32_t> p(n);
        for (uint32_t j = 0; j < n; ++j) p[j] = j;
        std::swap(p[i], p[i + 1]);
        expected.push_back(p);
      }
      bool match = true;
      std::vector<std::vector<uint32_t>> have;
      for (uint32_t k = 0; k < gens; ++k)
        have.emplace_back(perms.begin() + static_cast<size_t>(k) * n, perms.begin() + static_cast<size_t>(k + 1) * n);
      std::sort(have.begin(), have.end());
      std::sort(expected.begin(), expected.end());
      match = have == expected;
      if (match) {
        std::vector<unsigned __int128> sizes{1};
        for (uint32_t i = 1; i <= n; ++i) {
          std::vector<unsigned __int128> out(sizes.size() + i - 1);
          unsigned __int128 window = 0;
          for (size_t j = 0; j < out.size(); ++j) {
            if (j < sizes.size()) window += sizes[j];
            if (j >= i) window -= sizes[j - i];
            out[j] = window;
          }
          sizes.swap(out);
        }
        for (auto s : sizes) coxeter.push_back(s > UINT64_MAX ? UINT64_MAX : static_cast<uint64_t>(s));
      }
    }
  } else {
    packed = packed_matrix = false;
    state_bound = orbit_bound;
    // Canonical same-modulus entries bound the orbit (workload_geometry.py:21-36).
    bool same = !moduli.empty();
    for (uint32_t m : moduli) same = same && m == moduli[0];
    if (same && moduli[0]) {
      const uint32_t m = moduli[0];
      bool canonical = true;
      for (int64_t v : start) canonical = canonical && v >= 0 && v < static_cast<int64_t>(m);
      uint64_t b = 1;
      for (size_t i = 0; i < start.size(); ++i) b = sat_mul(b, m);
      if (!canonical) b = b == UINT64_MAX ? b : b + 1;
      state_bound = state_bound ? std::min(state_bound, b) : b;
      // Packing: entries of ceil(log2 m) bits, the word's top bit left clear
      // (so no state equals the empty marker), and every partial sum of a row
      // of |coefficients| times (m - 1) inside int64.
      uint32_t eb = 1;
      while ((1ull << eb) < m) ++eb;
      bool fits = canonical && static_cast<uint64_t>(n) * eb < 64 && cols <= kMatrixMaxCols;
      for (uint32_t k = 0; k < gens && fits; ++k)
        for (uint32_t i = 0; i < rows && fits; ++i) {
          unsigned __int128 sum = 0;
          for (uint32_t j = 0; j < rows; ++j) {
            const int64_t v = matrices[static_cast<size_t>(k) * rows * rows + i * rows + j];
            const unsigned __int128 a = v < 0 ? static_cast<unsigned __int128>(-(v + 1)) + 1 : v;
            sum += a * (m - 1);
          }
          fits = sum <= static_cast<unsigned __int128>(INT64_MAX);
        }
      if (fits) {
        packed = packed_matrix = true;
        bits = eb;
        key_mask = (1ull << (n * eb)) - 1;
        start_word = 0;
        for (uint32_t i = 0; i < n; ++i) start_word |= static_cast<uint64_t>(start[i]) << (eb * i);
        rank_total = b;  // m^entries, the radix-rank domain
        rank_ok = rank_total != UINT64_MAX;
      }
    }
    inverse_closed = matrix_inverse_closed();
  }
  build_program();
}

// Displacement-group programs of the packed generators.
void Graph::build_program() {
  term_begin.assign(1, 0);
  terms.clear();
  if (packed_matrix) {
    build_matrix_program();
    return;
  }
  if (!packed) return;
  const uint32_t n = elements;
  for (uint32_t k = 0; k < gens; ++k) {
    std::map<int, uint64_t> groups;  // displacement -> mask of destination symbols
    for (uint32_t i = 0; i < n; ++i) {
      const int src = static_cast<int>(perms[static_cast<size_t>(k) * n + i]);
      const uint64_t sym = (bits == 64) ? ~0ull : ((1ull << bits) - 1);
      groups[src - static_cast<int>(i)] |= sym << (bits * i);
    }
    for (auto& kv : groups) {
      Term t;
      t.mask = kv.second;
      const int shift = kv.first * static_cast<int>(bits);
      t.rshift = shift > 0 ? static_cast<uint32_t>(shift) : 0u;
      t.lshift = shift < 0 ? static_cast<uint32_t>(-shift) : 0u;
      terms.push_back(t);
    }
    term_begin.push_back(static_cast<uint32_t>(terms.size()));
  }
  // Parent-edge table, appended after the gens + 1 term offsets: inverse[g] =
  // first generator equal to g^-1.  Tags need ceil(log2(gens + 1)) spare bits
  // above the packed key; without them (or without inverse closure) the
  // kernels tag nothing and skip nothing.
  gen_shift = 0;
  std::vector<uint32_t> inverse(gens, 0xffffffffu);
  if (inverse_closed) {
    for (uint32_t k = 0; k < gens; ++k) {
      std::vector<uint32_t> inv(n);
      for (uint32_t i = 0; i < n; ++i) inv[perms[static_cast<size_t>(k) * n + i]] = i;
      for (uint32_t h = 0; h < gens && inverse[k] == 0xffffffffu; ++h)
        if (std::equal(inv.begin(), inv.end(), perms.begin() + static_cast<size_t>(h) * n)) inverse[k] = h;
    }
    const uint32_t key_bits = n * bits, tag_bits = 32 - __builtin_clz(gens);
    if (key_bits + tag_bits <= 64) gen_shift = key_bits;
  }
  term_begin.insert(term_begin.end(), inverse.begin(), inverse.end());
}

static std::vector<int64_t> mat_mul_mod(const std::vector<int64_t>& a, const std::vector<int64_t>& b, uint32_t n,
                                        uint32_t m, uint32_t mod);

// Program of packed modular matrices: generator g's rows x rows coefficients
// as term masks g * rows^2 .., then the parent-edge table: inverse[g] = the
// first generator h with M_h . M_g = I (mod m), whose child of a child of g
// is the parent itself.
void Graph::build_matrix_program() {
  const uint32_t r = rows, m = moduli[0];
  for (uint32_t k = 0; k < gens; ++k) {
    for (uint32_t i = 0; i < r; ++i) {
      std::vector<std::pair<uint32_t, uint64_t>> nz;
      for (uint32_t j = 0; j < r; ++j) {
        int64_t v = matrices[static_cast<size_t>(k) * r * r + i * r + j] % static_cast<int64_t>(m);
        if (v < 0) v += m;
        if (v) nz.emplace_back(j, static_cast<uint64_t>(v));
      }
      if (nz.size() == 1 && nz[0].second == 1) {
        terms.push_back(Term{1ull, nz[0].first, i | kMatrixCopy});
      } else {
        for (auto& z : nz) terms.push_back(Term{z.second, z.first, i});
      }
    }
    term_begin.push_back(static_cast<uint32_t>(terms.size()));
  }
  std::vector<int64_t> eye(static_cast<size_t>(r) * r, 0);
  for (uint32_t i = 0; i < r; ++i) eye[i * r + i] = 1;
  auto reduced = [&](uint32_t k) {
    std::vector<int64_t> a(matrices.begin() + static_cast<size_t>(k) * r * r,
                           matrices.begin() + static_cast<size_t>(k + 1) * r * r);
    for (auto& v : a) {
      v %= static_cast<int64_t>(m);
      if (v < 0) v += m;
    }
    return a;
  };
  std::vector<uint32_t> inverse(gens, 0xffffffffu);
  bool any = false;
  for (uint32_t k = 0; k < gens; ++k) {
    for (uint32_t h = 0; h < gens && inverse[k] == 0xffffffffu; ++h)
      if (mat_mul_mod(reduced(h), reduced(k), r, r, m) == eye) inverse[k] = h;
    any = any || inverse[k] != 0xffffffffu;
  }
  gen_shift = 0;
  const uint32_t key_bits = elements * bits, tag_bits = 32 - __builtin_clz(gens);
  if (any && key_bits + tag_bits <= 64) gen_shift = key_bits;
  term_begin.insert(term_begin.end(), inverse.begin(), inverse.end());
}

// graph_definition.py:93-108, restated over int64 with wrap-before-modulus.
static std::vector<int64_t> mat_mul_mod(const std::vector<int64_t>& a, const std::vector<int64_t>& b, uint32_t n,
                                        uint32_t m, uint32_t mod) {
  std::vector<int64_t> out(static_cast<size_t>(n) * m);
  for (uint32_t i = 0; i < n; ++i)
    for (uint32_t j = 0; j < m; ++j) {
      uint64_t total = 0;
      for (uint32_t k = 0; k < n; ++k)
        total += static_cast<uint64_t>(a[i * n + k]) * static_cast<uint64_t>(b[static_cast<size_t>(k) * m + j]);
      int64_t v = static_cast<int64_t>(total);
      if (mod) {
        v %= static_cast<int64_t>(mod);
        if (v < 0) v += mod;
      }
      out[static_cast<size_t>(i) * m + j] = v;
    }
  return out;
}

bool Graph::matrix_inverse_closed() const {
  const uint32_t n = rows;
  for (uint32_t m : moduli)
    if (m != moduli[0]) return false;
  const uint32_t mod = moduli[0];
  if (mod && (mod & (mod - 1))) {
    for (uint32_t k = 0; k < gens; ++k)
      for (uint32_t i = 0; i < n; ++i) {
        unsigned __int128 s = 0;
        for (uint32_t j = 0; j < n; ++j) {
          const int64_t v = matrices[static_cast<size_t>(k) * n * n + i * n + j];
          const unsigned __int128 a = v < 0 ? static_cast<unsigned __int128>(-(v + 1)) + 1 : v;
          s += a * (mod - 1);
        }
        if (s > static_cast<unsigned __int128>(INT64_MAX)) return false;
      }
  }
  std::vector<int64_t> eye(static_cast<size_t>(n) * n, 0);
  for (uint32_t i = 0; i < n; ++i) eye[i * n + i] = 1;
  auto gen = [&](uint32_t k) {
    return std::vector<int64_t>(matrices.begin() + static_cast<size_t>(k) * n * n,
                                matrices.begin() + static_cast<size_t>(k + 1) * n * n);
  };
  auto compose = [&](uint32_t a, uint32_t b) {
    std::vector<int64_t> right = gen(b);
    if (mod)
      for (auto& v : right) {
        v %= static_cast<int64_t>(mod);
        if (v < 0) v += mod;
      }
    return mat_mul_mod(gen(a), right, n, n, mod);
  };
  for (uint32_t a = 0; a < gens; ++a) {
    bool found = false;
    for (uint32_t b = 0; b < gens && !found; ++b) found = compose(a, b) == eye && compose(b, a) == eye;
    if (!found) return false;
  }
  for (uint32_t k = 0; k < gens; ++k)
    if (moduli[k])
      for (int64_t v : start)
        if (v < 0 || v >= static_cast<int64_t>(moduli[k])) return false;
  return true;
}

Graph::~Graph() {
  release();
  for (cudaEvent_t e : {ev_run[0], ev_run[1], ev_kernel[0], ev_kernel[1]})
    if (e) cudaEventDestroy(e);
  if (stream) cudaStreamDestroy(stream);
}

void Graph::release() {
  cudaSetDevice(device);
  // The pinned mirrors go back to the process-wide cache, where another
  // handle may take them: no copy of this handle's may still be in flight.
  if (stream) cudaStreamSynchronize(stream);
  // Nothing is in flight now: the buffers go to the device cache, where the
  // next handle on this device takes them without a pool allocation.
  for (DeviceBuffer* b : {&bitmap, &front, &next, &table, &bank[0], &bank[1], &bank[2], &program, &control_buf,
                          &scratch, &buckets, &shard_meta, &group_meta, &loop_buf, &transp_buf})
    b->release_to_cache(device);
  wide_release();
  if (host_control) {
    pinned_give(host_control);
    host_control = nullptr;
  }
  if (host_meta) {
    pinned_give(host_meta);
    host_meta = nullptr;
  }
  if (host_group) {
    pinned_give(host_group);
    host_group = nullptr;
  }
  front_grouped = false;
}

// Mapped buffers.  On a B200 a stream-ordered pool allocation of tens of GB
// took 0.07-1.8 s (8-64 GB, at random), giving it back up to 1 s, and a freed
// block that the pool keeps is no use to the next, larger one; creating and
// mapping 32 GB of physical memory took 27 ms, releasing it 22 ms.  So buffers
// from kMappedMin bytes up reserve a virtual range of the device's size once
// and grow in place by mapping the missing tail (a BFS near the memory's
// limit maps each byte once), give memory back at once when freed, and are
// kept mapped for the next handle when their handle is destroyed.  The
// driver's calls come through cudaGetDriverEntryPoint (no link against the
// driver library).
namespace {
constexpr size_t kMappedMin = 1ull << 30;

struct MappedApi {
  bool ok = false;
  size_t granularity = 0, total = 0;  // mapping granularity, device memory
  CUmemAllocationProp prop{};
  CUresult (*create)(CUmemGenericAllocationHandle*, size_t, const CUmemAllocationProp*, unsigned long long) = nullptr;
  CUresult (*reserve)(CUdeviceptr*, size_t, size_t, CUdeviceptr, unsigned long long) = nullptr;
  CUresult (*map)(CUdeviceptr, size_t, size_t, CUmemGenericAllocationHandle, unsigned long long) = nullptr;
  CUresult (*access)(CUdeviceptr, size_t, const CUmemAccessDesc*, size_t) = nullptr;
  CUresult (*unmap)(CUdeviceptr, size_t) = nullptr;
  CUresult (*release)(CUmemGenericAllocationHandle) = nullptr;
  CUresult (*address_free)(CUdeviceptr, size_t) = nullptr;
  CUresult (*granule)(size_t*, const CUmemAllocationProp*, CUmemAllocationGranularity_flags) = nullptr;
};

std::mutex mapped_lock;
std::map<int, MappedApi> mapped_apis;
std::map<int, uint64_t> mapped_total;  // physical bytes mapped by this process, per device

template <typename F>
bool entry_point(const char* name, F* fn) {
  void* p = nullptr;
  cudaDriverEntryPointQueryResult found = cudaDriverEntryPointSymbolNotFound;
  if (cudaGetDriverEntryPoint(name, &p, cudaEnableDefault, &found) != cudaSuccess ||
      found != cudaDriverEntryPointSuccess || !p) {
    cudaGetLastError();
    return false;
  }
  *fn = reinterpret_cast<F>(p);
  return true;
}

const MappedApi& mapped_api(int device) {
  std::lock_guard<std::mutex> hold(mapped_lock);
  auto it = mapped_apis.find(device);
  if (it != mapped_apis.end()) return it->second;
  MappedApi& a = mapped_apis[device];
  a.prop.type = CU_MEM_ALLOCATION_TYPE_PINNED;
  a.prop.location.type = CU_MEM_LOCATION_TYPE_DEVICE;
  a.prop.location.id = device;
  a.ok = entry_point("cuMemCreate", &a.create) && entry_point("cuMemAddressReserve", &a.reserve) &&
         entry_point("cuMemMap", &a.map) && entry_point("cuMemSetAccess", &a.access) &&
         entry_point("cuMemUnmap", &a.unmap) && entry_point("cuMemRelease", &a.release) &&
         entry_point("cuMemAddressFree", &a.address_free) &&
         entry_point("cuMemGetAllocationGranularity", &a.granule) &&
         a.granule(&a.granularity, &a.prop, CU_MEM_ALLOC_GRANULARITY_RECOMMENDED) == CUDA_SUCCESS &&
         a.granularity > 0;
  size_t free_now = 0;
  if (a.ok && cudaMemGetInfo(&free_now, &a.total) != cudaSuccess) {
    cudaGetLastError();
    a.ok = false;
  }
  return a;
}

uint64_t mapped_bytes(int device) {
  std::lock_guard<std::mutex> hold(mapped_lock);
  auto it = mapped_total.find(device);
  return it == mapped_total.end() ? 0 : it->second;
}

void mapped_add(int device, int64_t delta) {
  std::lock_guard<std::mutex> hold(mapped_lock);
  mapped_total[device] += static_cast<uint64_t>(delta);
}

size_t round_up(size_t x, size_t g) { return (x + g - 1) / g * g; }
}  // namespace

namespace {
// Mapped buffers given back by destroyed handles, per device, still mapped: a
// new handle takes one (the smallest that holds its request, else the largest,
// grown in place) without a driver call.  Beyond kMappedCacheEntries the
// smallest is unmapped.
constexpr size_t kMappedCacheEntries = 16;
std::map<int, std::vector<DeviceBuffer>> mapped_cache;  // under mapped_lock
std::map<int, uint64_t> mapped_cache_total;

// Unmaps and releases a mapped buffer with no work in flight.
void unmap_buffer(DeviceBuffer* b) {
  const MappedApi& a = mapped_api(b->device);
  CUdeviceptr at = reinterpret_cast<CUdeviceptr>(b->ptr);
  for (const auto& c : b->chunks) {
    a.unmap(at, c.second);
    a.release(c.first);
    at += c.second;
  }
  a.address_free(reinterpret_cast<CUdeviceptr>(b->ptr), b->span);
  mapped_add(b->device, -static_cast<int64_t>(b->bytes));
  b->chunks.clear();
  b->span = 0;
  b->ptr = nullptr;
  b->bytes = 0;
}

// The smallest cached buffer that holds `want`, else the largest smaller
// one, to be grown.  With `tight` (little free device memory) a buffer of
// more than twice `want` is left in the cache: it would keep memory that the
// request does not use, where other buffers of the run need it (a grouped
// S14 BFS followed by a routed one in the same process).
bool mapped_cache_take(int device, size_t want, DeviceBuffer* b, bool tight) {
  std::lock_guard<std::mutex> hold(mapped_lock);
  std::vector<DeviceBuffer>& v = mapped_cache[device];
  size_t pick = v.size();
  for (size_t i = 0; i < v.size(); ++i) {
    const size_t have = v[i].bytes;
    if (tight && have >= want && have / 2 > want) continue;
    if (pick == v.size()) {
      pick = i;
      continue;
    }
    const bool fits = have >= want, best_fits = v[pick].bytes >= want;
    if (fits ? (!best_fits || have < v[pick].bytes) : (!best_fits && have > v[pick].bytes)) pick = i;
  }
  if (pick == v.size()) return false;
  b->ptr = v[pick].ptr;
  b->bytes = v[pick].bytes;
  b->span = v[pick].span;
  b->device = v[pick].device;
  b->chunks.swap(v[pick].chunks);
  mapped_cache_total[device] -= b->bytes;
  v.erase(v.begin() + static_cast<std::ptrdiff_t>(pick));
  return true;
}

void mapped_cache_give(DeviceBuffer* b) {
  DeviceBuffer evicted;
  {
    std::lock_guard<std::mutex> hold(mapped_lock);
    std::vector<DeviceBuffer>& v = mapped_cache[b->device];
    v.push_back(*b);
    mapped_cache_total[b->device] += b->bytes;
    if (v.size() > kMappedCacheEntries) {
      size_t small = 0;
      for (size_t i = 1; i < v.size(); ++i)
        if (v[i].bytes < v[small].bytes) small = i;
      evicted = v[small];
      mapped_cache_total[b->device] -= evicted.bytes;
      v.erase(v.begin() + static_cast<std::ptrdiff_t>(small));
    }
  }
  b->chunks.clear();
  b->span = 0;
  b->ptr = nullptr;
  b->bytes = 0;
  if (evicted.span) unmap_buffer(&evicted);
}

uint64_t mapped_cache_bytes(int device) {
  std::lock_guard<std::mutex> hold(mapped_lock);
  auto it = mapped_cache_total.find(device);
  return it == mapped_cache_total.end() ? 0 : it->second;
}

// Unmaps every cached mapped buffer of `device` (none has work in flight).
void mapped_cache_drain(int device) {
  std::vector<DeviceBuffer> v;
  {
    std::lock_guard<std::mutex> hold(mapped_lock);
    v.swap(mapped_cache[device]);
    mapped_cache_total[device] = 0;
  }
  for (DeviceBuffer& b : v) unmap_buffer(&b);
}
}  // namespace

// Maps the tail [bytes, target) of a mapped buffer.  A buffer that is not yet
// mapped first gives back its pool block and takes a cached mapped buffer, or
// reserves a virtual range of the device's size.  The mapped part keeps its
// contents.  A chunk that finds no free memory is retried once after the
// device caches and the pool's idle memory are given back.
static int grow_mapped(DeviceBuffer* b, int device, size_t want, bool exact) {
  const MappedApi& a = mapped_api(device);
  if (!b->span) {
    b->free();
    // Tight: under a quarter of the device free outside the caches.
    size_t free_bytes = 0;
    const bool tight = device_free_bytes(device, &free_bytes) == MGBFS2_OK && free_bytes < a.total / 4;
    if (!mapped_cache_take(device, want, b, tight)) {
      const size_t span = round_up(std::max(want, a.total), a.granularity);
      CUdeviceptr va = 0;
      if (a.reserve(&va, span, 0, 0, 0) != CUDA_SUCCESS) return MGBFS2_OUT_OF_MEMORY;
      b->ptr = reinterpret_cast<void*>(va);
      b->span = span;
      b->device = device;
    }
    if (want <= b->bytes) return MGBFS2_OK;
  }
  size_t target = round_up(want, a.granularity);
  if (!exact) target = std::max(target, round_up(b->bytes + b->bytes / 4, a.granularity));
  if (target > b->span) return MGBFS2_OUT_OF_MEMORY;
  const size_t delta = target - b->bytes;
  CUmemGenericAllocationHandle h = 0;
  CUresult r = a.create(&h, delta, &a.prop, 0);
  if (r == CUDA_ERROR_OUT_OF_MEMORY) {
    cudaMemPool_t pool;
    device_cache_drain(device, b->stream);
    if (cudaStreamSynchronize(b->stream) == cudaSuccess && cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess &&
        cudaMemPoolTrimTo(pool, 0) == cudaSuccess)
      r = a.create(&h, delta, &a.prop, 0);
    cudaGetLastError();
  }
  if (r != CUDA_SUCCESS) return r == CUDA_ERROR_OUT_OF_MEMORY ? MGBFS2_OUT_OF_MEMORY : MGBFS2_CUDA_BASE + static_cast<int>(r);
  const CUdeviceptr at = reinterpret_cast<CUdeviceptr>(b->ptr) + b->bytes;
  CUmemAccessDesc rw{};
  rw.location = a.prop.location;
  rw.flags = CU_MEM_ACCESS_FLAGS_PROT_READWRITE;
  if ((r = a.map(at, delta, 0, h, 0)) != CUDA_SUCCESS) {
    a.release(h);
    return MGBFS2_CUDA_BASE + static_cast<int>(r);
  }
  if ((r = a.access(at, delta, &rw, 1)) != CUDA_SUCCESS) {
    a.unmap(at, delta);
    a.release(h);
    return MGBFS2_CUDA_BASE + static_cast<int>(r);
  }
  b->chunks.emplace_back(h, delta);
  b->bytes = target;
  mapped_add(device, static_cast<int64_t>(delta));
  return MGBFS2_OK;
}

// Stream-ordered allocations from the device's default memory pool, which
// keeps freed memory reserved (release threshold = max) so that regrowing a
// buffer, or a new graph handle in the same process, reuses it without device
// synchronisation.  Growth is geometric (x1.5) so a BFS regrows O(log) times.
// From kMappedMin bytes on, mapped buffers (grow_mapped).
int DeviceBuffer::ensure(size_t want, bool exact) {
  if (want <= bytes) return MGBFS2_OK;
  int device = 0;
  if (cudaGetDevice(&device) != cudaSuccess) {
    cudaGetLastError();
    return MGBFS2_CUDA_BASE;
  }
  if (span || (want >= kMappedMin && mapped_api(device).ok)) return grow_mapped(this, device, want, exact);
  const size_t grown = exact ? want : std::max(want, bytes + bytes / 2);
  free();
  void* p = nullptr;
  size_t cached = 0;
  if (device_cache_take(device, grown, &p, &cached)) {
    ptr = p;
    bytes = cached;
    return MGBFS2_OK;
  }
  cudaError_t e = cudaMallocAsync(&p, grown, stream);
  if (e == cudaErrorMemoryAllocation && device_cache_bytes(device)) {
    // Plans count the cached buffers as free memory: give them back to the
    // pool (stream-ordered, so this stream may reuse them at once) and retry.
    cudaGetLastError();
    device_cache_drain(device, stream);
    e = cudaMallocAsync(&p, grown, stream);
  }
  cudaMemPool_t pool;
  if (e == cudaErrorMemoryAllocation && pool_idle_bytes(device) &&
      cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
    // The pool keeps what it was given back (release threshold: all), in
    // blocks that may each be too small for this one: once the frees in
    // flight are done, hand the idle memory to the driver and retry.
    cudaGetLastError();
    if (cudaStreamSynchronize(stream) == cudaSuccess && cudaMemPoolTrimTo(pool, 0) == cudaSuccess)
      e = cudaMallocAsync(&p, grown, stream);
  }
  if (e != cudaSuccess) {
    cudaGetLastError();
    return e == cudaErrorMemoryAllocation ? MGBFS2_OUT_OF_MEMORY : cuda_status(e);
  }
  ptr = p;
  bytes = grown;
  return MGBFS2_OK;
}

void DeviceBuffer::free() {
  if (span) {
    // Work in flight may still use the range: unmap once the stream is done.
    cudaStreamSynchronize(stream);
    unmap_buffer(this);
  } else if (ptr) {
    cudaFreeAsync(ptr, stream);
  }
  ptr = nullptr;
  bytes = 0;
}

void DeviceBuffer::release_to_cache(int device) {
  if (span) mapped_cache_give(this);
  if (ptr) device_cache_give(device, ptr, bytes);
  ptr = nullptr;
  bytes = 0;
}

namespace {
std::mutex device_cache_mutex;
std::map<int, std::multimap<size_t, void*>> device_cache;  // device -> (bytes -> buffer)
std::map<int, uint64_t> device_cache_total;
constexpr size_t kDeviceCacheEntries = 64;  // per device; the smallest are freed beyond it
}  // namespace

bool device_cache_take(int device, size_t want, void** ptr, size_t* bytes) {
  std::lock_guard<std::mutex> lock(device_cache_mutex);
  auto d = device_cache.find(device);
  if (d == device_cache.end()) return false;
  auto it = d->second.lower_bound(want);
  if (it == d->second.end()) return false;
  *ptr = it->second;
  *bytes = it->first;
  device_cache_total[device] -= it->first;
  d->second.erase(it);
  return true;
}

void device_cache_give(int device, void* ptr, size_t bytes) {
  void* evicted = nullptr;
  {
    std::lock_guard<std::mutex> lock(device_cache_mutex);
    auto& entries = device_cache[device];
    entries.emplace(bytes, ptr);
    device_cache_total[device] += bytes;
    if (entries.size() > kDeviceCacheEntries) {
      evicted = entries.begin()->second;
      device_cache_total[device] -= entries.begin()->first;
      entries.erase(entries.begin());
    }
  }
  // An evicted buffer has no work in flight either: free it in stream order
  // on the legacy stream of the current device, which is `device` here.
  if (evicted) cudaFreeAsync(evicted, 0);
}

uint64_t device_cache_bytes(int device) {
  uint64_t mapped = mapped_cache_bytes(device);
  std::lock_guard<std::mutex> lock(device_cache_mutex);
  auto it = device_cache_total.find(device);
  return mapped + (it == device_cache_total.end() ? 0 : it->second);
}

// Frees every cached buffer of `device` into its pool, in the order of
// `stream` (the current device must be `device`).
void device_cache_drain(int device, cudaStream_t stream) {
  std::multimap<size_t, void*> entries;
  {
    std::lock_guard<std::mutex> lock(device_cache_mutex);
    entries.swap(device_cache[device]);
    device_cache_total[device] = 0;
  }
  for (auto& kv : entries) cudaFreeAsync(kv.second, stream);
  mapped_cache_drain(device);
}

// Frees every cached buffer of `device` and returns the pool's unused memory
// to the device.
int device_cache_release(int device) {
  std::multimap<size_t, void*> entries;
  {
    std::lock_guard<std::mutex> lock(device_cache_mutex);
    entries.swap(device_cache[device]);
    device_cache_total[device] = 0;
  }
  int previous = 0;
  cudaError_t e = cudaGetDevice(&previous);
  if (e == cudaSuccess) e = cudaSetDevice(device);
  for (auto& kv : entries)
    if (e == cudaSuccess) e = cudaFreeAsync(kv.second, 0);
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  if (e == cudaSuccess) mapped_cache_drain(device);
  cudaMemPool_t pool;
  if (e == cudaSuccess) e = cudaDeviceGetDefaultMemPool(&pool, device);
  if (e == cudaSuccess) e = cudaMemPoolTrimTo(pool, 0);
  cudaSetDevice(previous);
  return cuda_status(e);
}

namespace {
std::mutex pinned_mutex;
std::multimap<size_t, void*> pinned_free;   // capacity -> idle buffer
std::map<void*, size_t> pinned_size;        // every buffer the cache made -> capacity
size_t pinned_idle_bytes = 0;
constexpr size_t kPinnedIdleLimit = 64ull << 20;
}  // namespace

int pinned_take(size_t bytes, void** out) {
  size_t cap = 4096;
  while (cap < bytes) cap *= 2;
  {
    std::lock_guard<std::mutex> lock(pinned_mutex);
    auto it = pinned_free.find(cap);
    if (it != pinned_free.end()) {
      *out = it->second;
      pinned_free.erase(it);
      pinned_idle_bytes -= cap;
      return MGBFS2_OK;
    }
  }
  void* p = nullptr;
  if (int rc = cuda_status(cudaMallocHost(&p, cap))) return rc;
  std::lock_guard<std::mutex> lock(pinned_mutex);
  pinned_size[p] = cap;
  *out = p;
  return MGBFS2_OK;
}

void pinned_give(void* ptr) {
  if (!ptr) return;
  std::unique_lock<std::mutex> lock(pinned_mutex);
  const auto it = pinned_size.find(ptr);
  if (it == pinned_size.end()) return;
  const size_t cap = it->second;
  if (pinned_idle_bytes + cap <= kPinnedIdleLimit) {
    pinned_free.emplace(cap, ptr);
    pinned_idle_bytes += cap;
    return;
  }
  pinned_size.erase(it);
  lock.unlock();
  cudaFreeHost(ptr);
}

int retain_pool_memory(int device) {
  cudaMemPool_t pool;
  cudaError_t e = cudaDeviceGetDefaultMemPool(&pool, device);
  if (e != cudaSuccess) return cuda_status(e);
  uint64_t threshold = UINT64_MAX;
  return cuda_status(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &threshold));
}

// Bytes the pool holds reserved but unused: allocatable without new mappings.
// Free device memory, as cudaMemGetInfo reports it.  On shared hosts the call
// itself sometimes takes tens of milliseconds (44-98 ms seen in a sequence of
// 30 plans), which a plan per handle would pay at random.  So the first query
// of a device is synchronous; afterwards plans read the last answer, corrected
// by the change in this process's pool reservation since it was taken (the
// memory the library itself allocated or gave back in between), and an answer
// older than two seconds is refreshed by a background thread.
namespace {

struct FreeMemory {
  std::chrono::steady_clock::time_point when;
  size_t free = 0;
  uint64_t reserved = 0;
  bool valid = false;
};

std::mutex free_memory_lock;
std::map<int, FreeMemory> free_memory;
bool free_memory_refreshing = false;  // one refresh at a time, any device

// Device memory this process holds through the library: the pool's
// reservation and the mapped buffers.
uint64_t pool_reserved_bytes(int device) {
  cudaMemPool_t pool;
  uint64_t reserved = 0;
  if (cudaDeviceGetDefaultMemPool(&pool, device) != cudaSuccess ||
      cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReservedMemCurrent, &reserved) != cudaSuccess) {
    cudaGetLastError();
    reserved = 0;
  }
  return reserved + mapped_bytes(device);
}

// The refresher thread of the process; joined at exit (a query in flight
// ends first).
struct FreeMemoryRefresher {
  std::thread worker;
  ~FreeMemoryRefresher() {
    if (worker.joinable()) worker.join();
  }
};
FreeMemoryRefresher free_memory_refresher;

void refresh_free_memory(int device) {
  size_t free_now = 0, total = 0;
  const bool ok = cudaSetDevice(device) == cudaSuccess && cudaMemGetInfo(&free_now, &total) == cudaSuccess;
  const uint64_t reserved = pool_reserved_bytes(device);
  if (!ok) cudaGetLastError();
  std::lock_guard<std::mutex> hold(free_memory_lock);
  FreeMemory& e = free_memory[device];
  if (ok) {
    e.when = std::chrono::steady_clock::now();
    e.free = free_now;
    e.reserved = reserved;
    e.valid = true;
  }
  free_memory_refreshing = false;
}

}  // namespace

int device_free_bytes(int device, size_t* free_bytes, bool fresh) {
  const uint64_t reserved = pool_reserved_bytes(device);
  if (!fresh) {
    std::lock_guard<std::mutex> hold(free_memory_lock);
    FreeMemory& e = free_memory[device];
    if (e.valid) {
      const int64_t grown = static_cast<int64_t>(reserved) - static_cast<int64_t>(e.reserved);
      const int64_t est = static_cast<int64_t>(e.free) - grown;
      *free_bytes = est > 0 ? static_cast<size_t>(est) : 0;
      if (!free_memory_refreshing && std::chrono::steady_clock::now() - e.when > std::chrono::seconds(2)) {
        free_memory_refreshing = true;
        // The previous refresh has cleared the flag, its last use of the
        // lock: joining it here cannot wait on this lock.
        if (free_memory_refresher.worker.joinable()) free_memory_refresher.worker.join();
        free_memory_refresher.worker = std::thread(refresh_free_memory, device);
      }
      return MGBFS2_OK;
    }
  }
  size_t free_now = 0, total = 0;
  const cudaError_t err = cudaMemGetInfo(&free_now, &total);
  if (err != cudaSuccess) return cuda_status(err);
  std::lock_guard<std::mutex> hold(free_memory_lock);
  FreeMemory& e = free_memory[device];
  e.when = std::chrono::steady_clock::now();
  e.free = free_now;
  e.reserved = reserved;
  e.valid = true;
  *free_bytes = free_now;
  return MGBFS2_OK;
}

uint64_t pool_idle_bytes(int device) {
  cudaMemPool_t pool;
  if (cudaDeviceGetDefaultMemPool(&pool, device) != cudaSuccess) return 0;
  uint64_t reserved = 0, used = 0;
  if (cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReservedMemCurrent, &reserved) != cudaSuccess ||
      cudaMemPoolGetAttribute(pool, cudaMemPoolAttrUsedMemCurrent, &used) != cudaSuccess)
    return 0;
  return reserved > used ? reserved - used : 0;
}

// ---------------------------------------------------------------------------
// Plain planner.

int Graph::make_plan(const mgbfs2_plan_request* req, mgbfs2_plan_info* out) {
  TraceRange range("mgbfs2.plan");
  mgbfs2_plan_request r{};
  if (req) r = *req;
  if (r.visited > MGBFS2_VISITED_HASH3 || r.dedup > MGBFS2_DEDUP_GROUPED || r.planner > MGBFS2_PLANNER_LEARNED)
    return MGBFS2_INVALID_ARGUMENT;
  MG_CHECK(cudaSetDevice(device));
  size_t free_bytes = 0;
  if (int rc = device_free_bytes(device, &free_bytes)) return rc;
  free_bytes += pool_idle_bytes(device) + device_cache_bytes(device);
  const uint64_t reserve = r.reserve_bytes ? r.reserve_bytes : (2ull << 30);
  if (free_bytes <= reserve) return MGBFS2_OUT_OF_MEMORY;
  const uint64_t budget = free_bytes - reserve;
  memory_reserve = reserve;
  mgbfs2_plan_info p{};
  p.packed = packed;
  p.bits_per_symbol = packed ? bits : 64;
  p.key_words = packed ? 1 : wide_key_words();
  p.state_bound = state_bound;
  p.inverse_closed = inverse_closed;
  p.planner = r.planner;
  // The learned planner replaces the worst-case bound by its prediction
  // where the bound only sizes or chooses; exactness never depends on it.
  const bool learned = r.planner == MGBFS2_PLANNER_LEARNED;
  if (learned && !r.predicted_states) return MGBFS2_INVALID_ARGUMENT;
  const uint64_t expected = learned ? (state_bound ? std::min(state_bound, r.predicted_states) : r.predicted_states)
                                    : state_bound;
  learned_peak = learned ? r.predicted_peak : 0;
  // Routed and grouped layers rank over the whole Lehmer domain; asked for
  // explicitly, they keep it even where the product domain is smaller.
  use_product = product && r.dedup != MGBFS2_DEDUP_BUCKET && r.dedup != MGBFS2_DEDUP_GROUPED;
  if (r.group_chunk && (r.group_chunk < 256 || r.group_chunk > (1u << 20))) return MGBFS2_INVALID_ARGUMENT;
  if (r.blocks_per_sm > 32) return MGBFS2_INVALID_ARGUMENT;
  if (r.parents_per_thread && r.parents_per_thread != 1 && r.parents_per_thread != 2 && r.parents_per_thread != 4)
    return MGBFS2_INVALID_ARGUMENT;
  parents_per_thread = r.parents_per_thread;
  if (r.route_chunk % kRouteChunkAlign) return MGBFS2_INVALID_ARGUMENT;
  route_chunk = r.route_chunk;
  group_chunk = r.group_chunk ? r.group_chunk : kGroupChunk;
  blocks_per_sm = static_cast<int>(r.blocks_per_sm);
  p.group_chunk = group_chunk;
  p.blocks_per_sm = r.blocks_per_sm;
  p.parents_per_thread = r.parents_per_thread ? r.parents_per_thread : (gens <= 4 ? 4 : 2);
  p.shards = r.shards ? r.shards : 64;
  p.block = kBlock;
  uint32_t visited = r.visited;
  if (!packed) {
    if (visited == MGBFS2_VISITED_BITMAP) return MGBFS2_UNSUPPORTED;
    if (visited == MGBFS2_VISITED_AUTO) visited = inverse_closed ? MGBFS2_VISITED_HASH3 : MGBFS2_VISITED_HASH;
  }
  const uint64_t bitmap_bytes = rank_ok ? ((rank_domain() + 63) / 64) * 8 : UINT64_MAX;
  if (visited == MGBFS2_VISITED_AUTO) {
    // The bitmap costs total/8 bytes, an exact hash ~16 B per state: take the
    // bitmap when it is the smaller exact structure and fits comfortably.
    const bool dense = expected && rank_domain() / 128 <= expected;
    if (rank_ok && bitmap_bytes <= budget / 2 && (dense || bitmap_bytes <= (64ull << 20)))
      visited = MGBFS2_VISITED_BITMAP;
    else
      visited = inverse_closed ? MGBFS2_VISITED_HASH3 : MGBFS2_VISITED_HASH;
  }
  if (visited == MGBFS2_VISITED_BITMAP && !rank_ok) return MGBFS2_UNSUPPORTED;
  if (visited == MGBFS2_VISITED_HASH3 && !inverse_closed) return MGBFS2_INVALID_ARGUMENT;
  uint32_t dedup = r.dedup;
  if (dedup == MGBFS2_DEDUP_AUTO) {
    // A bitmap that fits in L2 takes plain atomics.  A larger Lehmer bitmap
    // takes grouped layers when every generator fills the child's first K
    // positions from the parent's first K with at most one exception (then a
    // parent group's children fall into at most N-K target groups per
    // generator), else owner-routed layers, whose shard slices fit in L2
    // whatever the generators.
    dedup = MGBFS2_DEDUP_ATOMIC;
    if (visited == MGBFS2_VISITED_BITMAP && lehmer && !use_product && bitmap_bytes > (64ull << 20) && elements <= 16) {
      const uint32_t n = elements, K = group_prefix_for(n);
      bool local = n <= 14;
      for (uint32_t k = 0; k < gens && local; ++k) {
        uint32_t outside = 0;
        for (uint32_t i = 0; i < K; ++i) outside += perms[static_cast<size_t>(k) * n + i] >= K ? 1 : 0;
        local = outside <= 1;
      }
      if (local) dedup = MGBFS2_DEDUP_GROUPED;
      else if (n * (n - 1) <= kMaxShards) dedup = MGBFS2_DEDUP_BUCKET;
    }
    // A radix bitmap larger than L2 routes by its top entry (m shards of
    // m^(E-1) bits each).
    if (visited == MGBFS2_VISITED_BITMAP && packed_matrix && bitmap_bytes > (64ull << 20) &&
        moduli[0] <= kMaxShards)
      dedup = MGBFS2_DEDUP_BUCKET;
  }
  if (visited != MGBFS2_VISITED_BITMAP && dedup == MGBFS2_DEDUP_WARP) dedup = MGBFS2_DEDUP_ATOMIC;
  const bool hash_routed =
      dedup == MGBFS2_DEDUP_BUCKET && visited == MGBFS2_VISITED_HASH && packed && !packed_matrix;
  const bool radix_routed = dedup == MGBFS2_DEDUP_BUCKET && visited == MGBFS2_VISITED_BITMAP && packed_matrix &&
                            moduli[0] <= kMaxShards;
  if ((dedup == MGBFS2_DEDUP_BUCKET || dedup == MGBFS2_DEDUP_GROUPED) &&
      !(visited == MGBFS2_VISITED_BITMAP && lehmer && !use_product) && !hash_routed && !radix_routed)
    return MGBFS2_UNSUPPORTED;
  // Sort-unique tiles hold kSortTile children: at least 16 parents per tile.
  if (dedup == MGBFS2_DEDUP_SORT && (!packed || packed_matrix || gens > kSortTile / 16)) return MGBFS2_UNSUPPORTED;
  if (radix_routed) {
    bucket_prefix = 1;
    bucket_shards = moduli[0];
    p.shards = bucket_shards;
    bucket_margin = r.bucket_margin == 0 ? 4096 : (r.bucket_margin == UINT32_MAX ? 0 : r.bucket_margin);
    bucket_min_work = r.bucket_min_work ? r.bucket_min_work : (1ull << 22);
  }
  if (dedup == MGBFS2_DEDUP_BUCKET && !hash_routed && !radix_routed) {
    // Shards = states sharing their first K symbols: N!/(N-K)! shards whose
    // bitmap slices hold (N-K)! bits.  Default: the smallest K (1 or 2) whose
    // slice is at most 8 MiB, so the slices the resident accept blocks work
    // on stay in L2; a requested shard count picks K = 2 when N < shards.
    const uint32_t n = elements;
    uint64_t fact[17] = {1};
    for (uint32_t i = 1; i <= 16; ++i) fact[i] = fact[i - 1] * i;
    uint32_t K = 1;
    if (r.shards) K = (n < r.shards && n * (n - 1) <= kMaxShards) ? 2 : 1;
    else if (fact[n - 1] / 8 > (8ull << 20) && n * (n - 1) <= kMaxShards) K = 2;
    if (n < 2 || fact[n] / fact[n - K] > kMaxShards) return MGBFS2_UNSUPPORTED;
    bucket_prefix = K;
    bucket_shards = static_cast<uint32_t>(fact[n] / fact[n - K]);
    p.shards = bucket_shards;
    bucket_margin = r.bucket_margin == 0 ? 4096 : (r.bucket_margin == UINT32_MAX ? 0 : r.bucket_margin);
    bucket_min_work = r.bucket_min_work ? r.bucket_min_work : (1ull << 22);
  }
  if (dedup == MGBFS2_DEDUP_GROUPED) {
    // Groups = states sharing their first K symbols (group_prefix_for).
    const uint32_t n = elements;
    if (n < 2 || n > 16) return MGBFS2_UNSUPPORTED;
    uint64_t fact[17] = {1};
    for (uint32_t i = 1; i <= 16; ++i) fact[i] = fact[i - 1] * i;
    const uint32_t K = group_prefix_for(n);
    if (fact[n] / fact[n - K] > kMaxGroups) return MGBFS2_UNSUPPORTED;
    group_prefix = K;
    groups = static_cast<uint32_t>(fact[n] / fact[n - K]);
    plan_group_order();
    if (int rc = plan_transpositions(!(r.options & MGBFS2_OPTION_FULL_RANK))) return rc;
    bucket_prefix = K;
    p.shards = groups;
    bucket_margin = r.bucket_margin == 0 ? 1024 : (r.bucket_margin == UINT32_MAX ? 0 : r.bucket_margin);
    bucket_min_work = r.bucket_min_work ? r.bucket_min_work : (1ull << 22);
  }
  p.visited = visited;
  p.dedup = dedup;
  parent_skip = packed && gen_shift && !(r.options & MGBFS2_OPTION_NO_PARENT_SKIP);
  host_loop_only = (r.options & MGBFS2_OPTION_HOST_LOOP) != 0;
  p.parent_skip = parent_skip;
  p.bucket_prefix = bucket_prefix;
  p.history_layers = visited == MGBFS2_VISITED_HASH3 ? 3 : 1;
  p.bitmap_bits = visited == MGBFS2_VISITED_BITMAP ? rank_domain() : 0;
  p.rank_components = visited == MGBFS2_VISITED_BITMAP ? (use_product ? product_domain.components : 1) : 0;
  // Frontier capacity: the orbit bound (or the caller's cap) within memory.
  uint64_t fixed = visited == MGBFS2_VISITED_BITMAP ? bitmap_bytes : 0;
  if (fixed >= budget) return MGBFS2_OUT_OF_MEMORY;
  uint64_t cap = state_bound ? state_bound : UINT64_MAX;
  if (!coxeter.empty()) cap = std::min(cap, *std::max_element(coxeter.begin(), coxeter.end()));
  if (r.capacity) cap = std::min(cap, r.capacity);
  const uint64_t per_state = packed ? 16 : 16ull * (wide_key_words() + 2);
  const uint64_t hash_per_state = visited == MGBFS2_VISITED_BITMAP ? 0 : (visited == MGBFS2_VISITED_HASH3 ? 48 : 16);
  cap = std::min(cap, (budget - fixed) / (per_state + hash_per_state));
  if (cap == 0) return MGBFS2_OUT_OF_MEMORY;
  p.capacity = cap;
  hash_quotient = false;
  if (visited == MGBFS2_VISITED_HASH) {
    // All-visited table: sized for the state bound (or the frontier cap) at
    // the growth threshold.  Fused layers of one-word keys take 32-bit
    // quotient slots when the key bits beyond the slot index leave at least
    // 8 bits for the probe distance.
    // The learned plan sizes it for the prediction plus a quarter.
    const uint64_t predicted = learned ? expected + expected / 4 + 1024 : 0;
    const uint64_t want = std::min(learned ? predicted : (state_bound ? state_bound : cap), cap);
    const uint32_t key_bits = key_mask == ~0ull ? 64u : 64u - static_cast<uint32_t>(__builtin_clzll(key_mask));
    const bool quotient_ok = packed && !hash_routed && (dedup == MGBFS2_DEDUP_ATOMIC) &&
                             !(r.options & MGBFS2_OPTION_WIDE_SLOTS);
    // Longer linear-probe chains, not table bytes, cost the most: a half-full
    // threshold (S11: 2^27 slots, load 0.3) measured 1.6x faster than 3/4.
    const uint32_t load = r.hash_load_percent ? std::min<uint32_t>(95, std::max<uint32_t>(10, r.hash_load_percent))
                                              : 50u;
    const uint64_t slots = std::max<uint64_t>(1024, next_pow2((want * 100 + load - 1) / load));
    uint32_t s_bits = 0;
    while ((1ull << s_bits) < slots) ++s_bits;
    hash_quotient = quotient_ok && key_bits <= s_bits + 24;
    hash_load = load;
    p.table_slots = slots;
    p.table_slot_bytes = hash_quotient ? 4 : 8;
    p.hash_load_percent = load;
    // Quotient-slot layers stage a tile's children in 2048 entries: one
    // parent per thread fits a tile in one flush with the most tiles in
    // flight (S11 LRX: 3.85 ms; 3.96 ms with two parents; 4.78 ms with four
    // and a flush per generator).
    if (hash_quotient && !parents_per_thread) parents_per_thread = p.parents_per_thread = 1;
  }
  if (hash_routed) {
    // Hash-routed layers: shard = table region of a key's home slot, regions
    // of about 16 MB (L2-sized), a power of two between 1 and kMaxShards.
    uint32_t regions = 1;
    while (regions < kMaxShards && p.table_slots * 8 / (2ull * regions) >= (16ull << 20)) regions *= 2;
    bucket_prefix = 0;
    bucket_shards = regions;
    p.shards = regions;
    bucket_margin = r.bucket_margin == 0 ? 4096 : (r.bucket_margin == UINT32_MAX ? 0 : r.bucket_margin);
    bucket_min_work = r.bucket_min_work ? r.bucket_min_work : (1ull << 22);
  }
  p.device_bytes = fixed + (visited == MGBFS2_VISITED_HASH ? p.table_slots * p.table_slot_bytes : 0);
  if (!packed) {
    int rc = wide_plan(&p, budget);
    if (rc) return rc;
  }
  // Fixed allocations of the plan.
  int rc = MGBFS2_OK;
  if (p.visited == MGBFS2_VISITED_BITMAP) rc = bitmap.ensure(bitmap_bytes);
  if (!rc) rc = control_buf.ensure(sizeof(Control));
  if (!rc && packed) rc = program.ensure(terms.size() * sizeof(Term) + term_begin.size() * sizeof(uint32_t) + 16);
  if (!rc && !host_control) rc = pinned_take(sizeof(Control), reinterpret_cast<void**>(&host_control));
  if (rc) return rc;
  if (packed) {
    MG_CHECK(cudaMemcpyAsync(program.ptr, terms.data(), terms.size() * sizeof(Term), cudaMemcpyHostToDevice, stream));
    MG_CHECK(cudaMemcpyAsync(static_cast<char*>(program.ptr) + terms.size() * sizeof(Term), term_begin.data(),
                             term_begin.size() * sizeof(uint32_t), cudaMemcpyHostToDevice, stream));
    MG_CHECK(cudaStreamSynchronize(stream));
  }
  plan = p;
  planned = true;
  if (out) *out = p;
  return MGBFS2_OK;
}

// ---------------------------------------------------------------------------
// Kernel selection.

using ExpandFn = void (*)(ExpandParams);

// Bitmap graphs with at least this many generators take the kernels with the
// candidate-parallel small-layer mode (S10 Coxeter, 9 generators: 1.38 ->
// 1.10 ms per BFS); with fewer a thread's generators are few enough that the
// mode does not pay (S11 LRX, 3 generators: 2.15 -> 2.31 ms with it).
constexpr uint32_t kCandidateMinGens = 5;

template <int V, bool W, bool C>
static ExpandFn pick_lehmer(uint32_t n) {
  switch (n) {
#define MG_CASE(K) \
  case K:          \
    return expand_packed<V, K, W, C>;
    MG_CASE(2) MG_CASE(3) MG_CASE(4) MG_CASE(5) MG_CASE(6) MG_CASE(7) MG_CASE(8) MG_CASE(9) MG_CASE(10)
    MG_CASE(11) MG_CASE(12) MG_CASE(13) MG_CASE(14) MG_CASE(15) MG_CASE(16)
#undef MG_CASE
    default:
      return nullptr;
  }
}

static ExpandFn pick_sorted(int visit, uint32_t n) {
  switch (visit) {
    case V_LEHMER:
      switch (n) {
#define MG_CASE(K) \
  case K:          \
    return expand_sorted<V_LEHMER, K>;
        MG_CASE(2) MG_CASE(3) MG_CASE(4) MG_CASE(5) MG_CASE(6) MG_CASE(7) MG_CASE(8) MG_CASE(9) MG_CASE(10)
        MG_CASE(11) MG_CASE(12) MG_CASE(13) MG_CASE(14) MG_CASE(15) MG_CASE(16)
#undef MG_CASE
        default:
          return nullptr;
      }
    case V_MULTISET:
      return expand_sorted<V_MULTISET, 0>;
    case V_PRODUCT:
      return expand_sorted<V_PRODUCT, 0>;
    case V_HASH:
      return expand_sorted<V_HASH, 0>;
    default:
      return expand_sorted<V_HASH3, 0>;
  }
}

// Bitmap kernels with many generators (cand) carry the candidate-parallel
// mode for small layers; hash and matrix kernels always do.
static ExpandFn pick_expand(int visit, bool warp, uint32_t n, bool matrix, bool cand) {
  if (matrix) {
    switch (visit) {
      case V_RADIX:
        return warp ? expand_packed<V_RADIX, kMatrixN, true, true> : expand_packed<V_RADIX, kMatrixN, false, true>;
      case V_HASH:
        return expand_packed<V_HASH, kMatrixN, false, true>;
      case V_HASHQ:
        return expand_packed<V_HASHQ, kMatrixN, false, true>;
      case V_HASH3:
        return expand_packed<V_HASH3, kMatrixN, false, true>;
      default:
        return nullptr;
    }
  }
  switch (visit) {
    case V_LEHMER:
      if (cand) return warp ? pick_lehmer<V_LEHMER, true, true>(n) : pick_lehmer<V_LEHMER, false, true>(n);
      return warp ? pick_lehmer<V_LEHMER, true, false>(n) : pick_lehmer<V_LEHMER, false, false>(n);
    case V_MULTISET:
      if (cand) return warp ? expand_packed<V_MULTISET, 0, true, true> : expand_packed<V_MULTISET, 0, false, true>;
      return warp ? expand_packed<V_MULTISET, 0, true, false> : expand_packed<V_MULTISET, 0, false, false>;
    case V_PRODUCT:
      if (cand) return warp ? expand_packed<V_PRODUCT, 0, true, true> : expand_packed<V_PRODUCT, 0, false, true>;
      return warp ? expand_packed<V_PRODUCT, 0, true, false> : expand_packed<V_PRODUCT, 0, false, false>;
    case V_HASH:
      return expand_packed<V_HASH, 0, false, true>;
    case V_HASHQ:
      return expand_packed<V_HASHQ, 0, false, true>;
    default:
      return expand_packed<V_HASH3, 0, false, true>;
  }
}

using RouteFn = void (*)(RouteParams);
using AcceptFn = void (*)(AcceptParams);

static void pick_bucket(uint32_t n, uint32_t prefix, RouteFn* route, AcceptFn* accept) {
  switch (n) {
#define MG_CASE(K)                                                       \
  case K:                                                                \
    *route = prefix == 1 ? route_lehmer<K, 1> : route_lehmer<K, 2>;      \
    *accept = prefix == 1 ? accept_lehmer<K, 1> : accept_lehmer<K, 2>;   \
    return;
    MG_CASE(2) MG_CASE(3) MG_CASE(4) MG_CASE(5) MG_CASE(6) MG_CASE(7) MG_CASE(8) MG_CASE(9) MG_CASE(10)
    MG_CASE(11) MG_CASE(12) MG_CASE(13) MG_CASE(14) MG_CASE(15) MG_CASE(16)
#undef MG_CASE
    default:
      *route = nullptr;
      *accept = nullptr;
  }
}

using GroupedFn = void (*)(GroupedParams);

static GroupedFn pick_grouped(uint32_t n, uint32_t prefix) {
  if (prefix == 4) return n == 14 ? expand_grouped<14, 4, false> : nullptr;
  switch (n) {
#define MG_CASE(K)                                                                               \
  case K:                                                                                        \
    return prefix == 1 ? expand_grouped<K, 1, false>                                             \
                       : (prefix == 2 ? expand_grouped<K, 2, false> : expand_grouped<K, 3, false>);
    MG_CASE(4) MG_CASE(5) MG_CASE(6) MG_CASE(7) MG_CASE(8) MG_CASE(9) MG_CASE(10) MG_CASE(11) MG_CASE(12)
    MG_CASE(13) MG_CASE(14) MG_CASE(15) MG_CASE(16)
#undef MG_CASE
    case 2:
    case 3:
      return prefix == 1 ? (n == 2 ? expand_grouped<2, 1, false> : expand_grouped<3, 1, false>) : nullptr;
    default:
      return nullptr;
  }
}

// The incremental-rank instantiations: adjacent-transposition generators and a
// 32-bit in-group rank (8 <= N - K <= 12).
static GroupedFn pick_grouped_transp(uint32_t n, uint32_t prefix) {
  switch (n * 4 + prefix) {
#define MG_CASE(N, K) \
  case N * 4 + K:     \
    return expand_grouped<N, K, true>;
    MG_CASE(9, 1) MG_CASE(10, 1) MG_CASE(11, 1) MG_CASE(12, 1) MG_CASE(13, 1)
    MG_CASE(10, 2) MG_CASE(11, 2) MG_CASE(12, 2) MG_CASE(13, 2) MG_CASE(14, 2)
    MG_CASE(11, 3) MG_CASE(12, 3) MG_CASE(13, 3) MG_CASE(14, 3) MG_CASE(15, 3)
#undef MG_CASE
    default:
      return nullptr;
  }
}

// Visiting order of the groups.  A generator whose child keeps all of its
// first K symbols among the parent's first K sends a parent group to one
// target group; otherwise its target groups are fixed by the parent
// positions it does take from the first K (LRX: L takes positions 1, 2 and R
// positions 0, 1).  Groups are enumerated lexicographically over their
// symbols with the positions most of those generators share outermost, so
// consecutive work items reuse the same target groups while they are in L2.
void Graph::plan_group_order() {
  const uint32_t n = elements, K = group_prefix;
  std::vector<uint32_t> weight(K, 0);
  for (uint32_t k = 0; k < gens; ++k) {
    const uint32_t* g = perms.data() + static_cast<size_t>(k) * n;
    bool inside = true;
    for (uint32_t i = 0; i < K; ++i) inside = inside && g[i] < K;
    if (inside) continue;
    for (uint32_t i = 0; i < K; ++i)
      if (g[i] < K) ++weight[g[i]];
  }
  std::vector<uint32_t> pos(K);
  for (uint32_t i = 0; i < K; ++i) pos[i] = i;
  std::stable_sort(pos.begin(), pos.end(), [&](uint32_t a, uint32_t b) { return weight[a] > weight[b]; });
  group_order.clear();
  std::vector<uint32_t> sym(K, 0);
  std::vector<uint8_t> used(n, 0);
  // Depth-first over positions pos[0], pos[1], ...; at full depth the group is
  // the mixed-radix number of the Lehmer digits of (sym[0], ..., sym[K-1]).
  std::vector<uint32_t> next_symbol(K, 0);
  uint32_t depth = 0;
  while (true) {
    if (depth == K) {
      uint64_t index = 0;
      for (uint32_t i = 0; i < K; ++i) {
        uint32_t digit = sym[i];
        for (uint32_t j = 0; j < i; ++j) digit -= sym[j] < sym[i] ? 1 : 0;
        index = index * (n - i) + digit;
      }
      group_order.push_back(static_cast<uint32_t>(index));
      --depth;
      used[sym[pos[depth]]] = 0;
      continue;
    }
    uint32_t& c = next_symbol[depth];
    while (c < n && used[c]) ++c;
    if (c == n) {
      c = 0;
      if (depth == 0) break;
      --depth;
      used[sym[pos[depth]]] = 0;
      continue;
    }
    sym[pos[depth]] = c;
    used[c] = 1;
    ++c;
    ++depth;
  }
}

// Adjacent-transposition generators (g swaps positions t-1 and t): the
// incremental-rank form of the grouped layers needs, per generator, t and the
// weights of Lehmer digits t-1 and t in the group number (the first K digits,
// mixed radix N, N-1, ...) and in the in-group rank (the other digits,
// weight (N-1-j)!).
int Graph::plan_transpositions(bool allowed) {
  const uint32_t n = elements, K = group_prefix;
  group_transp = false;
  if (!allowed || gens > kMaxTranspGens || !pick_grouped_transp(n, K)) return MGBFS2_OK;
  std::vector<uint32_t> info;
  auto wg = [&](uint32_t j) {
    if (j >= K) return 0u;
    uint32_t w = 1;
    for (uint32_t k = j + 1; k < K; ++k) w *= n - k;
    return w;
  };
  auto wi = [&](uint32_t j) {
    if (j < K) return 0u;
    uint32_t w = 1;
    for (uint32_t k = 2; k <= n - 1 - j; ++k) w *= k;
    return w;
  };
  for (uint32_t k = 0; k < gens; ++k) {
    const uint32_t* g = perms.data() + static_cast<size_t>(k) * n;
    uint32_t moved = 0, t = 0;
    for (uint32_t i = 0; i < n; ++i)
      if (g[i] != i) {
        ++moved;
        t = i;  // the larger moved position
      }
    if (moved != 2 || t == 0 || g[t] != t - 1 || g[t - 1] != t) return MGBFS2_OK;
    info.insert(info.end(), {t, wg(t - 1), wg(t), wi(t - 1), wi(t)});
  }
  int rc = transp_buf.ensure(info.size() * sizeof(uint32_t));
  if (rc) return rc;
  MG_CHECK(cudaMemcpyAsync(transp_buf.ptr, info.data(), info.size() * sizeof(uint32_t), cudaMemcpyHostToDevice,
                           stream));
  MG_CHECK(cudaStreamSynchronize(stream));
  group_transp = true;
  return MGBFS2_OK;
}

// Meta layout of a grouped layer (R = groups + 1 regions, the spill last), in
// uint64 words: region_begin[R] | region_count[R] | item_prefix[R + 1] |
// next_begin[R] | next_cap[R] | next_count[R] | work, then region_order[R] as
// uint32.
static size_t group_meta_words(uint32_t groups) { return 6 * static_cast<size_t>(groups + 1) + 2; }
static size_t group_meta_bytes(uint32_t groups) {
  return group_meta_words(groups) * sizeof(unsigned long long) + (groups + 1) * sizeof(uint32_t);
}

// Lays out the next frontier of a grouped layer and uploads the layer's meta.
// Group regions get the current layer's distribution of `count` scaled by the
// last growth ratio, plus 25 % and bucket_margin; the spill region gets the exact
// bound `cap`, so every winner has a place, where the device memory holds it
// with room to spare; else at least half the group regions, as far as the memory
// goes (S14 under LRX: the exact bound of its 4.6e9-state layer would need 74 GB
// of spill beside two 46 GB frontiers).  A winner that finds no place raises
// ERR_FRONTIER_OVERFLOW: the run ends, no state is lost.
int Graph::grouped_setup(uint64_t count, uint64_t prev_count, uint64_t cap, void** fn, size_t* smem_total,
                         size_t smem, uint64_t* items, uint32_t* grid) {
  const uint32_t G = groups, R = groups + 1;
  int rc = MGBFS2_OK;
  const size_t words = group_meta_words(G), bytes = group_meta_bytes(G);
  if (!host_group && (rc = pinned_take(bytes, reinterpret_cast<void**>(&host_group)))) return rc;
  if ((rc = group_meta.ensure(bytes))) return rc;
  uint32_t* order = reinterpret_cast<uint32_t*>(host_group + words);
  unsigned long long* rb = host_group;
  unsigned long long* rcnt = rb + R;
  unsigned long long* ip = rcnt + R;
  unsigned long long* nb = ip + R + 1;
  unsigned long long* nc = nb + R;
  unsigned long long* ncount = nc + R;
  if (front_grouped) {
    for (uint32_t r = 0; r < R; ++r) {
      rb[r] = front_begin[r];
      rcnt[r] = front_count[r];
    }
  } else {
    for (uint32_t r = 0; r < R; ++r) rb[r] = rcnt[r] = 0;
    rcnt[G] = count;  // a contiguous frontier is all spill
  }
  for (uint32_t j = 0; j < G; ++j) order[j] = group_order[j];
  order[G] = G;  // the spill last
  uint64_t run = 0;
  for (uint32_t j = 0; j < R; ++j) {
    ip[j] = run;
    run += (rcnt[order[j]] + group_chunk - 1) / group_chunk;
  }
  ip[R] = run;
  *items = run;
  const double growth = prev_count ? static_cast<double>(count) / static_cast<double>(prev_count) : gens;
  const double predicted = std::min(static_cast<double>(cap), growth * static_cast<double>(count));
  next_begin.assign(R, 0);
  next_cap.assign(R, 0);
  uint64_t total = 0;
  for (uint32_t g = 0; g < G; ++g) {
    const double frac = front_grouped && count ? static_cast<double>(rcnt[g]) / static_cast<double>(count)
                                              : 1.0 / static_cast<double>(G);
    const uint64_t c = static_cast<uint64_t>(frac * predicted * 1.25) + bucket_margin;
    nb[g] = next_begin[g] = total;
    nc[g] = next_cap[g] = c;
    total += c;
  }
  constexpr uint64_t W = sizeof(unsigned long long);
  uint64_t spill = cap;
  if ((total + spill + 2) * W > next.bytes) {
    // Growing `next` frees it first: its bytes count as free here.  Before a
    // memory-bounded layout the device is asked afresh.
    uint64_t room = 0;
    for (bool fresh : {false, true}) {
      size_t free_bytes = 0;
      if ((rc = device_free_bytes(device, &free_bytes, fresh))) return rc;
      const uint64_t avail = free_bytes + pool_idle_bytes(device) + device_cache_bytes(device) + next.bytes;
      room = avail > memory_reserve ? (avail - memory_reserve) / W : 0;
      if ((total + spill + 2) / 2 * 3 <= room) break;
    }
    if ((total + spill + 2) / 2 * 3 <= room) {
      if ((rc = next.ensure((total + spill + 2) * W))) return rc;
    } else {
      // Memory-bounded: a spill of at least half the group regions (or the
      // bound), the buffer grown with 25 % headroom within the memory, so
      // that it is reallocated every few layers rather than every layer.
      if (room < total + bucket_margin + 2) return MGBFS2_OUT_OF_MEMORY;
      const uint64_t least = total + std::min<uint64_t>(cap, total / 2) + 2;
      if (next.bytes / W < least && (rc = next.ensure(std::min<uint64_t>(room, least + least / 4) * W, true)))
        return rc;
      spill = std::min<uint64_t>(cap, next.bytes / W - total - 2);
    }
  }
  nb[G] = next_begin[G] = total;
  nc[G] = next_cap[G] = spill;
  total += spill;
  for (uint32_t r = 0; r < R; ++r) ncount[r] = 0;
  ncount[R] = 0;  // work counter
  MG_CHECK(cudaMemcpyAsync(group_meta.ptr, host_group, bytes, cudaMemcpyHostToDevice, stream));
  GroupedFn f = group_transp ? pick_grouped_transp(elements, group_prefix) : pick_grouped(elements, group_prefix);
  if (!f) return MGBFS2_UNSUPPORTED;
  *fn = reinterpret_cast<void*>(f);
  *smem_total = sizeof(GroupedSmem) + smem + (group_transp ? 5 * sizeof(uint32_t) * gens : 0);
  MG_CHECK(cudaFuncSetAttribute(reinterpret_cast<const void*>(f), cudaFuncAttributeMaxDynamicSharedMemorySize,
                                static_cast<int>(*smem_total)));
  // Eight blocks per SM (the 164 KB configuration, 92 KB left as L1) for the
  // plain kernel; the transposition kernel's registers allow five.
  const int blocks = set_carveout(reinterpret_cast<const void*>(f), *smem_total, want_blocks(kGroupBlocksPerSM));
  *grid = static_cast<uint32_t>(std::max<uint64_t>(1, std::min<uint64_t>(static_cast<uint64_t>(blocks) * sm_count, *items)));
  return MGBFS2_OK;
}

// After a grouped layer: the per-region counts (read back into host_group)
// become the layout of the buffer that is about to be the frontier.
int Graph::grouped_finish() {
  const uint32_t G = groups, R = groups + 1;
  const unsigned long long* ncount = host_group + 5 * static_cast<size_t>(R) + 1;
  front_begin = next_begin;
  front_count.assign(R, 0);
  for (uint32_t r = 0; r < R; ++r) front_count[r] = std::min<uint64_t>(ncount[r], next_cap[r]);
  (void)G;
  return MGBFS2_OK;
}

// Copies the grouped `front` into `next` as one contiguous array and swaps.
int Graph::gather_front(uint64_t count) {
  if (!front_grouped) return MGBFS2_OK;
  const uint32_t R = groups + 1;
  int rc = MGBFS2_OK;
  if ((rc = group_meta.ensure(group_meta_bytes(groups)))) return rc;
  unsigned long long* rb = host_group;
  unsigned long long* rcnt = rb + R;
  unsigned long long* op = rcnt + R;
  uint64_t run = 0;
  for (uint32_t r = 0; r < R; ++r) {
    rb[r] = front_begin[r];
    rcnt[r] = front_count[r];
    op[r] = run;
    run += front_count[r];
  }
  if (run != count) return MGBFS2_STATE;
  if ((rc = next.ensure((count + 2) * sizeof(unsigned long long)))) return rc;
  MG_CHECK(cudaMemcpyAsync(group_meta.ptr, host_group, 3 * R * sizeof(unsigned long long), cudaMemcpyHostToDevice,
                           stream));
  const unsigned long long* meta = static_cast<const unsigned long long*>(group_meta.ptr);
  gather_regions<<<std::min<uint32_t>(R, 4 * sm_count), kBlock, 0, stream>>>(
      static_cast<const unsigned long long*>(front.ptr), meta, meta + R, meta + 2 * R, R,
      static_cast<unsigned long long*>(next.ptr));
  ++launches;
  MG_CHECK(cudaGetLastError());
  // The copy reads host_group at execution time: finish before it is reused.
  MG_CHECK(cudaStreamSynchronize(stream));
  std::swap(front, next);
  front_grouped = false;
  return MGBFS2_OK;
}

// Per-shard bucket capacities for `work` routed successors: the previous
// routed layer's shard distribution plus 20% and a fixed margin (uniform x2
// before any history), or exactly the counts of the failed attempt when
// `exact` (the redo after an overflow, which cannot overflow again).
int Graph::bucket_setup(uint64_t work, bool exact) {
  const uint32_t S = bucket_shards;
  int rc = MGBFS2_OK;
  const size_t meta_bytes = (3 * kMaxShards + 1) * sizeof(unsigned long long);
  if (!host_meta && (rc = pinned_take(meta_bytes, reinterpret_cast<void**>(&host_meta)))) return rc;
  if ((rc = shard_meta.ensure(meta_bytes))) return rc;
  unsigned long long* begin = host_meta;
  unsigned long long* cap = host_meta + kMaxShards;
  const unsigned long long* counts = host_meta + 2 * kMaxShards;
  uint64_t total = 0;
  for (uint32_t s = 0; s < S; ++s) {
    uint64_t c;
    if (exact) {
      c = counts[s];
    } else if (shard_history_total) {
      const double frac = static_cast<double>(shard_history[s]) / static_cast<double>(shard_history_total);
      c = static_cast<uint64_t>(frac * static_cast<double>(work) * 1.2) + bucket_margin;
    } else {
      c = 2 * (work / S) + bucket_margin;
    }
    begin[s] = total;
    cap[s] = c;
    total += c;
  }
  bucket_work = work;
  if ((rc = buckets.ensure(total * sizeof(unsigned long long), bucket_alloc_exact))) return rc;
  MG_CHECK(cudaMemcpyAsync(shard_meta.ptr, host_meta, 2 * kMaxShards * sizeof(unsigned long long),
                           cudaMemcpyHostToDevice, stream));
  // Zero the shard counts and the accept work counter.
  MG_CHECK(cudaMemsetAsync(static_cast<unsigned long long*>(shard_meta.ptr) + 2 * kMaxShards, 0,
                           (kMaxShards + 1) * sizeof(unsigned long long), stream));
  return MGBFS2_OK;
}

int Graph::bucket_launch(const void* route_fn, const void* accept_fn, const ExpandParams& p, size_t smem) {
  unsigned long long* meta = static_cast<unsigned long long*>(shard_meta.ptr);
  RouteParams rp{};
  rp.frontier = p.frontier;
  rp.count = p.count;
  rp.terms = p.terms;
  rp.term_begin = p.term_begin;
  rp.gens = p.gens;
  rp.total_terms = p.total_terms;
  rp.gen_shift = p.gen_shift;
  // Parents per thread and generators per flush: at most kMaxEntries staged
  // successors per thread.
  rp.ppt = p.gens <= 3 ? 4 : (p.gens <= 6 ? 2 : 1);
  rp.group = kMaxEntries / rp.ppt;
  rp.prefix = bucket_prefix;
  rp.shards = bucket_shards;
  rp.buckets = static_cast<unsigned long long*>(buckets.ptr);
  rp.shard_begin = meta;
  rp.shard_cap = meta + kMaxShards;
  rp.shard_count = meta + 2 * kMaxShards;
  rp.control = p.control;
  rp.mat = p.mat;
  if (visit_kind() == V_HASH) {
    uint32_t shift = 0;
    while ((1ull << shift) < table_slots) ++shift;
    uint32_t rbits = 0;
    while ((1u << rbits) < bucket_shards) ++rbits;
    rp.table_mask = table_slots - 1;
    rp.key_mask = key_mask;
    rp.region_shift = shift - rbits;
  }
  const uint64_t tiles = (p.count + kBlock * rp.ppt - 1) / (kBlock * rp.ppt);
  const size_t route_smem = sizeof(RouteSmem) + smem;
  MG_CHECK(cudaFuncSetAttribute(route_fn, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(route_smem)));
  reinterpret_cast<RouteFn>(const_cast<void*>(route_fn))<<<grid_for(route_fn, route_smem, tiles), kBlock, route_smem,
                                                           stream>>>(rp);
  ++launches;
  MG_CHECK(cudaGetLastError());
  AcceptParams ap{};
  ap.buckets = static_cast<const unsigned long long*>(buckets.ptr);
  ap.shard_begin = meta;
  ap.shard_count = meta + 2 * kMaxShards;
  ap.shards = bucket_shards;
  ap.work = meta + 3 * kMaxShards;
  ap.bitmap = p.bitmap;
  ap.next = p.next;
  ap.capacity = p.capacity;
  ap.control = p.control;
  ap.table = p.table;
  ap.table_mask = p.table_mask;
  ap.key_mask = key_mask;
  ap.probe_limit = p.probe_limit;
  ap.mat = p.mat;
  reinterpret_cast<AcceptFn>(const_cast<void*>(accept_fn))<<<grid_for(accept_fn, 0, UINT32_MAX), kBlock, 0, stream>>>(ap);
  ++launches;
  MG_CHECK(cudaGetLastError());
  return MGBFS2_OK;
}

// Sizes a routed layer's next frontier (up to the exact bound `*cap`) and its
// shard buckets (the estimate of bucket_setup: the last distribution + 20 %,
// or x2 uniform, plus bucket_margin per shard) together.  Where both fit the
// device memory with room to spare the layer is one route and one accept
// pass, with the buffers' usual geometric growth.  Otherwise, and for the
// rest of the run, both grow only to sizes chosen here, with 25 % headroom so
// that a run near the memory's limit reallocates them every few layers, not
// every layer: the next frontier takes up to `*cap` (lowered to what the
// memory holds: a layer larger than that ends the run with
// ERR_FRONTIER_OVERFLOW), the buckets what is left, and a layer whose buckets
// do not fit them is routed in parent chunks of `*chunk`.  S14 under LRX with
// routed layers needs this: its 4.6e9-state layer has 13.8e9 successors, 110
// GB of buckets, on a 180 GB GPU.
int Graph::routed_setup(uint64_t count, uint64_t* cap, uint64_t* chunk) {
  const uint64_t margin = static_cast<uint64_t>(bucket_shards) * bucket_margin;
  const double per_parent = static_cast<double>(gens) * (shard_history_total ? 1.2 : 2.0);
  const auto bucket_words = [&](uint64_t parents) {
    return static_cast<uint64_t>(per_parent * static_cast<double>(parents)) + margin + 1;
  };
  constexpr uint64_t W = sizeof(unsigned long long);
  *chunk = count;
  if (route_chunk && route_chunk < count) {
    *chunk = route_chunk;
    return next.ensure((*cap + 2) * W);
  }
  const uint64_t need_next = *cap + 2, need_buckets = bucket_words(count);
  if (need_next * W <= next.bytes && need_buckets * W <= buckets.bytes) return MGBFS2_OK;
  uint64_t room = 0;
  for (bool fresh : {false, true}) {
    size_t free_bytes = 0;
    if (int rc = device_free_bytes(device, &free_bytes, fresh)) return rc;
    const uint64_t avail =
        free_bytes + pool_idle_bytes(device) + device_cache_bytes(device) + next.bytes + buckets.bytes;
    room = avail > memory_reserve ? (avail - memory_reserve) / W : 0;
    if (!bucket_alloc_exact && (need_next + need_buckets) / 2 * 3 <= room) return next.ensure(need_next * W);
  }
  bucket_alloc_exact = true;
  const uint64_t least = bucket_words(std::min<uint64_t>(count, kRouteChunkAlign));
  if (room < least + 2 + bucket_margin) return MGBFS2_OUT_OF_MEMORY;
  if (need_next * W > next.bytes) {
    const uint64_t target = std::min<uint64_t>(need_next + need_next / 4, room - least);
    if (target + buckets.bytes / W > room) buckets.free();
    if (int rc = next.ensure(target * W, true)) return rc;
  }
  *cap = std::min<uint64_t>(*cap, next.bytes / W - 2);
  const uint64_t left = room > next.bytes / W ? room - next.bytes / W : 0;
  if (need_buckets * W > buckets.bytes && (need_buckets <= left || buckets.bytes / W < left / 2)) {
    // The whole layer's buckets where they fit, else all that is left (an
    // older block is kept while it holds at least half of that).
    const uint64_t target = need_buckets <= left ? std::min<uint64_t>(need_buckets + need_buckets / 4, left) : left;
    buckets.free();
    if (int rc = buckets.ensure(target * W, true)) return rc;
  }
  const uint64_t have = buckets.bytes / W;
  if (need_buckets <= have) return MGBFS2_OK;
  const uint64_t parents =
      have > margin + 1 ? static_cast<uint64_t>(static_cast<double>(have - margin - 1) / per_parent) : 0;
  // Chunks start on 16-byte boundaries: the route kernels read parents in pairs.
  *chunk = std::max<uint64_t>(kRouteChunkAlign, parents / kRouteChunkAlign * kRouteChunkAlign);
  return MGBFS2_OK;
}

// A routed layer in parent chunks (routed_setup): route and accept one chunk at
// a time, each redone once with its exact shard counts when its buckets
// overflowed (the bitmap untouched, the next frontier's count kept).  The
// next frontier's count runs on across the chunks.
int Graph::bucket_chunks(const void* route_fn, const void* accept_fn, const ExpandParams& p, size_t smem,
                         uint64_t chunk, uint32_t* redo) {
  unsigned int* error = &static_cast<Control*>(control_buf.ptr)->error;
  unsigned long long* counts = static_cast<unsigned long long*>(shard_meta.ptr) + 2 * kMaxShards;
  for (uint64_t off = 0; off < p.count; off += chunk) {
    ExpandParams q = p;
    q.frontier = p.frontier + off;
    q.count = std::min<uint64_t>(chunk, p.count - off);
    for (int attempt = 0; attempt < 2; ++attempt) {
      int rc = bucket_setup(q.count * gens, attempt == 1);
      if (!rc) rc = bucket_launch(route_fn, accept_fn, q, smem);
      if (rc) return rc;
      MG_CHECK(cudaMemcpyAsync(host_control, control_buf.ptr, sizeof(Control), cudaMemcpyDeviceToHost, stream));
      MG_CHECK(cudaMemcpyAsync(host_meta + 2 * kMaxShards, counts, bucket_shards * sizeof(unsigned long long),
                               cudaMemcpyDeviceToHost, stream));
      MG_CHECK(cudaStreamSynchronize(stream));
      if (host_control->error != ERR_BUCKET_OVERFLOW) break;
      ++*redo;
      MG_CHECK(cudaMemsetAsync(error, 0, sizeof(unsigned int), stream));
    }
    if (host_control->error) break;
  }
  return MGBFS2_OK;
}

int Graph::visit_kind() const {
  if (plan.visited == MGBFS2_VISITED_BITMAP) {
    if (packed_matrix) return V_RADIX;
    if (use_product) return V_PRODUCT;
    return (lehmer && elements >= 2) ? V_LEHMER : V_MULTISET;
  }
  if (plan.visited == MGBFS2_VISITED_HASH) return hash_quotient ? V_HASHQ : V_HASH;
  return V_HASH3;
}

QuotientSlots Graph::quotient_slots(uint64_t slots) const {
  QuotientSlots q{};
  q.slots = static_cast<unsigned int*>(table.ptr);
  q.mask = slots - 1;
  q.s = 0;
  while ((1ull << q.s) < slots) ++q.s;
  q.bits = key_mask == ~0ull ? 64u : 64u - static_cast<uint32_t>(__builtin_clzll(key_mask));
  const uint32_t rem = q.bits > q.s ? q.bits - q.s : 0u;
  q.d = 32 - rem;
  const uint64_t most = (q.d >= 32 ? (1ull << 32) : (1ull << q.d)) - 2;  // distance field holds j + 1 < 2^D
  q.limit = static_cast<uint32_t>(std::min<uint64_t>(most, 1u << 20));
  return q;
}

int size_carveout(const void* fn, size_t smem, int want, int threads) {
  // Left to itself the runtime may pick the largest shared-memory
  // configuration for occupancy, which leaves about 28 KB of L1; the layer
  // kernels ran up to 1.5x slower there, as the L1 also stages the loads and
  // atomics in flight.
  int device = 0, smem_per_sm = 233472, reserved = 1024;
  if (cudaGetDevice(&device) != cudaSuccess ||
      cudaDeviceGetAttribute(&smem_per_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, device) != cudaSuccess ||
      cudaDeviceGetAttribute(&reserved, cudaDevAttrReservedSharedMemoryPerBlock, device) != cudaSuccess) {
    cudaGetLastError();
    smem_per_sm = 233472;
    reserved = 1024;
  }
  int by_regs = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&by_regs, fn, threads, 0) != cudaSuccess || by_regs < 1) {
    cudaGetLastError();
    by_regs = 1;
  }
  cudaFuncAttributes attr{};
  if (cudaFuncGetAttributes(&attr, fn) != cudaSuccess) {
    cudaGetLastError();
    attr.sharedSizeBytes = 0;
  }
  const size_t per_block = attr.sharedSizeBytes + smem + static_cast<size_t>(reserved);
  int blocks = std::min(want, by_regs);
  blocks = std::max(1, std::min<int>(blocks, static_cast<int>(static_cast<size_t>(smem_per_sm) / per_block)));
  // Shared-memory configurations of compute capability 9.0 and 10.0, in KB;
  // the runtime rounds a preference up to the next one, so the floor of the
  // chosen configuration's share selects exactly it.
  static constexpr int kConfigKB[] = {0, 8, 16, 32, 64, 100, 132, 164, 196, 228};
  const size_t need = static_cast<size_t>(blocks) * per_block;
  int config = smem_per_sm;
  for (int kb : kConfigKB)
    if (static_cast<size_t>(kb) * 1024 >= need) {
      config = std::min(kb * 1024, smem_per_sm);
      break;
    }
  const int pct = static_cast<int>((100ll * config) / smem_per_sm);
  if (cudaFuncSetAttribute(fn, cudaFuncAttributePreferredSharedMemoryCarveout, pct) != cudaSuccess) cudaGetLastError();
  return blocks;
}

int Graph::set_carveout(const void* fn, size_t smem, int want) {
  const int blocks = size_carveout(fn, smem, want, kBlock);
  carveout_blocks[fn] = blocks;
  return blocks;
}

uint32_t Graph::grid_for(const void* fn, size_t smem, uint64_t work_blocks) {
  int per_sm = 0;
  const auto known = carveout_blocks.find(fn);
  if (known != carveout_blocks.end()) {
    per_sm = known->second;
  } else if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, kBlock, smem) != cudaSuccess || per_sm < 1) {
    cudaGetLastError();
    per_sm = 1;
  }
  const uint64_t full = static_cast<uint64_t>(per_sm) * static_cast<uint64_t>(sm_count);
  return static_cast<uint32_t>(std::max<uint64_t>(1, std::min<uint64_t>(full, work_blocks)));
}

// ---------------------------------------------------------------------------
// Layer loop.

uint64_t Graph::next_bound(uint32_t depth, uint64_t count, uint64_t visited) const {
  // Upper bound on |L_{d+1}|: every parent yields at most g new states, at
  // most g-1 for d >= 1 on inverse-closed graphs (one edge leads back to
  // L_{d-1}); never more than the unvisited part of the orbit bound; exact on
  // certified Coxeter graphs.
  const uint64_t per = (inverse_closed && depth >= 1 && gens > 1) ? gens - 1 : gens;
  uint64_t b = sat_mul(count, per);
  if (state_bound && state_bound >= visited) b = std::min(b, state_bound - visited);
  if (!coxeter.empty()) b = depth + 1 < coxeter.size() ? std::min(b, coxeter[depth + 1]) : 0;
  return b;
}

// Graph mode: the layer loop as ONE CUDA graph.  A conditional WHILE node
// repeats {expand the frontier, loop_finalize}; loop_finalize records the new
// layer's size and a globaltimer stamp, swaps the buffers and clears the loop
// condition when the frontier is exhausted, on a device error, or when the
// layer table is full (then the host loop takes over from the device state).
// Frontier buffers (`front`, `next`) already hold `cap` states each.
int Graph::run_device_loop(const void* fn, ExpandParams* pp, size_t smem, uint64_t cap, mgbfs2_status* st,
                           double* kernel_seconds, uint64_t* count, uint64_t* visited, uint32_t* depth,
                           bool* paused) {
  constexpr uint32_t kEntries = 4096;
  const size_t head = (sizeof(LoopState) + 255) / 256 * 256;
  int rc = loop_buf.ensure(head + 2 * kEntries * sizeof(unsigned long long));
  if (rc) return rc;
  char* base = static_cast<char*>(loop_buf.ptr);
  LoopState* ls = reinterpret_cast<LoopState*>(base);
  unsigned long long* layers = reinterpret_cast<unsigned long long*>(base + head);
  unsigned long long* stamps = layers + kEntries;
  // The loop starts from the caller's state: the start (depth 0), or a
  // resumed checkpoint's deepest layer.
  const uint64_t count0 = *count, visited0 = *visited;
  const uint32_t depth0 = *depth;
  if (depth0 + 2 >= kEntries) {
    *paused = true;  // too deep for the device loop's layer table: the host loop goes on
    return MGBFS2_OK;
  }
  LoopState h{};
  h.count = count0;
  h.visited = visited0;
  h.depth = depth0;
  h.capacity = cap;
  h.gens = gens;
  const int visit = visit_kind();
  if ((visit == V_HASH || visit == V_HASHQ) && !(state_bound && table_slots * hash_load / 100 >= state_bound))
    h.table_limit = table_slots * hash_load / 100;
  h.buf[0] = static_cast<unsigned long long*>(front.ptr);
  h.buf[1] = static_cast<unsigned long long*>(next.ptr);
  h.max_entries = kEntries;
  h.layers = layers;
  h.stamps = stamps;
  MG_CHECK(cudaMemcpyAsync(ls, &h, sizeof(h), cudaMemcpyHostToDevice, stream));
  MG_CHECK(cudaMemsetAsync(control_buf.ptr, 0, sizeof(Control), stream));
  ExpandParams p = *pp;
  p.loop = ls;
  p.capacity = cap;
  const uint32_t grid = grid_for(fn, smem, UINT32_MAX);
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  cudaStream_t cap_stream = nullptr;
  auto cleanup = [&]() {
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    if (cap_stream) cudaStreamDestroy(cap_stream);
  };
  // Persistent form first: one cooperative launch runs every layer, with two
  // grid barriers per layer instead of two graph nodes.  Its grid must be
  // co-resident; a device or carveout that cannot hold it falls back to the
  // graph form below.
  bool persistent_done = false;
  cudaError_t e = cudaSuccess;
  {
    int resident = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&resident, fn, kBlock, smem) != cudaSuccess) {
      cudaGetLastError();
      resident = 0;
    }
    const auto known = carveout_blocks.find(fn);
    const int per_sm = std::min(resident, known != carveout_blocks.end() ? known->second : resident);
    if (per_sm >= 1) {
      ExpandParams q = p;
      q.persistent = 1;
      void* args[] = {&q};
      e = cudaEventRecord(ev_kernel[0], stream);
      if (e == cudaSuccess) {
        loop_start<<<1, 1, 0, stream>>>(stamps + depth0);
        e = cudaGetLastError();
      }
      if (e == cudaSuccess) {
        e = cudaLaunchCooperativeKernel(fn, dim3(per_sm * sm_count), dim3(kBlock), args, smem, stream);
        if (e == cudaErrorCooperativeLaunchTooLarge || e == cudaErrorNotSupported) {
          cudaGetLastError();
          e = cudaSuccess;  // the graph form below runs the BFS instead
        } else if (e == cudaSuccess) {
          persistent_done = true;
        }
      }
    }
  }
  if (!persistent_done && e == cudaSuccess) e = cudaGraphCreate(&graph, 0);
  cudaGraphConditionalHandle handle{};
  if (!persistent_done && e == cudaSuccess) e = cudaGraphConditionalHandleCreate(&handle, graph, 1, cudaGraphCondAssignDefault);
  cudaGraphNodeParams cp = {};
  cp.type = cudaGraphNodeTypeConditional;
  cp.conditional.handle = handle;
  cp.conditional.type = cudaGraphCondTypeWhile;
  cp.conditional.size = 1;
  cudaGraphNode_t node;
  if (!persistent_done && e == cudaSuccess) e = cudaGraphAddNode(&node, graph, nullptr, 0, &cp);
  if (!persistent_done && e == cudaSuccess) e = cudaStreamCreateWithFlags(&cap_stream, cudaStreamNonBlocking);
  if (!persistent_done && e == cudaSuccess)
    e = cudaStreamBeginCaptureToGraph(cap_stream, cp.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                      cudaStreamCaptureModeRelaxed);
  if (!persistent_done && e == cudaSuccess) {
    reinterpret_cast<void (*)(ExpandParams)>(const_cast<void*>(fn))<<<grid, kBlock, smem, cap_stream>>>(p);
    loop_finalize<<<1, 1, 0, cap_stream>>>(ls, p.control, handle);
    cudaGraph_t body = cp.conditional.phGraph_out[0];
    e = cudaStreamEndCapture(cap_stream, &body);
  }
  if (!persistent_done && e == cudaSuccess) e = cudaGraphInstantiate(&exec, graph, 0);
  if (!persistent_done && e == cudaSuccess) e = cudaEventRecord(ev_kernel[0], stream);
  if (!persistent_done && e == cudaSuccess) {
    loop_start<<<1, 1, 0, stream>>>(stamps + depth0);
    e = cudaGetLastError();
  }
  if (!persistent_done && e == cudaSuccess) e = cudaGraphLaunch(exec, stream);
  if (e == cudaSuccess) e = cudaEventRecord(ev_kernel[1], stream);
  LoopState out{};
  std::vector<unsigned long long> sizes(kEntries), times(kEntries);
  if (e == cudaSuccess) e = cudaMemcpyAsync(&out, ls, sizeof(out), cudaMemcpyDeviceToHost, stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(host_control, control_buf.ptr, sizeof(Control), cudaMemcpyDeviceToHost, stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(sizes.data(), layers, kEntries * 8, cudaMemcpyDeviceToHost, stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(times.data(), stamps, kEntries * 8, cudaMemcpyDeviceToHost, stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
  cleanup();
  if (e != cudaSuccess) return cuda_status(e);
  float ms = 0.f;
  if (cudaEventElapsedTime(&ms, ev_kernel[0], ev_kernel[1]) == cudaSuccess) *kernel_seconds += ms * 1e-3;
  // Layers 1..out.depth were recorded; layers 0..out.depth were expanded
  // unless the table filled up (then layer out.depth is still to expand).
  const uint32_t D = out.depth;
  const uint32_t expanded = out.stop == 3 ? D : D + 1;  // layers depth0 .. expanded - 1 were expanded
  auto size_at = [&](uint32_t d) { return d == depth0 ? count0 : sizes[d]; };
  for (uint32_t d = depth0 + 1; d <= D; ++d) {
    layer_sizes.push_back(sizes[d]);
    layer_seconds.push_back(static_cast<double>(times[d] - times[d - 1]) * 1e-9);
  }
  for (uint32_t d = depth0; d < expanded; ++d) {
    const uint64_t c = size_at(d);
    st->successors += c * gens;
    st->visited_tests += c * gens - (parent_skip && d > 0 ? c : 0);
  }
  launches += persistent_done ? 2 : 1 + 2 * (expanded - depth0);
  if (out.parity) std::swap(front, next);
  *count = size_at(D);
  *visited = out.visited;
  *depth = D;
  *paused = out.stop == 3;
  if (out.stop == 2) {
    st->reason = MGBFS2_REASON_RESOURCE;
    st->fatal = host_control->error ? host_control->error : ERR_FRONTIER_OVERFLOW;
    return MGBFS2_OK;
  }
  if (out.stop == 1) st->complete = 1;
  // The deepest layer sits in `front`; the layer before it is intact in `next`
  // (the last expansion appended nothing, or the loop paused before it).
  if (D >= depth0 + 2 && D >= 2 && sizes[D - 1] < 1000) {
    std::vector<uint64_t> words(sizes[D - 1]);
    MG_CHECK(cudaMemcpyAsync(words.data(), next.ptr, words.size() * 8, cudaMemcpyDeviceToHost, stream));
    MG_CHECK(cudaStreamSynchronize(stream));
    keep_small(D - 1, std::move(words));
  }
  if (D >= depth0 + 1 && D >= 1 && sizes[D] < 1000) {
    std::vector<uint64_t> words(sizes[D]);
    MG_CHECK(cudaMemcpyAsync(words.data(), front.ptr, words.size() * 8, cudaMemcpyDeviceToHost, stream));
    MG_CHECK(cudaStreamSynchronize(stream));
    keep_small(D, std::move(words));
  }
  return MGBFS2_OK;
}

int Graph::run(const mgbfs2_run_limits* limits, mgbfs2_layer_callback cb, void* user, mgbfs2_status* status) {
  if (!planned) return MGBFS2_STATE;
  TraceRange range("mgbfs2.run");
  MG_CHECK(cudaSetDevice(device));
  if (!packed) return wide_run(limits, cb, user, status);
  mgbfs2_status st{};
  // A resumed run starts from the checkpoint's layer table, deepest layer
  // (in `front`), visited structure and small-layer samples.
  const bool resume = resume_pending;
  resume_pending = false;
  if (resume) {
    layer_sizes = resume_layers;
    layer_seconds.assign(layer_sizes.size() - 1, 0.0);
  } else {
    layer_sizes.assign(1, 1);
    layer_seconds.clear();
    for (int i = 0; i < 2; ++i) {
      small_layer[i].clear();
      small_depth[i] = UINT32_MAX;
    }
  }
  launches = 0;
  const auto started = Clock::now();
  const int visit = visit_kind();
  const bool warp = plan.dedup == MGBFS2_DEDUP_WARP;
  const bool sorted = plan.dedup == MGBFS2_DEDUP_SORT;
  ExpandFn fn = sorted ? pick_sorted(visit, elements) : pick_expand(visit, warp, elements, packed_matrix, gens >= kCandidateMinGens);
  if (!fn) return MGBFS2_UNSUPPORTED;
  // Bucketed layers for large frontiers; small layers use the fused kernel.
  const bool bucketed =
      plan.dedup == MGBFS2_DEDUP_BUCKET && (visit == V_LEHMER || visit == V_HASH || visit == V_RADIX);
  RouteFn route_fn = nullptr;
  AcceptFn accept_fn = nullptr;
  if (bucketed) {
    if (visit == V_HASH) {
      route_fn = route_lehmer<0, 0>;
      accept_fn = accept_hash;
    } else if (visit == V_RADIX) {
      route_fn = route_lehmer<kRadixDomain, 1>;
      accept_fn = accept_lehmer<kRadixDomain, 1>;
    } else {
      pick_bucket(elements, bucket_prefix, &route_fn, &accept_fn);
    }
    if (!route_fn) return MGBFS2_UNSUPPORTED;
  }
  shard_history.assign(bucket_shards, 0);
  shard_history_total = 0;
  bucket_alloc_exact = false;
  const bool grouped_mode = plan.dedup == MGBFS2_DEDUP_GROUPED && visit == V_LEHMER;
  if (grouped_mode && !pick_grouped(elements, group_prefix)) return MGBFS2_UNSUPPORTED;
  front_grouped = false;

  ExpandParams p{};
  p.terms = static_cast<const Term*>(program.ptr);
  p.term_begin = reinterpret_cast<const uint32_t*>(static_cast<const char*>(program.ptr) + terms.size() * sizeof(Term));
  p.gens = gens;
  p.total_terms = static_cast<uint32_t>(terms.size());
  p.gen_shift = parent_skip ? gen_shift : 0;
  p.control = static_cast<Control*>(control_buf.ptr);
  p.key_mask = key_mask;
  p.ppt = parents_per_thread ? parents_per_thread : (gens <= 4 ? 4 : 2);
  const size_t smem = terms.size() * sizeof(Term) + term_begin.size() * sizeof(uint32_t);
  if (!sorted)
    set_carveout(reinterpret_cast<const void*>(fn), smem,
                 want_blocks(visit == V_HASHQ ? kHashQBlocksPerSM : kPackedBlocksPerSM));
  if (visit == V_PRODUCT) p.pd = product_domain;
  p.mat = matrix_action();
  if (visit == V_MULTISET) {
    p.ms.n = elements;
    p.ms.bits = bits;
    p.ms.distinct = distinct;
    p.ms.total = rank_total;
    for (uint32_t c = 0; c < distinct && c < 16; ++c) p.ms.counts[c] = code_counts[c];
  }
  int rc = MGBFS2_OK;
  double kernel_seconds = 0.0;
  MG_CHECK(cudaEventRecord(ev_run[0], stream));
  // Initial state: visited structure cleared, start seeded, frontier = {start}
  // (a resumed run keeps what the checkpoint restored).
  MG_CHECK(cudaMemsetAsync(control_buf.ptr, 0, sizeof(Control), stream));
  if (bitmap_kind(visit)) {
    if (!resume) MG_CHECK(cudaMemsetAsync(bitmap.ptr, 0, bitmap.bytes, stream));
    p.bitmap = static_cast<unsigned long long*>(bitmap.ptr);
  } else if (visit == V_HASH) {
    if (!resume) {
      table_slots = plan.table_slots;
      if ((rc = table.ensure(table_slots * 8))) return rc;
      MG_CHECK(cudaMemsetAsync(table.ptr, 0xff, table_slots * 8, stream));
    }
  } else if (visit == V_HASHQ) {
    if (!resume) {
      table_slots = plan.table_slots;
      if ((rc = table.ensure(table_slots * 4))) return rc;
      MG_CHECK(cudaMemsetAsync(table.ptr, 0, table_slots * 4, stream));
    }
    p.q = quotient_slots(table_slots);
  } else if (resume) {
    return MGBFS2_UNSUPPORTED;  // three-bank histories are not checkpointed
  } else {
    for (int b = 0; b < 3; ++b) bank_slots[b] = 0;
    bank_slots[0] = 1024;
    if ((rc = bank[0].ensure(bank_slots[0] * 8))) return rc;
    MG_CHECK(cudaMemsetAsync(bank[0].ptr, 0xff, bank_slots[0] * 8, stream));
  }
  // Graph mode: the fused bitmap or all-visited hash layers with buffers sized
  // up front (frontier capacity for every layer, hash table for every state),
  // no limits and no callback.
  const bool limited = limits && (limits->max_seconds > 0 || limits->max_layers || limits->cancel);
  const uint64_t loop_cap = std::max<uint64_t>(1, plan.capacity);
  bool device_loop = !host_loop_only && !bucketed && !grouped_mode && !limited && !cb &&
                     (bitmap_kind(visit) || visit == V_HASH || visit == V_HASHQ) &&
                     2 * (loop_cap + 2) * 8 <= (16ull << 30);
  // The device loop never grows the table: it must hold every state below
  // the growth threshold, or (a table sized by the learned planner) the loop
  // pauses before the threshold could be passed and the host loop goes on.
  if (device_loop && (visit == V_HASH || visit == V_HASHQ))
    device_loop = plan.planner == MGBFS2_PLANNER_LEARNED ||
                  (state_bound && table_slots * hash_load / 100 >= state_bound);
  // A learned plan pre-sizes the host loop's frontier buffers for its
  // predicted peak layer, so a correct prediction costs no buffer growth.
  if (!device_loop && learned_peak) {
    const uint64_t reserve = std::min<uint64_t>(plan.capacity, learned_peak + learned_peak / 4 + 1024);
    if ((rc = front.ensure((reserve + 2) * 8)) || (rc = next.ensure((reserve + 2) * 8))) return rc;
  }
  if (device_loop) {
    // A resumed frontier is already in `front`: regrowing it must keep it.
    if (resume && front.bytes < (loop_cap + 2) * 8) {
      DeviceBuffer grown;
      grown.stream = stream;
      if ((rc = grown.ensure((loop_cap + 2) * 8))) return rc;
      MG_CHECK(cudaMemcpyAsync(grown.ptr, front.ptr, last_count * 8, cudaMemcpyDeviceToDevice, stream));
      front.free();
      front = grown;
      grown.ptr = nullptr;
      grown.bytes = 0;
    }
    if ((rc = front.ensure((loop_cap + 2) * 8))) return rc;
    if ((rc = next.ensure((loop_cap + 2) * 8))) return rc;
  }
  if (!resume) {
    if ((rc = front.ensure(16))) return rc;
    MG_CHECK(cudaMemcpyAsync(front.ptr, &start_word, 8, cudaMemcpyHostToDevice, stream));
  }
  if (!resume) {
    ExpandParams s = p;
    if (visit == V_HASH) {
      s.table = static_cast<unsigned long long*>(table.ptr);
      s.table_mask = table_slots - 1;
    } else if (visit == V_HASH3) {
      s.table = static_cast<unsigned long long*>(bank[0].ptr);
      s.table_mask = bank_slots[0] - 1;
    }
    s.probe_limit = 1u << 20;
    seed_packed<<<1, 32, 0, stream>>>(s, start_word, visit, elements);
    ++launches;
    MG_CHECK(cudaGetLastError());
  }
  uint64_t count = 1, visited = 1;
  uint32_t depth = 0;
  if (resume) {
    count = layer_sizes.back();
    visited = 0;
    for (uint64_t x : layer_sizes) visited += x;
    depth = static_cast<uint32_t>(layer_sizes.size() - 1);
  } else {
    keep_small(0, std::vector<uint64_t>(1, start_word));
  }
  uint64_t peak = plan.device_bytes;
  st.reason = MGBFS2_REASON_FRONTIER_EXHAUSTED;
  bool finished = false;
  if (device_loop) {
    if (visit == V_HASH) {
      p.table = static_cast<unsigned long long*>(table.ptr);
      p.table_mask = table_slots - 1;
      p.tag = 0;
    }
    p.probe_limit = 1u << 20;
    bool paused = false;
    TraceRange loop_range(sorted ? "layers.device_loop.sorted" : "layers.device_loop.fused");
    rc = run_device_loop(reinterpret_cast<const void*>(fn), &p, smem, loop_cap, &st, &kernel_seconds, &count,
                         &visited, &depth, &paused);
    finished = rc != MGBFS2_OK || !paused;
    peak = std::max<uint64_t>(peak, bitmap.bytes + front.bytes + next.bytes + table.bytes);
  }
  for (; !finished;) {
    const double elapsed = std::chrono::duration<double>(Clock::now() - started).count();
    if (limits && limits->cancel && *limits->cancel) { st.reason = MGBFS2_REASON_CANCELLED; break; }
    if (limits && limits->max_seconds > 0 && elapsed >= limits->max_seconds) { st.reason = MGBFS2_REASON_DEADLINE; break; }
    if (limits && limits->max_layers && layer_sizes.size() >= limits->max_layers) {
      st.reason = MGBFS2_REASON_LAYER_LIMIT;
      break;
    }
    const auto layer_start = Clock::now();
    const uint64_t bound = next_bound(depth, count, visited);
    uint64_t cap = std::min<uint64_t>(std::max<uint64_t>(bound, 1), plan.capacity);
    const bool group_layer = grouped_mode && count * gens >= bucket_min_work;
    const uint64_t work = count * gens;
    const bool routed = bucketed && work >= bucket_min_work;
    if (!group_layer && front_grouped && (rc = gather_front(count))) break;
    void* group_fn = nullptr;
    size_t group_smem = 0;
    uint32_t group_grid = 1;
    uint64_t group_items = 0;
    uint64_t route_chunk = count;
    if (group_layer) {
      const uint64_t prev_count = depth ? layer_sizes[depth - 1] : 0;
      if ((rc = grouped_setup(count, prev_count, cap, &group_fn, &group_smem, smem, &group_items, &group_grid))) break;
    } else if (routed) {
      if ((rc = routed_setup(count, &cap, &route_chunk))) break;
    } else if ((rc = next.ensure((cap + 2) * 8))) {
      break;
    }
    p.frontier = static_cast<const unsigned long long*>(front.ptr);
    p.count = count;
    p.next = static_cast<unsigned long long*>(next.ptr);
    p.capacity = cap;
    p.probe_limit = 1u << 20;
    if (visit == V_HASH) {
      // Grow (rehash) so the table stays at most half full after this layer.
      const uint64_t need = visited + bound;
      if (need > table_slots / 2) {
        const uint64_t slots = next_pow2(2 * need);
        DeviceBuffer grown;
        grown.stream = stream;
        if ((rc = grown.ensure(slots * 8))) break;
        MG_CHECK(cudaMemsetAsync(grown.ptr, 0xff, slots * 8, stream));
        rehash_table<<<grid_for(reinterpret_cast<const void*>(rehash_table), 0, (table_slots + kBlock - 1) / kBlock),
                       kBlock, 0, stream>>>(static_cast<const unsigned long long*>(table.ptr), table_slots,
                                            static_cast<unsigned long long*>(grown.ptr), slots - 1, key_mask,
                                            &p.control->error);
        ++launches;
        MG_CHECK(cudaGetLastError());
        MG_CHECK(cudaStreamSynchronize(stream));
        table.free();
        table = grown;
        grown.ptr = nullptr;
        grown.bytes = 0;
        table_slots = slots;
      }
      p.table = static_cast<unsigned long long*>(table.ptr);
      p.table_mask = table_slots - 1;
      p.tag = 0;
    } else if (visit == V_HASHQ) {
      // Grow (rehash) so the table stays below its threshold after this layer.
      const uint64_t need = visited + bound;
      if (need * 100 > table_slots * hash_load) {
        const uint64_t slots = next_pow2((need * 100 + hash_load - 1) / hash_load);
        DeviceBuffer grown;
        grown.stream = stream;
        if ((rc = grown.ensure(slots * 4))) break;
        MG_CHECK(cudaMemsetAsync(grown.ptr, 0, slots * 4, stream));
        const QuotientSlots from = quotient_slots(table_slots);
        QuotientSlots to = quotient_slots(slots);
        to.slots = static_cast<unsigned int*>(grown.ptr);
        rehash_qtable<<<grid_for(reinterpret_cast<const void*>(rehash_qtable), 0, (table_slots + kBlock - 1) / kBlock),
                        kBlock, 0, stream>>>(from, to, &p.control->error);
        ++launches;
        MG_CHECK(cudaGetLastError());
        MG_CHECK(cudaStreamSynchronize(stream));
        table.free();
        table = grown;
        grown.ptr = nullptr;
        grown.bytes = 0;
        table_slots = slots;
      }
      p.q = quotient_slots(table_slots);
    } else if (visit == V_HASH3) {
      const int ins = (depth + 1) % 3, cur = depth % 3, prev = (depth + 2) % 3;
      const uint64_t slots = std::max<uint64_t>(1024, next_pow2(2 * std::max<uint64_t>(bound, 1)));
      if ((rc = bank[ins].ensure(slots * 8))) break;
      bank_slots[ins] = slots;
      MG_CHECK(cudaMemsetAsync(bank[ins].ptr, 0xff, slots * 8, stream));
      p.table = static_cast<unsigned long long*>(bank[ins].ptr);
      p.table_mask = slots - 1;
      p.look0 = static_cast<const unsigned long long*>(bank[cur].ptr);
      p.look0_mask = bank_slots[cur] - 1;
      p.look1 = depth >= 1 ? static_cast<const unsigned long long*>(bank[prev].ptr) : nullptr;
      p.look1_mask = depth >= 1 ? bank_slots[prev] - 1 : 0;
    }
    TraceRange layer_range(routed ? "layer.bucket" : group_layer ? "layer.grouped" : sorted ? "layer.sorted"
                                                                                         : "layer.fused");
    // One attempt; a routed layer whose shard buckets overflowed left the
    // bitmap untouched and is redone once with the exact shard counts.
    for (int attempt = 0; attempt < 2; ++attempt) {
      MG_CHECK(cudaMemsetAsync(control_buf.ptr, 0, sizeof(Control), stream));
      const bool chunked = routed && route_chunk < count;
      if (routed && !chunked && (rc = bucket_setup(work, attempt == 1))) break;
      MG_CHECK(cudaEventRecord(ev_kernel[0], stream));
      if (chunked) {
        if ((rc = bucket_chunks(reinterpret_cast<const void*>(route_fn), reinterpret_cast<const void*>(accept_fn), p,
                                smem, route_chunk, &st.redo_layers)))
          break;
      } else if (routed) {
        if ((rc = bucket_launch(reinterpret_cast<const void*>(route_fn), reinterpret_cast<const void*>(accept_fn), p,
                                smem)))
          break;
      } else if (group_layer) {
        const uint32_t R = groups + 1;
        unsigned long long* meta = static_cast<unsigned long long*>(group_meta.ptr);
        GroupedParams gp{};
        gp.frontier = p.frontier;
        gp.region_begin = meta;
        gp.region_count = meta + R;
        gp.item_prefix = meta + 2 * R;
        gp.region_order = reinterpret_cast<const uint32_t*>(meta + group_meta_words(groups));
        gp.regions = R;
        gp.groups = groups;
        gp.terms = p.terms;
        gp.term_begin = p.term_begin;
        gp.gens = gens;
        gp.total_terms = p.total_terms;
        gp.gen_shift = p.gen_shift;
        gp.ppt = gens <= 4 ? 4 : 2;
        gp.bitmap = p.bitmap;
        gp.next = p.next;
        gp.next_begin = meta + 3 * R + 1;
        gp.next_cap = meta + 4 * R + 1;
        gp.next_count = meta + 5 * R + 1;
        gp.work = meta + 6 * R + 1;
        gp.chunk = group_chunk;
        // Test first where most tests will find a visited state: many
        // generators, or a layer whose parents won under 40 % of their tests
        // (LRX past its peak layer).
        {
          const uint64_t tested = depth ? layer_sizes[depth - 1] * (parent_skip && depth > 1 ? gens - 1 : gens) : 0;
          const bool lean = tested && static_cast<double>(count) < 0.4 * static_cast<double>(tested);
          gp.test_first = gens >= kTestFirstGens || lean ? 1u : 0u;
        }
        gp.control = p.control;
        gp.transp = static_cast<const uint32_t*>(transp_buf.ptr);
        reinterpret_cast<GroupedFn>(group_fn)<<<group_grid, kBlock, group_smem,
                                                 stream>>>(gp);
        ++launches;
        MG_CHECK(cudaGetLastError());
      } else {
        const uint64_t per_tile = sorted ? kSortTile / gens : kBlock * p.ppt;
        const uint64_t tiles = (count + per_tile - 1) / per_tile;
        const uint32_t grid = grid_for(reinterpret_cast<const void*>(fn), smem, tiles);
        fn<<<grid, kBlock, smem, stream>>>(p);
        ++launches;
        MG_CHECK(cudaGetLastError());
      }
      MG_CHECK(cudaEventRecord(ev_kernel[1], stream));
      MG_CHECK(cudaMemcpyAsync(host_control, control_buf.ptr, sizeof(Control), cudaMemcpyDeviceToHost, stream));
      if (routed)
        MG_CHECK(cudaMemcpyAsync(host_meta + 2 * kMaxShards, static_cast<unsigned long long*>(shard_meta.ptr) + 2 * kMaxShards,
                                 bucket_shards * sizeof(unsigned long long), cudaMemcpyDeviceToHost, stream));
      if (group_layer) {
        const size_t off = 5 * static_cast<size_t>(groups + 1) + 1;
        MG_CHECK(cudaMemcpyAsync(host_group + off, static_cast<unsigned long long*>(group_meta.ptr) + off,
                                 (groups + 1) * sizeof(unsigned long long), cudaMemcpyDeviceToHost, stream));
      }
      MG_CHECK(cudaStreamSynchronize(stream));
      float ms = 0.f;
      if (cudaEventElapsedTime(&ms, ev_kernel[0], ev_kernel[1]) == cudaSuccess) kernel_seconds += ms * 1e-3;
      if (!(routed && host_control->error == ERR_BUCKET_OVERFLOW)) break;
      ++st.redo_layers;
    }
    if (rc) break;
    if (routed && !host_control->error) {
      shard_history.assign(host_meta + 2 * kMaxShards, host_meta + 2 * kMaxShards + bucket_shards);
      shard_history_total = bucket_work;
    }
    st.successors += count * gens;
    // Every tagged parent (all but the start) skips exactly one generator.
    st.visited_tests += count * gens - (parent_skip && depth > 0 ? count : 0);
    const Control c = *host_control;
    peak = std::max<uint64_t>(peak, bitmap.bytes + front.bytes + next.bytes + table.bytes + bank[0].bytes +
                                        bank[1].bytes + bank[2].bytes);
    if (c.error) {
      st.reason = MGBFS2_REASON_RESOURCE;
      st.fatal = c.error;
      break;
    }
    if (c.next_count == 0) {
      st.complete = 1;
      break;
    }
    if (c.next_count > cap) {
      st.reason = MGBFS2_REASON_RESOURCE;
      st.fatal = ERR_FRONTIER_OVERFLOW;
      break;
    }
    const double secs = std::chrono::duration<double>(Clock::now() - layer_start).count();
    layer_sizes.push_back(c.next_count);
    layer_seconds.push_back(secs);
    if (group_layer) grouped_finish();
    std::swap(front, next);
    front_grouped = group_layer;
    count = c.next_count;
    visited += count;
    ++depth;
    if (count < 1000) {
      if (front_grouped && (rc = gather_front(count))) break;
      std::vector<uint64_t> words(count);
      MG_CHECK(cudaMemcpyAsync(words.data(), front.ptr, count * 8, cudaMemcpyDeviceToHost, stream));
      MG_CHECK(cudaStreamSynchronize(stream));
      keep_small(depth, std::move(words));
    }
    if (cb && cb(user, depth, count, secs)) {
      st.reason = MGBFS2_REASON_CANCELLED;
      break;
    }
  }
  if (!rc && front_grouped) rc = gather_front(count);  // samples read `front` as one array
  last_count = count;
  st.layers = static_cast<uint32_t>(layer_sizes.size());
  for (uint64_t s : layer_sizes) st.states += s;
  if (cudaEventRecord(ev_run[1], stream) == cudaSuccess && cudaEventSynchronize(ev_run[1]) == cudaSuccess) {
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, ev_run[0], ev_run[1]) == cudaSuccess) st.device_seconds = ms * 1e-3;
  }
  st.kernel_seconds = kernel_seconds;
  st.bfs_seconds = std::chrono::duration<double>(Clock::now() - started).count();
  st.kernel_launches = launches;
  st.peak_device_bytes = peak;
  if (status) *status = st;
  return rc;
}

// Small layers are copied to the host as they complete so that the
// "previous_small" sample survives the frontier buffers being reused.
void Graph::keep_small(uint32_t depth, std::vector<uint64_t>&& words) {
  small_layer[1] = std::move(small_layer[0]);
  small_depth[1] = small_depth[0];
  small_layer[0] = std::move(words);
  small_depth[0] = depth;
}

std::vector<int64_t> Graph::decode(uint64_t w) const {
  std::vector<int64_t> row(elements);
  const uint64_t mask = bits == 64 ? ~0ull : ((1ull << bits) - 1);
  for (uint32_t i = 0; i < elements; ++i) {
    const uint64_t f = (w >> (bits * i)) & mask;
    row[i] = packed_matrix ? static_cast<int64_t>(f) : labels[f];
  }
  return row;
}

int Graph::sample(uint32_t which, int64_t* out, size_t cap_rows, size_t* rows) {
  if (!rows) return MGBFS2_INVALID_ARGUMENT;
  *rows = 0;
  if (layer_sizes.empty()) return MGBFS2_STATE;
  if (!packed) return wide_sample(which, out, cap_rows, rows);
  const uint32_t deepest = static_cast<uint32_t>(layer_sizes.size() - 1);
  std::vector<uint64_t> words;
  if (which == 0) {
    const uint64_t n = std::min<uint64_t>(last_count, cap_rows);
    words.resize(n);
    if (n) {
      MG_CHECK(cudaMemcpyAsync(words.data(), front.ptr, n * 8, cudaMemcpyDeviceToHost, stream));
      MG_CHECK(cudaStreamSynchronize(stream));
    }
  } else {
    if (deepest == 0 || layer_sizes[deepest - 1] >= 1000) return MGBFS2_OK;
    const int k = small_depth[0] == deepest - 1 ? 0 : (small_depth[1] == deepest - 1 ? 1 : -1);
    if (k < 0) return MGBFS2_OK;
    words.assign(small_layer[k].begin(), small_layer[k].begin() + std::min<size_t>(small_layer[k].size(), cap_rows));
  }
  std::vector<std::vector<int64_t>> decoded;
  for (uint64_t w : words) decoded.push_back(decode(w));
  std::sort(decoded.begin(), decoded.end());
  for (size_t i = 0; i < decoded.size(); ++i)
    if (out) std::memcpy(out + i * elements, decoded[i].data(), elements * sizeof(int64_t));
  *rows = decoded.size();
  return MGBFS2_OK;
}

// Probes of the keys of an all-visited table: for every stored key, the
// slots an insert or a successful lookup of it reads (its distance from its
// home slot, plus one).  sums[0] += keys, sums[1] += probes.
static __global__ void table_probes_kernel(const void* table, unsigned long long slots, int quotient,
                                           uint32_t distance_bits, unsigned long long key_mask,
                                           unsigned long long* sums) {
  unsigned long long keys = 0, probes = 0;
  const unsigned int dmask = distance_bits >= 32 ? ~0u : ((1u << distance_bits) - 1u);
  for (unsigned long long t = blockIdx.x * static_cast<unsigned long long>(blockDim.x) + threadIdx.x; t < slots;
       t += static_cast<unsigned long long>(gridDim.x) * blockDim.x) {
    if (quotient) {
      const unsigned int v = static_cast<const unsigned int*>(table)[t];
      if (v) {
        ++keys;
        probes += v & dmask;  // the stored distance is probes - 1, kept as probes
      }
    } else {
      const unsigned long long v = static_cast<const unsigned long long*>(table)[t];
      if (v != kEmpty) {
        const unsigned long long home = mix64(v & key_mask) & (slots - 1);
        ++keys;
        probes += ((t - home) & (slots - 1)) + 1;
      }
    }
  }
  for (int o = 16; o; o >>= 1) {
    keys += __shfl_down_sync(kFullMask, keys, o);
    probes += __shfl_down_sync(kFullMask, probes, o);
  }
  if ((threadIdx.x & 31) == 0 && keys) {
    atomicAdd(&sums[0], keys);
    atomicAdd(&sums[1], probes);
  }
}

int Graph::table_probe_mean(double* mean, uint64_t* keys) {
  if (!planned || !packed) return MGBFS2_STATE;
  const int visit = visit_kind();
  if (visit != V_HASH && visit != V_HASHQ) return MGBFS2_UNSUPPORTED;
  if (!table.ptr || !table_slots) return MGBFS2_STATE;
  MG_CHECK(cudaSetDevice(device));
  int rc = scratch.ensure(2 * sizeof(unsigned long long));
  if (rc) return rc;
  MG_CHECK(cudaMemsetAsync(scratch.ptr, 0, 2 * sizeof(unsigned long long), stream));
  const uint32_t d = visit == V_HASHQ ? quotient_slots(table_slots).d : 0;
  const uint64_t work = (table_slots + kBlock - 1) / kBlock;
  table_probes_kernel<<<static_cast<uint32_t>(std::min<uint64_t>(work, 8ull * sm_count)), kBlock, 0, stream>>>(
      table.ptr, table_slots, visit == V_HASHQ, d, key_mask, static_cast<unsigned long long*>(scratch.ptr));
  MG_CHECK(cudaGetLastError());
  unsigned long long sums[2] = {0, 0};
  MG_CHECK(cudaMemcpyAsync(sums, scratch.ptr, sizeof(sums), cudaMemcpyDeviceToHost, stream));
  MG_CHECK(cudaStreamSynchronize(stream));
  if (keys) *keys = sums[0];
  if (mean) *mean = sums[0] ? static_cast<double>(sums[1]) / static_cast<double>(sums[0]) : 0.0;
  return MGBFS2_OK;
}

}  // namespace mgbfs2

// ---------------------------------------------------------------------------
// C ABI.

using mgbfs2::Graph;

extern "C" {

int mgbfs2_graph_create(const mgbfs2_graph_desc* desc, int device, mgbfs2_graph** out, char* error,
                        size_t error_capacity) {
  if (!out) return MGBFS2_INVALID_ARGUMENT;
  *out = nullptr;
  Graph* g = nullptr;
  int rc = Graph::create(desc, device, &g, error, error_capacity);
  if (rc) return rc;
  *out = new mgbfs2_graph{g};
  return MGBFS2_OK;
}

int mgbfs2_plan(mgbfs2_graph* graph, const mgbfs2_plan_request* request, mgbfs2_plan_info* plan) {
  if (!graph) return MGBFS2_INVALID_ARGUMENT;
  return graph->impl->make_plan(request, plan);
}

int mgbfs2_run(mgbfs2_graph* graph, const mgbfs2_run_limits* limits, mgbfs2_layer_callback callback, void* user,
               mgbfs2_status* status) {
  if (!graph) return MGBFS2_INVALID_ARGUMENT;
  return graph->impl->run(limits, callback, user, status);
}

int mgbfs2_layer_table(const mgbfs2_graph* graph, uint64_t* sizes, double* seconds, size_t capacity,
                       size_t* count) {
  if (!graph || !count) return MGBFS2_INVALID_ARGUMENT;
  const Graph* g = graph->impl;
  *count = g->layer_sizes.size();
  for (size_t i = 0; i < g->layer_sizes.size() && i < capacity; ++i) {
    if (sizes) sizes[i] = g->layer_sizes[i];
    if (seconds) seconds[i] = i == 0 ? 0.0 : g->layer_seconds[i - 1];
  }
  return MGBFS2_OK;
}

int mgbfs2_sample(mgbfs2_graph* graph, uint32_t which, int64_t* out, size_t capacity_rows, size_t* rows) {
  if (!graph || which > 1) return MGBFS2_INVALID_ARGUMENT;
  return graph->impl->sample(which, out, capacity_rows, rows);
}

const char* mgbfs2_status_string(int code) {
  switch (code) {
    case MGBFS2_OK: return "OK";
    case MGBFS2_INVALID_ARGUMENT: return "INVALID_ARGUMENT";
    case MGBFS2_UNSUPPORTED: return "UNSUPPORTED";
    case MGBFS2_OUT_OF_MEMORY: return "OUT_OF_MEMORY";
    case MGBFS2_CAPACITY: return "CAPACITY";
    case MGBFS2_DEVICE_STATUS: return "DEVICE_STATUS";
    case MGBFS2_STATE: return "STATE";
    case MGBFS2_NOT_FOUND: return "NOT_FOUND";
    default:
      if (code >= MGBFS2_CUDA_BASE) return cudaGetErrorString(static_cast<cudaError_t>(code - MGBFS2_CUDA_BASE));
      return "UNKNOWN";
  }
}

void mgbfs2_destroy(mgbfs2_graph* graph) {
  if (!graph) return;
  delete graph->impl;
  delete graph;
}

int mgbfs2_trim_memory(int device) { return mgbfs2::device_cache_release(device); }

int mgbfs2_table_probes(mgbfs2_graph* graph, double* mean_probes, uint64_t* keys) {
  if (!graph) return MGBFS2_INVALID_ARGUMENT;
  return graph->impl->table_probe_mean(mean_probes, keys);
}

void mgbfs2_trace_range_push(const char* label) { nvtxRangePushA(label ? label : "mgbfs2"); }

void mgbfs2_trace_range_pop(void) { nvtxRangePop(); }

}  // extern "C"
