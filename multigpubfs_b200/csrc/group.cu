// Order of a permutation group given by generators: deterministic
// Schreier-Sims (Sims 1970; the textbook form of Holt, Eick, O'Brien,
// "Handbook of Computational Group Theory", 2005, section 4.4.2).  Host code.
//
// For a permutation graph with distinct labels, the states reachable from the
// start are exactly start o G for the generated group G, so |G| is the exact
// number of states the BFS settles (for directed graphs too: in a finite group
// every inverse is a positive power).  The learned planner uses it as its
// orbit size; the reference only bounds the state space by the multinomial
// n!/prod(c!) (crates/mgbfs-runtime/src/generic_memory.rs:82-108).
#include <algorithm>
#include <array>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <numeric>
#include <thread>
#include <vector>

#include "../../include/mgbfs2.h"

namespace mgbfs2 {
namespace {

constexpr uint32_t kMaxPoints = 20;
// p[i] = image of point i for i < n; entries from n on stay fixed (p[i] = i),
// so every helper can work on all kMaxPoints entries without knowing n.
using Perm = std::array<uint8_t, kMaxPoints>;

Perm identity() {
  Perm r;
  for (uint32_t i = 0; i < kMaxPoints; ++i) r[i] = static_cast<uint8_t>(i);
  return r;
}

Perm compose(const Perm& a, const Perm& b) {  // (a b)(i) = a(b(i))
  Perm r;
  for (uint32_t i = 0; i < kMaxPoints; ++i) r[i] = a[b[i]];
  return r;
}

Perm inverse(const Perm& a) {
  Perm r;
  for (uint32_t i = 0; i < kMaxPoints; ++i) r[a[i]] = static_cast<uint8_t>(i);
  return r;
}

bool is_identity(const Perm& a) {
  for (uint32_t i = 0; i < kMaxPoints; ++i)
    if (a[i] != i) return false;
  return true;
}

uint32_t moved_point(const Perm& a) {
  for (uint32_t i = 0; i < kMaxPoints; ++i)
    if (a[i] != i) return i;
  return 0;
}

// Jordan's theorem (Wielandt, "Finite Permutation Groups", 1964, Theorem
// 13.9): a primitive group of degree n that contains a cycle of prime length
// p <= n - 3 contains the alternating group A_n.  True only when all three
// are shown: transitivity, primitivity (the smallest block system joining 0
// and x is the trivial one, for every x; Atkinson's closure), and a walk
// element with exactly one cycle of length divisible by a prime p <= n - 3,
// of length exactly p (a power of it is then a p-cycle).  False means
// "not shown", never "not A_n".
bool contains_alternating(const std::vector<Perm>& gens, uint32_t n) {
  if (n < 5 || gens.empty()) return false;
  std::array<uint8_t, kMaxPoints> parent{};
  auto find = [&](uint32_t x) {
    while (parent[x] != x) x = parent[x] = parent[parent[x]];
    return x;
  };
  auto reset = [&]() {
    for (uint32_t i = 0; i < n; ++i) parent[i] = static_cast<uint8_t>(i);
  };
  auto unite = [&](uint32_t a, uint32_t b) {
    a = find(a);
    b = find(b);
    if (a == b) return false;
    parent[b] = static_cast<uint8_t>(a);
    return true;
  };
  auto one_class = [&]() {
    const uint32_t r = find(0);
    for (uint32_t i = 1; i < n; ++i)
      if (find(i) != r) return false;
    return true;
  };
  reset();
  for (const Perm& g : gens)
    for (uint32_t x = 0; x < n; ++x) unite(x, g[x]);
  if (!one_class()) return false;
  std::vector<std::pair<uint8_t, uint8_t>> todo;
  for (uint32_t x = 1; x < n; ++x) {
    reset();
    todo.clear();
    unite(0, x);
    todo.emplace_back(0, x);
    while (!todo.empty()) {
      const auto [a, b] = todo.back();
      todo.pop_back();
      for (const Perm& g : gens)
        if (unite(g[a], g[b])) todo.emplace_back(g[a], g[b]);
    }
    if (!one_class()) return false;  // {0, x} lies in a proper block
  }
  static constexpr uint32_t kPrimes[] = {2, 3, 5, 7, 11, 13, 17};
  Perm walk = identity();
  uint64_t state = 0x2545f4914f6cdd1dull;
  for (uint32_t step = 0; step < 32 * n; ++step) {
    state ^= state << 13;
    state ^= state >> 7;
    state ^= state << 17;
    walk = compose(walk, gens[state % gens.size()]);
    std::array<uint8_t, kMaxPoints> seen{};
    std::array<uint8_t, kMaxPoints> lengths{};
    uint32_t cycles = 0;
    for (uint32_t x = 0; x < n; ++x) {
      if (seen[x]) continue;
      uint32_t length = 0;
      for (uint32_t y = x; !seen[y]; y = walk[y]) {
        seen[y] = 1;
        ++length;
      }
      lengths[cycles++] = static_cast<uint8_t>(length);
    }
    for (uint32_t p : kPrimes) {
      if (p + 3 > n) break;
      uint32_t divisible = 0, exact = 0;
      for (uint32_t c = 0; c < cycles; ++c) {
        divisible += lengths[c] % p == 0;
        exact += lengths[c] == p;
      }
      if (divisible == 1 && exact == 1) return true;
    }
  }
  return false;
}

struct StabChain {
  uint32_t n;
  std::vector<uint32_t> base;
  std::vector<Perm> strong;
  // Per level: transversal u[point] (maps base[level] to point), present[point].
  std::vector<std::vector<Perm>> u;
  std::vector<std::vector<uint8_t>> present;
  std::vector<uint8_t> fresh;

  bool fixes_prefix(const Perm& s, size_t level) const {
    for (size_t k = 0; k < level; ++k)
      if (s[base[k]] != base[k]) return false;
    return true;
  }
  std::vector<const Perm*> level_gens(size_t level) const {
    std::vector<const Perm*> out;
    for (const Perm& s : strong)
      if (fixes_prefix(s, level)) out.push_back(&s);
    return out;
  }
  void add_level(uint32_t point) {
    base.push_back(point);
    u.emplace_back();
    present.emplace_back();
    fresh.push_back(0);
  }
  // Orbit of base[level] under the level's generators, with transversal.
  void build(size_t level) {
    const auto gens = level_gens(level);
    u[level].assign(n, Perm{});
    present[level].assign(n, 0);
    const uint32_t beta = base[level];
    u[level][beta] = identity();
    present[level][beta] = 1;
    std::vector<uint32_t> queue{beta};
    for (size_t q = 0; q < queue.size(); ++q) {
      const uint32_t x = queue[q];
      for (const Perm* s : gens) {
        const uint32_t y = (*s)[x];
        if (!present[level][y]) {
          present[level][y] = 1;
          u[level][y] = compose(*s, u[level][x]);
          queue.push_back(y);
        }
      }
    }
    fresh[level] = 1;
  }
  // Strips h through levels start..; returns the residue and the level where
  // it stopped (base.size() when it passed every level).
  size_t sift(Perm& h, size_t start) {
    for (size_t j = start; j < base.size(); ++j) {
      if (!fresh[j]) build(j);
      const uint32_t y = h[base[j]];
      if (!present[j][y]) return j;
      h = compose(inverse(u[j][y]), h);
    }
    return base.size();
  }
};

int group_order(const uint32_t* permutations, uint32_t n, uint32_t generators, uint64_t* order) {
  if (!order || n == 0 || n > 20 || (generators && !permutations)) return MGBFS2_INVALID_ARGUMENT;
  StabChain c;
  c.n = n;
  for (uint32_t g = 0; g < generators; ++g) {
    Perm p = identity();
    std::vector<uint8_t> seen(n, 0);
    for (uint32_t i = 0; i < n; ++i) {
      const uint32_t v = permutations[static_cast<size_t>(g) * n + i];
      if (v >= n || seen[v]) return MGBFS2_INVALID_ARGUMENT;
      seen[v] = 1;
      p[i] = static_cast<uint8_t>(v);
    }
    if (!is_identity(p)) c.strong.push_back(p);
  }
  if (c.strong.empty()) {
    *order = 1;
    return MGBFS2_OK;
  }
  // G fixes every point outside the support of its generators and acts
  // faithfully on the support, so the test runs on the support relabelled
  // 0..m-1 (m! / 2 or m! when it contains A_m).
  std::array<uint8_t, kMaxPoints> label{};
  uint32_t m = 0;
  for (uint32_t x = 0; x < n; ++x) {
    bool moved = false;
    for (const Perm& g : c.strong) moved = moved || g[x] != x;
    label[x] = moved ? static_cast<uint8_t>(m++) : 0xff;
  }
  std::vector<Perm> support;
  for (const Perm& g : c.strong) {
    Perm r = identity();
    for (uint32_t x = 0; x < n; ++x)
      if (label[x] != 0xff) r[label[x]] = label[g[x]];
    support.push_back(r);
  }
  if (contains_alternating(support, m)) {
    // A_m <= G: G is S_m when some generator is odd, else A_m.
    uint64_t full = 1;
    for (uint32_t k = 2; k <= m; ++k) full *= k;
    bool odd = false;
    for (const Perm& g : c.strong) {
      std::array<uint8_t, kMaxPoints> seen{};
      uint32_t cycles = 0;
      for (uint32_t x = 0; x < n; ++x) {
        if (seen[x]) continue;
        ++cycles;
        for (uint32_t y = x; !seen[y]; y = g[y]) seen[y] = 1;
      }
      odd = odd || ((n - cycles) & 1u);
    }
    *order = odd ? full : full / 2;
    return MGBFS2_OK;
  }
  for (const Perm& s : c.strong)
    if (c.fixes_prefix(s, c.base.size())) c.add_level(moved_point(s));
  // Fast exact exit.  The product of the orbit lengths of any partial chain
  // built from group elements is a lower bound on |G|; n! (n!/2 when every
  // generator is even) is an upper bound.  Sifting a random walk over the
  // generators into the chain usually lifts the lower bound to the upper one
  // within a few dozen steps when G is the symmetric or alternating group (as
  // for random generators); equality proves the order.  Otherwise the
  // deterministic completion below finishes the chain.
  {
    uint64_t upper = 1;
    for (uint32_t k = 2; k <= n; ++k) upper *= k;
    bool all_even = true;
    for (const Perm& s : c.strong) {
      uint32_t cycles = 0;
      std::array<uint8_t, kMaxPoints> seen{};
      for (uint32_t x = 0; x < n; ++x) {
        if (seen[x]) continue;
        ++cycles;
        for (uint32_t y = x; !seen[y]; y = s[y]) seen[y] = 1;
      }
      if ((n - cycles) & 1u) all_even = false;
    }
    if (all_even) upper /= 2;
    const size_t gens0 = c.strong.size();
    Perm walk = identity();
    uint64_t state = 0x9e3779b97f4a7c15ull;
    for (uint32_t step = 0; step < 64 * n; ++step) {
      state ^= state << 13;
      state ^= state >> 7;
      state ^= state << 17;
      walk = compose(walk, c.strong[state % gens0]);
      Perm h = walk;
      const size_t j = c.sift(h, 0);
      if (is_identity(h)) continue;
      c.strong.push_back(h);
      if (j == c.base.size()) c.add_level(moved_point(h));
      for (size_t l = 0; l <= j && l < c.base.size(); ++l) c.fresh[l] = 0;
      uint64_t lower = 1;
      for (size_t l = 0; l < c.base.size(); ++l) {
        if (!c.fresh[l]) c.build(l);
        uint64_t orbit = 0;
        for (uint32_t q = 0; q < n; ++q) orbit += c.present[l][q];
        lower *= orbit;
      }
      if (lower == upper) {
        *order = upper;
        return MGBFS2_OK;
      }
    }
  }
  // Level i is complete when every Schreier generator of its orbit sifts to
  // the identity through the levels below it.
  long i = static_cast<long>(c.base.size()) - 1;
  while (i >= 0) {
    c.build(static_cast<size_t>(i));
    bool extended = false;
    const auto gens = c.level_gens(static_cast<size_t>(i));
    for (uint32_t gamma = 0; gamma < n && !extended; ++gamma) {
      if (!c.present[i][gamma]) continue;
      for (const Perm* s : gens) {
        Perm h = compose(inverse(c.u[i][(*s)[gamma]]), compose(*s, c.u[i][gamma]));
        if (is_identity(h)) continue;
        const size_t j = c.sift(h, static_cast<size_t>(i) + 1);
        if (is_identity(h)) continue;
        // New strong generator: it fixes base[0..j-1] and extends level j.
        c.strong.push_back(h);
        if (j == c.base.size()) c.add_level(moved_point(h));
        for (size_t l = static_cast<size_t>(i) + 1; l <= j; ++l) c.fresh[l] = 0;
        i = static_cast<long>(j);
        extended = true;
        break;
      }
    }
    if (!extended) --i;
  }
  uint64_t total = 1;
  for (size_t l = 0; l < c.base.size(); ++l) {
    if (!c.fresh[l]) c.build(l);
    uint64_t orbit = 0;
    for (uint32_t p = 0; p < n; ++p) orbit += c.present[l][p];
    total *= orbit;
  }
  *order = total;
  return MGBFS2_OK;
}

// One graph's planner features (the layout of mgbfs2_mlp_rollout_bf16's
// statics) and its settled-state count; the same arithmetic as the Python
// planner's graph_statics.
int graph_statics(const uint32_t* perms, uint32_t n, uint32_t k, const uint32_t* labels, float* out, uint64_t* states) {
  if (n == 0 || n > 20 || k == 0) return MGBFS2_INVALID_ARGUMENT;
  double sum_log = 0.0, max_log = 0.0, fixed = 0.0, cycles = 0.0;
  bool closed = true;
  for (uint32_t g = 0; g < k; ++g) {
    const uint32_t* p = perms + static_cast<size_t>(g) * n;
    std::array<uint8_t, kMaxPoints> seen{};
    uint64_t order = 1;
    uint32_t fixed_points = 0, count = 0;
    for (uint32_t x = 0; x < n; ++x) {
      if (p[x] >= n) return MGBFS2_INVALID_ARGUMENT;
      if (seen[x]) continue;
      uint64_t length = 0;
      for (uint32_t y = x; !seen[y]; y = p[y]) {
        seen[y] = 1;
        ++length;
      }
      ++count;
      fixed_points += length == 1;
      order = order / std::gcd(order, length) * length;
    }
    const double lo = std::log(static_cast<double>(order));
    sum_log += lo;
    max_log = g ? std::max(max_log, lo) : lo;
    fixed += static_cast<double>(fixed_points) / n;
    cycles += static_cast<double>(count) / n;
    // Inverse closure: g^-1 is one of the generators.
    std::array<uint32_t, kMaxPoints> inv{};
    for (uint32_t x = 0; x < n; ++x) inv[p[x]] = x;
    bool found = false;
    for (uint32_t h = 0; h < k && !found; ++h)
      found = std::equal(inv.begin(), inv.begin() + n, perms + static_cast<size_t>(h) * n);
    closed = closed && found;
  }
  // Distinct labels: the BFS settles |G| states; repeated labels: the
  // multinomial bound n! / prod(c!).
  std::array<uint32_t, 256> mult{};
  bool distinct = true;
  for (uint32_t i = 0; i < n; ++i) {
    if (labels[i] > 255) return MGBFS2_INVALID_ARGUMENT;
    distinct = distinct && mult[labels[i]] == 0;
    ++mult[labels[i]];
  }
  double log_orbit;
  if (distinct) {
    uint64_t order = 0;
    if (const int rc = group_order(perms, n, k, &order)) return rc;
    *states = order;
    log_orbit = std::log(static_cast<double>(order));
  } else {
    log_orbit = std::lgamma(n + 1.0);
    double bound = 1.0;
    for (uint32_t i = 2; i <= n; ++i) bound *= i;
    for (uint32_t c : mult) {
      if (c < 2) continue;
      log_orbit -= std::lgamma(c + 1.0);
      for (uint32_t i = 2; i <= c; ++i) bound /= i;
    }
    *states = static_cast<uint64_t>(bound + 0.5);
  }
  out[0] = static_cast<float>(log_orbit);
  out[1] = static_cast<float>(n / 16.0);
  out[2] = static_cast<float>(k / 8.0);
  out[3] = closed ? 1.0f : 0.0f;
  out[4] = static_cast<float>(sum_log / k);
  out[5] = static_cast<float>(max_log);
  out[6] = static_cast<float>(fixed / k);
  out[7] = static_cast<float>(cycles / k);
  return MGBFS2_OK;
}

}  // namespace
}  // namespace mgbfs2

extern "C" int mgbfs2_group_order(const uint32_t* permutations, uint32_t n, uint32_t generators, uint64_t* order) {
  return mgbfs2::group_order(permutations, n, generators, order);
}

extern "C" int mgbfs2_graph_statics(uint32_t count, const uint32_t* degree, const uint32_t* generators,
                                    const uint32_t* permutations, const uint32_t* labels, uint32_t threads,
                                    float* statics, uint64_t* states) {
  using namespace mgbfs2;
  if (count == 0) return MGBFS2_OK;
  if (!degree || !generators || !permutations || !labels || !statics || !states) return MGBFS2_INVALID_ARGUMENT;
  std::vector<size_t> perm_at(count), label_at(count);
  size_t pa = 0, la = 0;
  for (uint32_t i = 0; i < count; ++i) {
    perm_at[i] = pa;
    label_at[i] = la;
    pa += static_cast<size_t>(degree[i]) * generators[i];
    la += degree[i];
  }
  if (threads == 0) threads = std::max(1u, std::thread::hardware_concurrency());
  threads = std::min(threads, count);
  std::atomic<int> status{MGBFS2_OK};
  std::atomic<uint32_t> next{0};
  auto work = [&]() {
    for (uint32_t i; (i = next.fetch_add(1)) < count;) {
      const int rc = graph_statics(permutations + perm_at[i], degree[i], generators[i], labels + label_at[i],
                                   statics + 8 * static_cast<size_t>(i), states + i);
      if (rc) status.store(rc);
    }
  };
  std::vector<std::thread> pool;
  for (uint32_t t = 1; t < threads; ++t) pool.emplace_back(work);
  work();
  for (auto& t : pool) t.join();
  return status.load();
}
