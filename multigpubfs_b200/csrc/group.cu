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
#include <array>
#include <cstdint>
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

}  // namespace
}  // namespace mgbfs2

extern "C" int mgbfs2_group_order(const uint32_t* permutations, uint32_t n, uint32_t generators, uint64_t* order) {
  using namespace mgbfs2;
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
