"""Pins the CPU oracle (oracle/) to the reference's own outputs.

Golden vectors were produced by running the reference's Python code
(tests/golden/make_golden.py): GraphDefinition.exact_layers / successor /
inverse_closed, the packed LRX search scripts/cpu_small_bfs.py:exact_search,
the Coxeter certificate workload_geometry.py, and the shipped
data/reference/lrx13-layers.json table.  No GPU is used here.
"""
import itertools
import math
import os

import pytest

from oracle import graph_oracle as G
from oracle import packed_oracle as P


def test_lrx13_table_is_full_thirteen_factorial(lrx13):
    # tests/test_lrx_layers.py:44-48 of the reference
    assert sum(lrx13) == 6227020800
    assert len(lrx13) == 79
    assert max(lrx13) == 369741101


@pytest.mark.parametrize("n", range(3, 12))
def test_c_oracle_lrx_matches_reference_packed_search(n, lrx_layers):
    sizes, _, _ = P.packed_bfs(G.lrx_generators(n), list(range(n)), use_bitmap=True)
    assert sizes == lrx_layers[n]
    sizes_hash, _, _ = P.packed_bfs(G.lrx_generators(n), list(range(n)), use_bitmap=False)
    assert sizes_hash == lrx_layers[n]


def test_c_oracle_s14_prefix_matches_the_reference_search():
    """The first 24 layers of S14 LRX: the oracle's partial search against
    the reference's CPU search cancelled at the same depth."""
    from tests.conftest import golden
    fx = golden("lrx14_prefix.json")
    sizes, _, _ = P.packed_bfs(G.lrx_generators(14), list(range(14)), use_bitmap=False, max_layers=24,
                               partial=True, max_states=1 << 27)
    assert sizes == fx["layers"] and fx["states"] == math.factorial(14)


def test_c_oracle_s13_full_table(lrx13):
    # The whole 13! search takes ~10 minutes on 8 cores, so it runs only on
    # request; the GPU suite checks the engine against the same table.
    if not os.environ.get("MGBFS2_ORACLE_S13"):
        pytest.skip("set MGBFS2_ORACLE_S13=1 to run the 13! oracle search")
    sizes, _, _ = P.packed_bfs(G.lrx_generators(13), list(range(13)), use_bitmap=True)
    assert sizes == lrx13


def test_python_oracle_matches_reference_exact_layers(exact_cases):
    for case in exact_cases:
        g = case["graph"]
        if sum(case["layer_sizes"]) > 50000:
            continue
        layers = G.exact_layers(g, 1 << 24)
        assert [len(x) for x in layers] == case["layer_sizes"], case["name"]
        if case["last_layer"] is not None:
            assert layers[-1] == case["last_layer"], case["name"]
        if case["previous_layer"] is not None:
            assert layers[-2] == case["previous_layer"], case["name"]
        assert G.inverse_closed(g) == case["inverse_closed"], case["name"]
        for kat in case["successors"]:
            assert G.successor(g, kat["state"], kat["generator"]) == kat["child"], case["name"]


def test_c_oracle_matches_reference_on_permutation_cases(exact_cases):
    checked = 0
    for case in exact_cases:
        g = case["graph"]
        a = g["action"]
        if a["kind"] != "permutation":
            continue
        start = g["start"]
        distinct = len(set(start))
        bits = P.bits_for(distinct)
        if len(start) * bits > 64:
            continue
        sample = 2000
        sizes, last, prev = P.packed_bfs(a["generators"], start, use_bitmap=False,
                                         max_states=max(16, sum(case["layer_sizes"])), sample=sample)
        assert sizes == case["layer_sizes"], case["name"]
        if case["last_layer"] is not None:
            assert last == case["last_layer"], case["name"]
        if case["previous_layer"] is not None:
            assert prev == case["previous_layer"], case["name"]
        checked += 1
    assert checked >= 30


def test_wrap_known_answers():
    from tests.conftest import golden
    kat = golden("wrap_kat.json")
    g = G.matrix_graph(1, 1, [([2], 7)], [(1 << 63) - 1])
    assert G.successor(g, g["start"], 0) == kat["wrap_mod7"] == [5]
    h = G.matrix_graph(1, 1, [([2], 0)], [(1 << 63) - 1])
    assert G.successor(h, h["start"], 0) == kat["wrap_nomod"] == [-2]
    o = G.matrix_graph(1, 1, [([(1 << 63) - 1], 3)], [2])
    assert G.inverse_closed(o) == kat["overflow_guard_inverse_closed"] is False


def test_coxeter_layers_match_reference_certificate(coxeter_bounds):
    for n, b in coxeter_bounds.items():
        sizes = G.coxeter_layers(n)
        assert sum(sizes) == b["order"] == math.factorial(n)
        assert len(sizes) - 1 == b["depth"]
        assert max(sizes) == b["maximum_frontier"]
        assert max(sum(sizes[max(0, j - 2):j + 1]) for j in range(len(sizes))) == b["maximum_live_states"]


@pytest.mark.parametrize("n", range(2, 10))
def test_c_oracle_coxeter_matches_certificate(n):
    sizes, _, _ = P.packed_bfs(G.coxeter_generators(n), list(range(n)), use_bitmap=True)
    assert sizes == G.coxeter_layers(n)


def test_multiset_rank_is_lexicographic_index():
    # Restates tests/permutation_bitmap_gpu.cu: exhaustive next_permutation
    # order gives rank = position, for distinct and repeated labels.
    for start in ([0, 1, 2, 3], [-7, -7, 0, 99, 99], [1, 1, 2, 3, 3], [2, 0, 1], [5, 5, 5, 1]):
        ordered = sorted(set(itertools.permutations(sorted(start))))
        _, _, total = G.multiset_domain(start)
        assert len(ordered) == total
        for index, state in enumerate(ordered):
            assert G.multiset_rank(start, list(state)) == index
            assert G.multiset_unrank(start, index) == list(state)


def _unrank_unique(n, r):
    # Factorial-base unrank of distinct labels 0..n-1 (the reference test's
    # independent construction of states with known ranks).
    values = list(range(n))
    out = []
    for remain in range(n, 0, -1):
        f = math.factorial(remain - 1)
        j, r = divmod(r, f)
        out.append(values.pop(j))
    return out


@pytest.mark.parametrize("n", [13, 16, 20])
def test_large_distinct_ranks(n):
    total = math.factorial(n)
    for r in [0, 1, 4294967313, total // 2, total - 1]:
        state = _unrank_unique(n, r)
        assert G.multiset_rank(list(range(n)), state) == r
        if n <= 16:
            word = sum(s << (4 * i) for i, s in enumerate(state))
            assert P.lehmer_ranks([word], n)[0] == r


def test_domain_sizes():
    # permutation_bitmap.rs:204-293 domain sizes (full-multiset domains)
    assert G.multiset_domain([1, 1, 2, 3, 3])[2] == 30
    assert G.multiset_domain(list(range(10)))[2] == 3628800


# ---------------------------------------------------------------------------
# Position-component product domains: the reference's own known sizes
# (crates/mgbfs-runtime/src/permutation_bitmap.rs:263-293) and rank bijections.

PRODUCT_CASES = [
    ([-7, 8, 10, 12, 90, 91], [[1, 0, 3, 2, 4, 5]], 4),
    ([1, 1, 2, 3, 3], [[2, 1, 0, 4, 3], [1, 0, 2, 3, 4]], 3),
    ([2, 0, 1], [[1, 0, 2], [0, 2, 1]], 6),
]


def test_product_domain_sizes_match_reference():
    for start, gens, size in PRODUCT_CASES:
        assert G.product_domain(start, gens)[1] == size
        for r in range(size):
            assert G.product_rank(start, gens, G.product_unrank(start, gens, r)) == r
    # S10 acting on 10 of 14 points: the four fixed points shrink the domain to 10!.
    start = list(range(14))
    gens = []
    for i in range(9):
        g = list(range(14))
        g[i], g[i + 1] = g[i + 1], g[i]
        gens.append(g)
    comps, size = G.product_domain(start, gens)
    assert size == 3628800 and len(comps) == 5
    for r in (0, 1, 1024, size - 1):
        s = G.product_unrank(start, gens, r)
        assert s[10:] == start[10:] and G.product_rank(start, gens, s) == r
    bad = list(start)
    bad[0], bad[13] = bad[13], bad[0]
    with pytest.raises(ValueError):
        G.product_rank(start, gens, bad)
    with pytest.raises(ValueError):
        G.position_components(3, [[0, 0, 1]])


def test_matrix_oracle_matches_the_reference_sl2_table():
    from tests.conftest import golden
    fx = golden("matrix_groups.json")["cases"]["sl2_mod31"]
    assert G.layer_sizes(fx["graph"]) == fx["layers"]
    assert sum(fx["layers"]) == 31 * (31 * 31 - 1)


@pytest.mark.parametrize("p", [5, 7, 11])
def test_gl2_workload_is_the_whole_group(p):
    """GL(2, p) from the identity under the workload's six generators: the
    oracle's orbit is (p^2 - 1)(p^2 - p), the certified bound p^4 above it."""
    from multigpubfs_b200 import workloads
    g = workloads.gl2_graph(p)
    assert workloads.primitive_root(p) == min(r for r in range(2, p) if len({pow(r, k, p) for k in range(1, p)}) == p - 1)
    assert sum(G.layer_sizes(g)) == (p * p - 1) * (p * p - p) < p ** 4
