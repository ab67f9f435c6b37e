"""Bitmaps over position-component product domains (generators that keep
groups of positions apart): the device rank against the oracle's restatement
of the reference's PositionOrbitDomain, and whole BFS runs on multi-component
graphs against the oracles."""
import ctypes as C
import itertools

import pytest

from oracle import graph_oracle as G
from oracle import packed_oracle as P
from tests.test_oracle import PRODUCT_CASES

pytestmark = pytest.mark.gpu


def _device_ranks(start, gens, states):
    import torch
    from multigpubfs_b200 import native
    lib = native.require_device()
    codes, labels = P.codes_of(start)
    bits = P.bits_for(len(labels))
    index = {v: k for k, v in enumerate(labels)}
    words = torch.tensor([P.pack([index[v] for v in s], bits) for s in states], dtype=torch.int64, device="cuda")
    ranks = torch.zeros_like(words)
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    n = len(start)
    c_codes = (C.c_uint32 * n)(*codes)
    flat = (C.c_uint32 * (n * len(gens)))(*[x for g in gens for x in g])
    size = C.c_uint64()
    rc = lib.mgbfs2_rank_components(n, bits, len(labels), c_codes, len(gens), flat, words.data_ptr(), words.numel(),
                                    ranks.data_ptr(), C.byref(size), err.data_ptr(), native.stream_handle())
    torch.cuda.synchronize()
    assert rc == 0
    return [int(r) & ((1 << 64) - 1) for r in ranks.tolist()], int(size.value), int(err.item())


@pytest.mark.parametrize("case", range(len(PRODUCT_CASES)))
def test_component_rank_is_the_reference_bijection(case):
    start, gens, size = PRODUCT_CASES[case]
    states = [G.product_unrank(start, gens, r) for r in range(size)]
    ranks, domain, err = _device_ranks(start, gens, states)
    assert domain == size and err == 0
    assert ranks == list(range(size))


def test_component_rank_rejects_states_outside_the_domain():
    start = list(range(6))
    gens = [[1, 0, 2, 3, 4, 5], [0, 1, 2, 4, 3, 5]]   # components {0,1}, {2}, {3,4}, {5}
    inside = [G.product_unrank(start, gens, r) for r in range(4)]
    outside = [[2, 1, 0, 3, 4, 5]]                     # 2 left its component
    ranks, domain, err = _device_ranks(start, gens, inside + outside)
    assert domain == 4 and ranks[:4] == [0, 1, 2, 3]
    assert ranks[4] == (1 << 64) - 1 and err & 4


def _s10_on_14():
    gens = []
    for i in range(9):
        g = list(range(14))
        g[i], g[i + 1] = g[i + 1], g[i]
        gens.append(g)
    return G.permutation_graph(gens, list(range(14)))


def test_s10_on_14_points_uses_the_10_factorial_bitmap():
    """Adjacent transpositions of the first 10 of 14 points: the plain
    multiset domain would be 14! bits (10.9 GB); the product domain is 10!."""
    from multigpubfs_b200 import GraphDefinition
    from multigpubfs_b200.engine import NativeGraph
    with NativeGraph(GraphDefinition.from_dict(_s10_on_14())) as e:
        info = e.plan(visited="bitmap")
        r = e.run()
    assert info["bitmap_bits"] == 3628800 and info["rank_components"] == 5
    assert r.complete and r.layer_sizes == G.coxeter_layers(10)


@pytest.mark.parametrize("variant", [dict(visited="bitmap", dedup="atomic"), dict(visited="bitmap", dedup="warp"),
                                     dict(visited="bitmap", dedup="sort"),
                                     dict(visited="bitmap", dedup="atomic", host_loop=True)])
def test_multi_component_graphs_match_the_oracle(variant):
    from multigpubfs_b200 import GraphDefinition
    from multigpubfs_b200.engine import NativeGraph
    graphs = [
        # L and R on positions 0..5, a transposition on 6..9, labels repeated across components
        G.permutation_graph([[1, 2, 3, 4, 5, 0, 6, 7, 8, 9], [5, 0, 1, 2, 3, 4, 6, 7, 8, 9],
                             [0, 1, 2, 3, 4, 5, 7, 6, 9, 8], [0, 1, 2, 3, 4, 5, 8, 9, 6, 7]],
                            [0, 0, 1, 1, 2, 3, 4, 4, 5, 6]),
        # two 3-cycles and a swap of components {0,1,2}, {3,4,5}, {6,7}
        G.permutation_graph([[1, 2, 0, 3, 4, 5, 6, 7], [0, 1, 2, 4, 5, 3, 6, 7], [0, 2, 1, 3, 4, 5, 7, 6]],
                            [5, 6, 7, 5, 6, 7, 1, 2]),
    ] + [G.permutation_graph(gens, start) for start, gens, _ in PRODUCT_CASES]
    for g in graphs:
        expect, last, prev = P.packed_bfs(g["action"]["generators"], g["start"], use_bitmap=False, sample=1000)
        with NativeGraph(GraphDefinition.from_dict(g)) as e:
            info = e.plan(**variant)
            r = e.run()
            assert e.sample(0, 1000) == last and e.sample(1, 1000) == prev
        assert r.complete and r.layer_sizes == expect, g
        if len(G.position_components(len(g["start"]), g["action"]["generators"])) > 1:
            assert info["rank_components"] > 1
            assert info["bitmap_bits"] == G.product_domain(g["start"], g["action"]["generators"])[1]
