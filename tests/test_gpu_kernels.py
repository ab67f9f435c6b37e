"""Kernel-level contract tests of the C-ABI building blocks against the oracle.

Mirrors the reference's kernel harnesses: tests/generic_graph_gpu.py (every
child vs GraphDefinition.successor, int64 wrap, 300-cycle) and
tests/permutation_bitmap_gpu.cu (exhaustive rank bijection, large-n known
ranks, rejection of invalid states, claim uniqueness under concurrent streams).
"""
import itertools
import math

import numpy as np
import pytest

from oracle import graph_oracle as G
from oracle import packed_oracle as P

pytestmark = pytest.mark.gpu


def _torch():
    import torch
    return torch


def test_successors_i64_matches_oracle(exact_cases):
    torch = _torch()
    from multigpubfs_b200 import GraphDefinition
    from multigpubfs_b200.kernels import successors_i64
    checked = 0
    for case in exact_cases:
        g = GraphDefinition.from_dict(case["graph"])
        states = [k["state"] for k in case["successors"]]
        uniq = [list(s) for s in dict.fromkeys(tuple(s) for s in states)]
        out = successors_i64(g, torch.tensor(uniq, dtype=torch.int64, device="cuda")).cpu().tolist()
        for kat in case["successors"]:
            row = uniq.index(kat["state"])
            assert out[row][kat["generator"]] == kat["child"], case["name"]
            checked += 1
    assert checked > 200


def test_successor_wrap_known_answers():
    from multigpubfs_b200 import GraphDefinition
    assert GraphDefinition.matrix(1, 1, [([2], 7)], [(1 << 63) - 1]).successor([(1 << 63) - 1], 0) == [5]
    assert GraphDefinition.matrix(1, 1, [([2], 0)], [(1 << 63) - 1]).successor([(1 << 63) - 1], 0) == [-2]
    g = GraphDefinition.matrix(1, 1, [([2], 5), ([3], 7)], [4])
    assert g.successor([4], 0) == [3] and g.successor([4], 1) == [5]
    cyc = GraphDefinition.permutation([list(range(1, 300)) + [0]], list(range(300)))
    assert cyc.successor(list(range(300)), 0) == list(range(1, 300)) + [0]


@pytest.mark.parametrize("n,bits", [(8, 4), (13, 4), (16, 4), (8, 8)])
def test_packed_successors_match_oracle(n, bits):
    torch = _torch()
    from multigpubfs_b200.kernels import successors_packed
    rng = np.random.default_rng(n * 100 + bits)
    gens = [list(map(int, rng.permutation(n))) for _ in range(5)] + G.lrx_generators(n)
    states = [list(map(int, rng.permutation(n))) for _ in range(257)]
    words = torch.tensor([P.pack(s, bits) - (1 << 64 if P.pack(s, bits) >= 1 << 63 else 0) for s in states],
                         dtype=torch.int64, device="cuda")
    out = successors_packed(n, bits, gens, words).cpu().tolist()
    for i, s in enumerate(states):
        for k, g in enumerate(gens):
            assert out[i][k] & ((1 << 64) - 1) == P.pack([s[j] for j in g], bits)


def _words(states, bits):
    torch = _torch()
    vals = [P.pack(s, bits) for s in states]
    return torch.tensor([v - (1 << 64) if v >= 1 << 63 else v for v in vals], dtype=torch.int64, device="cuda")


@pytest.mark.parametrize("start", [[0, 1, 2, 3], [0, 0, 1, 2, 2], [0, 1, 1, 1, 2, 3], [0, 1, 2, 3, 4, 5, 6]])
def test_rank_exhaustive_bijection(start):
    from multigpubfs_b200.kernels import rank_packed
    ordered = sorted(set(itertools.permutations(start)))
    counts = [start.count(c) for c in sorted(set(start))]
    ranks, err = rank_packed(len(start), 4, counts, _words([list(s) for s in ordered], 4))
    assert int(err.item()) == 0
    assert ranks.cpu().tolist() == list(range(len(ordered)))


@pytest.mark.parametrize("n", [13, 16])
def test_rank_known_large(n):
    from multigpubfs_b200.kernels import rank_packed
    total = math.factorial(n)
    want = [0, 1, 4294967313, total // 2, total - 1]
    states = [G.multiset_unrank(list(range(n)), r) for r in want]
    ranks, err = rank_packed(n, 4, [1] * n, _words(states, 4))
    assert int(err.item()) == 0
    assert [r & ((1 << 64) - 1) for r in ranks.cpu().tolist()] == want


def test_rank_rejects_invalid_states():
    from multigpubfs_b200.kernels import rank_packed
    # duplicate symbol in a distinct domain, and an out-of-alphabet symbol
    ranks, err = rank_packed(4, 4, [1, 1, 1, 1], _words([[0, 0, 2, 3], [0, 1, 2, 9], [3, 2, 1, 0]], 4))
    r = ranks.cpu().tolist()
    assert r[0] == -1 and r[1] == -1 and r[2] == 23 and int(err.item()) & 4
    ranks, err = rank_packed(5, 4, [2, 1, 2], _words([[0, 0, 0, 1, 2], [2, 2, 1, 0, 0]], 4))
    assert ranks.cpu().tolist()[0] == -1 and ranks.cpu().tolist()[1] == 29


@pytest.mark.parametrize("warp", [True, False])
def test_bitmap_claim_exactly_once_under_concurrency(warp):
    torch = _torch()
    from multigpubfs_b200.kernels import bitmap_claim
    domain = 5040
    rng = np.random.default_rng(1)
    ranks = torch.tensor(rng.integers(0, domain, size=200000), dtype=torch.int64, device="cuda")
    bitmap = torch.zeros((domain + 63) // 64, dtype=torch.int64, device="cuda")
    s1, s2 = torch.cuda.Stream(), torch.cuda.Stream()
    with torch.cuda.stream(s1):
        won1, e1 = bitmap_claim(ranks[:100000], bitmap, domain, warp)
    with torch.cuda.stream(s2):
        won2, e2 = bitmap_claim(ranks[100000:], bitmap, domain, warp)
    torch.cuda.synchronize()
    won = torch.cat([won1, won2]).bool()
    winners = ranks[won].cpu().numpy()
    assert len(winners) == len(set(winners.tolist())) == len(np.unique(ranks.cpu().numpy()))
    assert int(e1.item()) == 0 and int(e2.item()) == 0


def test_hash_insert_exact():
    torch = _torch()
    from multigpubfs_b200.kernels import hash_insert
    rng = np.random.default_rng(2)
    keys = torch.tensor(rng.integers(0, 1 << 40, size=100000) % 30011, dtype=torch.int64, device="cuda")
    table = torch.full((1 << 16,), -1, dtype=torch.int64, device="cuda")
    inserted, err = hash_insert(keys, table)
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    winners = keys[inserted.bool()].cpu().numpy()
    assert sorted(winners.tolist()) == sorted(np.unique(keys.cpu().numpy()).tolist())
    again, _ = hash_insert(keys, table)
    assert int(again.sum().item()) == 0


@pytest.mark.parametrize("key_bits", [13, 33, 52, 63])
def test_sort_unique_tiles(key_bits):
    torch = _torch()
    from multigpubfs_b200.kernels import sort_unique_tiles
    rng = np.random.default_rng(key_bits)
    count = 4096 * 5 + 123
    raw = rng.integers(0, 1 << min(key_bits, 62), size=count, dtype=np.int64)
    idx = rng.integers(1, count, size=count // 3)
    raw[idx] = raw[idx - 1]  # plenty of duplicates inside each tile
    keys = torch.tensor(raw, device="cuda")
    out, counts = sort_unique_tiles(keys, key_bits)
    out = out.cpu().numpy()
    counts = counts.cpu().numpy()
    for t in range(len(counts)):
        tile = raw[t * 4096:(t + 1) * 4096]
        expect = np.unique(tile)
        assert counts[t] == len(expect)
        assert np.array_equal(out[t * 4096:t * 4096 + counts[t]], expect)


def test_bucket_keys():
    torch = _torch()
    from multigpubfs_b200.kernels import bucket_keys
    rng = np.random.default_rng(3)
    raw = rng.integers(0, 64 << 20, size=300000, dtype=np.int64)
    buckets, counts, err = bucket_keys(torch.tensor(raw, device="cuda"), 20, 64, 8192)
    assert int(err.item()) == 0
    counts = counts.cpu().numpy()
    buckets = buckets.cpu().numpy()
    for s in range(64):
        want = np.sort(raw[(raw >> 20) == s])
        assert counts[s] == len(want)
        assert np.array_equal(np.sort(buckets[s, :counts[s]]), want)
    # overflow: exact counts, error bit 3
    buckets, counts, err = bucket_keys(torch.tensor(raw, device="cuda"), 20, 64, 16)
    assert int(err.item()) & 8
    assert counts.sum().item() == len(raw)


def _layer_bfs(n, gens):
    """BFS driven entirely by mgbfs2_expand_layer_bitmap calls."""
    torch = _torch()
    from multigpubfs_b200.kernels import expand_layer_bitmap
    bitmap = torch.zeros((math.factorial(n) + 63) // 64, dtype=torch.int64, device="cuda")
    start = P.pack(list(range(n)), 4)
    bitmap[0] = 1  # rank of the identity is 0
    frontier = torch.tensor([start], dtype=torch.int64, device="cuda")
    layers = [frontier.cpu().tolist()]
    while frontier.numel():
        nxt, err = expand_layer_bitmap(n, gens, frontier, bitmap, frontier.numel() * len(gens))
        assert err == 0
        frontier = nxt.clone()
        if frontier.numel():
            layers.append(frontier.cpu().tolist())
    return layers


@pytest.mark.parametrize("n,family", [(9, "lrx"), (8, "coxeter"), (13, "lrx_prefix")])
def test_expand_layer_bitmap_bfs(n, family, lrx_layers):
    if family == "lrx_prefix":
        # S13 uses two-symbol shards; run the first 20 layers only.
        torch = _torch()
        from multigpubfs_b200.kernels import expand_layer_bitmap
        gens = G.lrx_generators(n)
        bitmap = torch.zeros((math.factorial(n) + 63) // 64, dtype=torch.int64, device="cuda")
        bitmap[0] = 1
        frontier = torch.tensor([P.pack(list(range(n)), 4)], dtype=torch.int64, device="cuda")
        sizes = [1]
        for _ in range(19):
            frontier, err = expand_layer_bitmap(n, gens, frontier, bitmap, frontier.numel() * 3)
            frontier = frontier.clone()
            assert err == 0
            sizes.append(frontier.numel())
        from tests.conftest import golden
        assert sizes == golden("lrx13_layers.json")["layers"][:20]
        return
    gens = G.lrx_generators(n) if family == "lrx" else G.coxeter_generators(n)
    layers = _layer_bfs(n, gens)
    expect = lrx_layers[n] if family == "lrx" else G.coxeter_layers(n)
    assert [len(x) for x in layers] == expect
    assert all(len(set(x)) == len(x) for x in layers)


def test_expand_layer_bitmap_states_match_oracle():
    n = 7
    gens = G.lrx_generators(n)
    exact = G.exact_layers(G.permutation_graph(gens, list(range(n))), 1 << 16)
    layers = _layer_bfs(n, gens)
    assert len(layers) == len(exact)
    for got, want in zip(layers, exact):
        assert sorted(P.unpack(w & ((1 << 64) - 1), n, 4) for w in got) == want


def test_expand_layer_bitmap_capacity_and_scratch_checks():
    torch = _torch()
    from multigpubfs_b200 import native
    from multigpubfs_b200.kernels import expand_layer_bitmap
    n = 8
    gens = G.lrx_generators(n)
    bitmap = torch.zeros((math.factorial(n) + 63) // 64, dtype=torch.int64, device="cuda")
    bitmap[0] = 1
    frontier = torch.tensor([P.pack(list(range(n)), 4)], dtype=torch.int64, device="cuda")
    nxt, err = expand_layer_bitmap(n, gens, frontier, bitmap, 1)  # 3 new states, room for 1
    assert err & 1 and nxt.numel() == 1
    small = torch.empty(16, dtype=torch.uint8, device="cuda")
    with pytest.raises(native.NativeError):
        expand_layer_bitmap(n, gens, frontier, bitmap, 8, scratch=small)
