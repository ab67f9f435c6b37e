"""Autotuner host logic on CPU: candidates, the keep-the-default rule, the
pilot prefix, the cache and the size profile.  The pilots themselves run in
tests/test_gpu_autotune.py."""
import pytest

from multigpubfs_b200 import GraphDefinition, autotune
from oracle import graph_oracle as G


def _lrx(n):
    return GraphDefinition.permutation(G.lrx_generators(n), list(range(n)))


def test_candidates_for_lrx_and_matrix_graphs():
    plans = autotune.candidate_plans(_lrx(11))
    assert plans[0] == autotune.DEFAULT
    assert {"visited": "bitmap", "dedup": "bucket", "shards": 256} in plans
    assert {"visited": "hash3", "dedup": "atomic"} in plans  # L, R inverse pair and X an involution
    mat = GraphDefinition.from_dict(G.matrix_graph(2, 2, [([1, 1, 0, 1], 7), ([1, 0, 1, 1], 7)], [1, 0, 0, 1]))
    kinds = {(p["visited"], p["dedup"]) for p in autotune.candidate_plans(mat)}
    assert ("bitmap", "atomic") not in kinds and ("hash", "atomic") in kinds


def test_keep_the_default_unless_ten_percent_faster():
    d = {"visited": "auto", "dedup": "auto"}
    a = {"visited": "bitmap", "dedup": "atomic"}
    assert autotune.pick([{"plan": d, "seconds": 1.0}, {"plan": a, "seconds": 0.95}]) == d
    assert autotune.pick([{"plan": d, "seconds": 1.0}, {"plan": a, "seconds": 0.89}]) == a
    assert autotune.pick([{"plan": d, "seconds": None}, {"plan": a, "seconds": 3.0}]) == a
    assert autotune.pick([{"plan": d, "seconds": None}, {"plan": a, "seconds": None}]) == d


def test_pilot_depth_is_the_shortest_prefix_reaching_the_work():
    sizes = [1, 3, 9, 27, 81]
    assert autotune.pilot_depth(sizes, 3, work=3 * 13) == 3
    assert autotune.pilot_depth(sizes, 3, work=1 << 40) == len(sizes)


def test_cache_roundtrip(tmp_path):
    path = tmp_path / "sub" / "cache.json"
    assert autotune.load_cache(path) == {}
    autotune.store_cache(path, {"k": {"plan": {"visited": "hash"}}})
    assert autotune.load_cache(path)["k"]["plan"] == {"visited": "hash"}
    key = autotune.cache_key(_lrx(9), "B200", "abc")
    assert key.startswith(_lrx(9).digest()) and key.endswith("|B200|abc")


def test_small_graphs_take_the_size_profile_without_pilots(tmp_path):
    got = autotune.choose_profile(_lrx(9), 0, cache=tmp_path / "c.json")
    assert got == {"plan": autotune.DEFAULT, "source": "size", "trials": []}
    assert not (tmp_path / "c.json").exists()


def test_cache_path_override(monkeypatch, tmp_path):
    monkeypatch.setenv("MGBFS2_AUTOTUNE_CACHE", str(tmp_path / "x.json"))
    assert autotune.cache_path() == tmp_path / "x.json"


def test_shape_candidates_vary_the_kept_path_only():
    grouped = autotune.shape_candidates({"visited": "bitmap", "dedup": "grouped"},
                                        {"visited": "bitmap", "dedup": "grouped"})
    assert grouped[0] == {"visited": "bitmap", "dedup": "grouped"}
    assert {"visited": "bitmap", "dedup": "grouped", "group_chunk": 2048, "blocks_per_sm": 6} in grouped
    assert all(set(p) <= {"visited", "dedup", "group_chunk", "blocks_per_sm"} for p in grouped)
    hashed = autotune.shape_candidates(dict(autotune.DEFAULT), {"visited": "hash", "dedup": "atomic"})
    assert hashed[0] == autotune.DEFAULT and {"visited": "auto", "dedup": "auto", "hash_load_percent": 70} in hashed
    assert {"visited": "auto", "dedup": "auto", "parents_per_thread": 2} in hashed
    quotient = autotune.shape_candidates(dict(autotune.DEFAULT),
                                         {"visited": "hash", "dedup": "atomic", "parents_per_thread": 1})
    assert {"visited": "auto", "dedup": "auto", "parents_per_thread": 2} in quotient
    two = autotune.shape_candidates(dict(autotune.DEFAULT),
                                    {"visited": "hash", "dedup": "atomic", "parents_per_thread": 2})
    assert {"visited": "auto", "dedup": "auto", "parents_per_thread": 1} in two
    bucket = autotune.shape_candidates({"visited": "bitmap", "dedup": "bucket", "shards": 1},
                                       {"visited": "bitmap", "dedup": "bucket"})
    assert [p.get("bucket_margin") for p in bucket] == [None, 1024, 16384]
    assert autotune.shape_candidates(dict(autotune.DEFAULT), {"visited": "hash3", "dedup": "atomic"}) == \
        [autotune.DEFAULT]


def test_sweep_sample_spreads_over_the_sweep():
    assert autotune.sweep_sample(10) == list(range(10))
    picked = autotune.sweep_sample(512, 64)
    assert len(picked) == 64 and picked[0] == 0 and picked[-1] == 504
    assert all(b - a == 8 for a, b in zip(picked, picked[1:]))
    assert autotune.SWEEP_SHAPES[0] == {}   # the default shape is the first trial


def test_sweep_cache_key_depends_on_every_instance():
    from oracle import graph_oracle as G
    a = [G.sweep_instance(i, False) for i in range(4)]
    b = a[:3] + [G.sweep_instance(9, False)]
    assert autotune.sweep_cache_key(a, "B200", "x") == autotune.sweep_cache_key(list(a), "B200", "x")
    assert autotune.sweep_cache_key(a, "B200", "x") != autotune.sweep_cache_key(b, "B200", "x")
    assert autotune.sweep_cache_key(a, "B200", "x").startswith("sweep:")
