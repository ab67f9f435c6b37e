"""Autotuner pilots on the device: every candidate expands the same layer
prefix exactly, the choice is cached, and run_graph with autotune on stays
exact."""
import json

import pytest

from oracle import graph_oracle as G

pytestmark = pytest.mark.gpu


def _lrx(n):
    from multigpubfs_b200 import GraphDefinition
    return GraphDefinition.permutation(G.lrx_generators(n), list(range(n)))


def test_pilots_compare_every_candidate_then_cache(tmp_path, lrx_layers):
    from multigpubfs_b200 import autotune
    from multigpubfs_b200.engine import NativeGraph
    g = _lrx(11)
    cache = tmp_path / "tune.json"
    got = autotune.choose_profile(g, 0, cache=cache)
    assert got["source"] == "pilot"
    cands = autotune.candidate_plans(g)
    # Stage 1: every path; stage 2: the shapes of the kept path, its default first.
    plans = [t["plan"] for t in got["trials"]]
    assert plans[:len(cands)] == cands and len(plans) > len(cands)
    shapes = plans[len(cands):]
    assert all({k: v for k, v in s.items() if k in ("visited", "dedup", "shards")} == shapes[0] for s in shapes)
    assert all(t["seconds"] is not None and t["seconds"] > 0 for t in got["trials"]), got["trials"]
    assert got["plan"] in plans
    again = autotune.choose_profile(g, 0, cache=cache)
    assert again["source"] == "cache" and again["plan"] == got["plan"]
    assert len(json.loads(cache.read_text())) == 1
    with NativeGraph(g) as e:
        e.plan(**got["plan"])
        assert e.run().layer_sizes == lrx_layers[11]


def test_run_graph_with_autotune_is_exact(tmp_path, monkeypatch, lrx_layers):
    from multigpubfs_b200.launch import run_graph
    monkeypatch.setenv("MGBFS2_AUTOTUNE_CACHE", str(tmp_path / "tune.json"))
    report = run_graph(_lrx(11), tmp_path / "out", autotune=True)
    assert report["status"] == "COMPLETE" and report["layer_sizes"] == lrx_layers[11]
    assert report["autotune"]["source"] == "pilot"
    report2 = run_graph(_lrx(11), tmp_path / "out2", autotune=True)
    assert report2["autotune"]["source"] == "cache" and report2["layer_sizes"] == lrx_layers[11]
    small = run_graph(_lrx(8), tmp_path / "out3", autotune=True)
    assert small["autotune"]["source"] == "size" and small["layer_sizes"] == lrx_layers[8]


def test_sweep_shape_pilots_stay_exact_then_cache(tmp_path):
    from multigpubfs_b200 import autotune, workloads
    from multigpubfs_b200.batch import BatchSweep
    graphs = workloads.sweep(48)
    cache = tmp_path / "tune.json"
    got = autotune.choose_sweep_shape(graphs, 0, sample=16, cache=cache)
    assert got["source"] == "pilot" and len(got["sample"]) == 16
    assert [t["plan"] for t in got["trials"]] == autotune.SWEEP_SHAPES
    assert all(t["seconds"] is not None and t["seconds"] > 0 for t in got["trials"]), got["trials"]
    assert got["shape"] in autotune.SWEEP_SHAPES
    again = autotune.choose_sweep_shape(graphs, 0, sample=16, cache=cache)
    assert again["source"] == "cache" and again["shape"] == got["shape"]
    with BatchSweep(graphs, 0) as sweep:
        sweep.run()
        plain = sweep.layer_tables()
        for shape in autotune.SWEEP_SHAPES[1:]:
            sweep.run(**shape)
            assert sweep.layer_tables() == plain, shape
