"""The learned planner's kernels against the float64 CPU oracle, its training,
and the guarantee that it never changes results."""
import math

import numpy as np
import pytest

from oracle import graph_oracle as G
from oracle import mlp_oracle as M
from oracle import packed_oracle as P

pytestmark = pytest.mark.gpu


def _net(seed=1):
    from multigpubfs_b200.planner import PlannerNet, INPUTS
    rng = np.random.default_rng(seed)
    params = rng.normal(0, 0.3, M.param_count(INPUTS)).astype(np.float32)
    return PlannerNet(0, params=params), params, rng


def test_gradients_match_float64_oracle():
    from multigpubfs_b200.planner import INPUTS
    net, params, rng = _net()
    X = rng.normal(size=(300, INPUTS)).astype(np.float32)
    T = rng.normal(size=(300, 2)).astype(np.float32)
    loss, grad = net.loss_and_grad(X, T, weights=(1.0, 0.5))
    loss64, grad64 = M.loss_and_grad(params, X, T, INPUTS, (1.0, 0.5))
    assert abs(loss - loss64) <= 1e-4 * max(1.0, abs(loss64))
    # fp32 kernels vs float64 oracle: relative error per component, with an
    # absolute floor for near-zero components.
    assert np.max(np.abs(grad - grad64) / (np.abs(grad64) + 1e-3)) < 5e-3
    fd = M.finite_difference(params, X, T, INPUTS, (1.0, 0.5), idx=rng.integers(0, len(params), 20))
    for i, v in fd.items():
        assert abs(grad64[i] - v) <= 1e-5 * max(1.0, abs(v))


def test_forward_and_bf16_inference_match_oracle():
    from multigpubfs_b200.planner import INPUTS
    net, params, rng = _net(2)
    X = rng.normal(size=(1000, INPUTS)).astype(np.float32)
    y64, _ = M.forward(params, X, INPUTS)
    assert np.max(np.abs(net.predict_fp32(X) - y64)) < 1e-3 * max(1.0, np.abs(y64).max())
    # bf16 parameters/activations (8-bit mantissa), fp32 accumulation
    assert np.max(np.abs(net.predict(X) - y64)) < 0.05 * max(1.0, np.abs(y64).max())


def test_training_reduces_loss_and_predicts_layers():
    from multigpubfs_b200.planner import PlannerNet, training_set, rollout
    graphs = [G.sweep_instance(i, closed) for i in range(24) for closed in (False, True)]
    tables = [P.packed_bfs(g["action"]["generators"], g["start"])[0] for g in graphs]
    X, T = training_set(graphs, tables)
    net = PlannerNet(0, seed=3)
    hist = net.fit(X, T, steps=600, lr=3e-3)
    assert hist[-1] < 0.25 * hist[0]
    # The rollout's predicted peak is within a factor of 4 of the true peak
    # for most training graphs.
    prof = rollout(net, graphs)
    ratios = [max(p) / max(t) for p, t in zip(prof, tables)]
    assert np.median([abs(math.log(r)) for r in ratios]) < math.log(4)
    # The one-launch device rollout follows the host-stepped rollout (same
    # features, same bf16 kernel arithmetic; the orbit reaches the device as
    # fp32, so the last layer's clamp may differ by rounding).
    from multigpubfs_b200.planner import rollout_device
    peak, total, depth = rollout_device(net, graphs)
    for p, pk, tt, dp in zip(prof, peak, total, depth):
        assert abs(pk - max(p)) <= 1e-3 * max(p)
        assert abs(tt - sum(p)) <= 1e-3 * sum(p)
        assert abs(int(dp) - len(p)) <= 1


def test_learned_capacities_never_change_results():
    from multigpubfs_b200.batch import BatchSweep
    from multigpubfs_b200.planner import PlannerNet, training_set, predicted_capacities
    train = [G.sweep_instance(i, True) for i in range(16)]
    tables = [P.packed_bfs(g["action"]["generators"], g["start"])[0] for g in train]
    net = PlannerNet(0, seed=4)
    net.fit(*training_set(train, tables), steps=300)
    graphs = [G.sweep_instance(100 + i, True) for i in range(16)]
    expect = [P.packed_bfs(g["action"]["generators"], g["start"])[0] for g in graphs]
    caps = predicted_capacities(net, graphs, margin=0.5, floor=0)  # deliberately tight: forces layer redos
    with BatchSweep(graphs) as sweep:
        st = sweep.run(capacities=caps)
        assert sweep.layer_tables() == expect
    assert st["complete_instances"] == 16


# ---------------------------------------------------------------------------
# The learned planner on single graphs (mgbfs2_plan with MGBFS2_PLANNER_LEARNED).

def _projective_graph():
    """PGL(2,13) on the 14 points of the projective line over Z/13 (x -> x+1,
    x -> 2x, x -> -1/x; 13 stands for infinity): transitive, |G| = 2,184,
    while the plain planner's worst-case bound is 14! and its rank domain a
    10.9 GB bitmap."""
    inf = 13

    def inv(x):
        return pow(x, 11, 13)  # x^(p-2) mod p
    shift = [(x + 1) % 13 for x in range(13)] + [inf]
    scale = [(2 * x) % 13 for x in range(13)] + [inf]
    flip = [inf] + [(-inv(x)) % 13 for x in range(1, 13)] + [0]
    return G.permutation_graph([shift, scale, flip], list(range(14)))


def test_learned_plan_needs_a_prediction():
    from multigpubfs_b200 import GraphDefinition
    from multigpubfs_b200.engine import NativeGraph
    from multigpubfs_b200.native import NativeError
    with NativeGraph(GraphDefinition.from_dict(_projective_graph())) as e:
        with pytest.raises(NativeError) as info:
            e.plan(planner="learned")
        assert info.value.code == 1  # MGBFS2_INVALID_ARGUMENT: not a silent no-op


def test_learned_plan_differs_from_plain_with_identical_tables():
    from multigpubfs_b200 import GraphDefinition, native
    from multigpubfs_b200.engine import NativeGraph
    from multigpubfs_b200.planner import PlannerNet, predict_graph
    g = _projective_graph()
    assert native.group_order(g["action"]["generators"]) == 2184
    expect, _, _ = P.packed_bfs(g["action"]["generators"], g["start"], use_bitmap=False, max_states=1 << 16)
    net = PlannerNet(0, seed=1)  # the states are exact (|G|) whatever the network
    kw = predict_graph(g, net, margin=1.5)
    assert kw["predicted_states"] == 2184 and kw["exact_states"]
    kw.pop("exact_states")
    with NativeGraph(GraphDefinition.from_dict(g)) as e:
        plain = e.plan()
        r_plain = e.run()
        learned = e.plan(**kw)
        r_learned = e.run()
        # An under-prediction: the table starts far too small, the device loop
        # pauses before the threshold and the host loop grows it by rehash.
        small = e.plan(planner="learned", predicted_states=40, predicted_peak=8)
        r_small = e.run()
    assert plain["visited"] == "bitmap" and plain["bitmap_bits"] == 87178291200
    # 56-bit keys in a small table leave too few bits for quotient slots.
    assert learned["planner"] == "learned" and learned["visited"] == "hash" and learned["table_slot_bytes"] == 8
    assert learned["table_slots"] <= (1 << 13) and small["table_slots"] < learned["table_slots"]
    assert r_plain.layer_sizes == r_learned.layer_sizes == r_small.layer_sizes == expect
    assert r_plain.complete and r_learned.complete and r_small.complete


def test_run_graph_learned_planner_reports_its_prediction(tmp_path):
    import json
    from multigpubfs_b200 import GraphDefinition, run_graph
    g = GraphDefinition.from_dict(_projective_graph())
    report = run_graph(g, tmp_path / "learned", planner="learned", autotune=False)
    assert report["planner"]["name"] == "learned" and report["planner"]["predicted_states"] == 2184
    assert report["plan"]["visited"] == "hash" and sum(report["layer_sizes"]) == 2184
    plain = run_graph(g, tmp_path / "plain", autotune=False)
    assert plain["layer_sizes"] == report["layer_sizes"] and plain["plan"]["visited"] == "bitmap"
    assert json.loads((tmp_path / "learned" / "report.json").read_text())["status"] == "COMPLETE"


def test_learned_underprediction_grows_the_quotient_table():
    """S9 LRX (36-bit keys) with a prediction of 500 states: a 4096-slot
    quotient table that the run grows by rehash, layer table unchanged."""
    from multigpubfs_b200 import GraphDefinition
    from multigpubfs_b200.engine import NativeGraph
    from tests.conftest import golden
    g = GraphDefinition.from_dict(G.permutation_graph(G.lrx_generators(9), list(range(9))))
    with NativeGraph(g) as e:
        info = e.plan(visited="hash", planner="learned", predicted_states=500, predicted_peak=100)
        r = e.run()
    assert info["table_slot_bytes"] == 4 and info["table_slots"] == 4096
    assert r.complete and r.layer_sizes == golden("lrx_layers.json")["layers"]["9"]
