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
    caps = predicted_capacities(net, graphs, margin=0.5, floor=0)  # deliberately tight: forces reruns
    with BatchSweep(graphs) as sweep:
        st = sweep.run(capacities=caps)
        assert sweep.layer_tables() == expect
    assert st["complete_instances"] == 16
