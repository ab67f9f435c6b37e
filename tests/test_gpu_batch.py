"""Batched sweep parity: every instance's layer table bit-exact vs the C oracle.

Instances follow the sweep definition (n uniform in {7,8,9,10}, 2-3 seeded
uniform random permutations; directed, and an inverse-closed variant adding
inverses), run together, each wave as one persistent cooperative launch (or,
compared, a CUDA-graph WHILE loop or a host-driven loop).
"""
import pytest

from oracle import graph_oracle as G
from oracle import packed_oracle as P

pytestmark = pytest.mark.gpu


def _instances(count, closed, seed_base=20261203):
    return [G.sweep_instance(i, closed, seed_base) for i in range(count)]


def _oracle_tables(graphs):
    return [P.packed_bfs(g["action"]["generators"], g["start"])[0] for g in graphs]


@pytest.mark.parametrize("closed", [False, True])
def test_batch_matches_oracle(closed):
    from multigpubfs_b200.batch import BatchSweep
    graphs = _instances(40, closed)
    expect = _oracle_tables(graphs)
    with BatchSweep(graphs) as sweep:
        st = sweep.run()
        # One wave: its seed and ONE persistent launch for all layers.
        assert st["complete_instances"] == 40 and st["waves"] == 1 and st["redo_instances"] == 0
        assert st["graph_launches"] == 0 and st["kernel_launches"] == 2 and st["layer_steps"] > 10
        assert sweep.layer_tables() == expect
        assert st["states"] == sum(map(sum, expect))


def test_batch_loop_modes_agree():
    from multigpubfs_b200.batch import BatchSweep
    graphs = _instances(24, True, 777)
    expect = _oracle_tables(graphs)
    with BatchSweep(graphs) as sweep:
        a = sweep.run(host_loop=True)
        ta = sweep.layer_tables()
        b = sweep.run(graph_loop=True)
        tb = sweep.layer_tables()
        c = sweep.run()
        tc = sweep.layer_tables()
        # Several waves: the persistent kernel starts from fresh barrier state
        # in each.
        d = sweep.run(memory_bytes=96 << 20)
        td = sweep.layer_tables()
    assert ta == tb == tc == td == expect
    assert a["graph_launches"] == 0 and b["graph_launches"] >= 1 and c["graph_launches"] == 0
    assert c["kernel_launches"] == 2 * c["waves"] and d["waves"] > 1 and d["kernel_launches"] == 2 * d["waves"]
    with pytest.raises(ValueError):
        sweep_opts = BatchSweep(graphs)
        try:
            sweep_opts.run(host_loop=True, graph_loop=True)
        finally:
            sweep_opts.close()


def test_batch_overflow_redoes_layers_exactly():
    from multigpubfs_b200.batch import BatchSweep
    graphs = _instances(24, False, 99)
    expect = _oracle_tables(graphs)
    with BatchSweep(graphs) as sweep:
        # Capacities far too small: every instance overflows, and each
        # overflowing layer is redone in a larger segment from the wave's pool
        # (with the whole device's budget the pool never runs out).
        st = sweep.run(capacities=[4] * len(graphs))
        assert sweep.layer_tables() == expect
        assert st["redo_layers"] >= len(graphs) and st["redo_instances"] == 0 and st["waves"] == 1
        # The same through the graph and host loops (the moves as their own launch).
        for kw in ({"graph_loop": True}, {"host_loop": True}):
            other = sweep.run(capacities=[4] * len(graphs), **kw)
            assert sweep.layer_tables() == expect
            assert other["redo_layers"] >= len(graphs) and other["redo_instances"] == 0
        # A tighter budget: redos while the pool lasts, reruns after.
        tight = sweep.run(capacities=[4] * len(graphs), memory_bytes=96 << 20)
        assert sweep.layer_tables() == expect and tight["redo_layers"] > 0


def test_batch_exhausted_pool_reruns_exactly_and_waves():
    from multigpubfs_b200.batch import BatchSweep
    graphs = _instances(24, False, 99)
    expect = _oracle_tables(graphs)
    with BatchSweep(graphs) as sweep:
        # A budget so small that the redo pool runs out: those instances are
        # rerun from depth 0 with their orbit bound in later waves.
        st = sweep.run(capacities=[4] * len(graphs), memory_bytes=16 << 20)
        assert sweep.layer_tables() == expect
        assert st["redo_instances"] > 0 and st["waves"] > 1


def test_batch_rejects_unsupported():
    from multigpubfs_b200.batch import BatchSweep
    from multigpubfs_b200.native import NativeError
    with pytest.raises(NativeError):
        BatchSweep([G.permutation_graph([[1, 0, 2]], [0, 0, 1])])  # repeated labels
    with pytest.raises(ValueError):
        BatchSweep([G.matrix_graph(1, 1, [([2], 7)], [3])])


def test_batch_results_tables(tmp_path):
    import csv
    from multigpubfs_b200.batch import BatchSweep
    graphs = _instances(12, True, 31)
    expect = _oracle_tables(graphs)
    with BatchSweep(graphs) as sweep:
        st = sweep.run()
        secs = [sweep.layer_seconds(i) for i in range(len(graphs))]
        sweep.write_results(tmp_path)
    for table, s in zip(expect, secs):
        assert len(s) == len(table) and s[0] == 0.0 and all(x > 0 for x in s[1:])
    # Every instance of the one wave shares the wave's step times.
    deepest = max(range(len(expect)), key=lambda i: len(expect[i]))
    for s in secs:
        assert s == secs[deepest][:len(s)]
    assert sum(secs[deepest]) <= st["device_seconds"] * 1.01 + 1e-4
    with open(tmp_path / "layers.csv", newline="") as f:
        rows = list(csv.DictReader(f))
    got = {}
    for r in rows:
        got.setdefault(int(r["instance"]), []).append(int(r["count"]))
    assert [got[i] for i in range(len(expect))] == expect


# ---------------------------------------------------------------------------
# The batched workloads exactly as the benchmark runs them, against the
# oracle's tables in tests/golden/sweep_tables.json.

def test_sweep512_matches_fixture():
    """All 512 sweep instances in one run (one wave on a B200)."""
    from multigpubfs_b200 import workloads
    from multigpubfs_b200.batch import BatchSweep
    from tests.conftest import sweep_fixture
    expect = sweep_fixture("sweep512")["tables"]
    with BatchSweep(workloads.sweep(512)) as sweep:
        st = sweep.run()
        assert sweep.layer_tables() == expect
    assert st["complete_instances"] == 512 and st["states"] == sum(map(sum, expect))


def test_heldout_sweep_matches_fixture_in_many_waves():
    """The held-out sweep under a 256 MiB budget: dozens of waves."""
    from multigpubfs_b200 import workloads
    from multigpubfs_b200.batch import BatchSweep
    from tests.conftest import sweep_fixture
    expect = sweep_fixture("sweep512_heldout")["tables"]
    with BatchSweep(workloads.sweep(512, seed_base=20261203 + 4096)) as sweep:
        st = sweep.run(memory_bytes=256 << 20)
        assert sweep.layer_tables() == expect
    assert st["waves"] > 10 and st["complete_instances"] == 512


def test_planner_s12_instances_match_fixture():
    """Eight S12 planner instances (2-4 random generators plus inverses), with
    the plain capacities and with capacities far below their peak layers
    (every instance overflows and is recovered exactly)."""
    from multigpubfs_b200 import workloads
    from multigpubfs_b200.batch import BatchSweep
    from tests.conftest import sweep_fixture
    fixture = sweep_fixture("planner_s12")
    graphs = [workloads.planner_instance(i) for i in fixture["indices"]]
    with BatchSweep(graphs) as sweep:
        plain = sweep.run()
        assert sweep.layer_tables() == fixture["tables"]
        small = sweep.run(capacities=[max(t) // 3 for t in fixture["tables"]])
        assert sweep.layer_tables() == fixture["tables"]
    assert plain["redo_layers"] == plain["redo_instances"] == 0
    assert small["redo_layers"] >= len(graphs) and small["redo_instances"] == 0
