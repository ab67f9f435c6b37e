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


def test_batch_overflow_reruns_exactly_and_waves():
    from multigpubfs_b200.batch import BatchSweep
    graphs = _instances(24, False, 99)
    expect = _oracle_tables(graphs)
    with BatchSweep(graphs) as sweep:
        # Capacities far too small: every instance overflows once and is rerun
        # with its orbit bound; a small memory budget forces several waves.
        st = sweep.run(capacities=[4] * len(graphs), memory_bytes=96 << 20)
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
