"""Seeded random parity sweep: random permutation graphs (distinct and
repeated labels, directed and inverse-closed generator sets, 2 to 7
generators on 5 to 10 points) and random modular-matrix graphs, each run
under a random choice of the plan shapes a caller or the autotuner can ask
for (visited set, claim mode, parents per thread, resident blocks, host or
device loop, parent-edge skip), against the oracle's layer tables and
samples.  The seed is fixed, so a failure names a reproducible case."""
import random

import pytest

from oracle import graph_oracle as G
from oracle import packed_oracle as P

pytestmark = pytest.mark.gpu

SEED = 20261204
CASES = 128


def _permutation_case(rng):
    n = rng.randint(5, 10)
    gens = [rng.sample(range(n), n) for _ in range(rng.randint(2, 4))]
    if rng.random() < 0.5:
        gens = G.add_inverses(gens)
    labels = list(range(n))
    if rng.random() < 0.35:
        labels = [rng.randint(0, max(1, n // 2)) for _ in range(n)]
        labels[0] = 0
    return gens, labels


def _plan(rng, distinct, closed):
    choices = [dict(visited="auto")]
    choices += [dict(visited="bitmap", dedup=d) for d in ("atomic", "warp")]
    choices += [dict(visited="hash"), dict(visited="hash", wide_slots=True)]
    if closed:
        choices.append(dict(visited="hash3"))
    choices.append(dict(visited="bitmap", dedup="sort"))
    if distinct:
        choices.append(dict(visited="bitmap", dedup="bucket", bucket_min_work=1))
        choices.append(dict(visited="bitmap", dedup="grouped", bucket_min_work=1))
    plan = dict(rng.choice(choices))
    if plan.get("dedup") in (None, "atomic", "warp") and plan.get("visited") != "hash3":
        plan["parents_per_thread"] = rng.choice([0, 1, 2, 4])
    plan["blocks_per_sm"] = rng.choice([0, 0, 2, 8])
    plan["host_loop"] = rng.random() < 0.3
    plan["parent_skip"] = rng.random() < 0.8
    return plan


@pytest.mark.parametrize("case", range(CASES))
def test_random_permutation_graph_under_a_random_plan(case):
    from multigpubfs_b200 import GraphDefinition
    from multigpubfs_b200.engine import NativeGraph
    from multigpubfs_b200.native import NativeError
    rng = random.Random(SEED * 1000 + case)
    gens, labels = _permutation_case(rng)
    distinct = len(set(labels)) == len(labels)
    closed = G.inverse_closed(G.permutation_graph(gens, labels))
    plan = _plan(rng, distinct, closed)
    expect, last, prev = P.packed_bfs(gens, labels, use_bitmap=False, sample=1000)
    with NativeGraph(GraphDefinition.permutation(gens, labels)) as e:
        try:
            e.plan(**plan)
        except NativeError as exc:
            assert exc.code == 5, (gens, labels, plan)  # UNSUPPORTED for this graph: nothing ran
            return
        r = e.run()
        got_last, got_prev = e.sample(0, 1000), e.sample(1, 1000)
    assert r.complete and r.layer_sizes == expect, (gens, labels, plan)
    # A layer of at most 1000 states is sampled whole; a larger one gives
    # 1000 of its states (frontier order), which must all belong to it.
    if expect[-1] <= 1000:
        assert got_last == last, (gens, labels, plan)
    else:
        assert len(got_last) == 1000 and got_last == sorted(got_last)
        if expect[-1] <= 20000:
            _, whole, _ = P.packed_bfs(gens, labels, use_bitmap=False, sample=expect[-1])
            members = {tuple(x) for x in whole}
            assert all(tuple(x) in members for x in got_last), (gens, labels, plan)
    if len(expect) > 1 and expect[-2] < 1000:
        assert got_prev == prev, (gens, labels, plan)


@pytest.mark.parametrize("case", range(24))
def test_random_matrix_graph_under_a_random_plan(case):
    from multigpubfs_b200 import GraphDefinition
    from multigpubfs_b200.engine import NativeGraph
    rng = random.Random(SEED * 7 + case)
    rows, cols = rng.choice([(2, 2), (2, 1), (3, 1), (2, 3)])
    p = rng.choice([q for q in (3, 5, 7, 11, 13) if q ** (rows * cols) <= 1 << 17])
    gens = []
    for _ in range(rng.randint(2, 4)):
        m = [rng.randint(-2, p + 2) for _ in range(rows * rows)]
        gens.append((m, p))
    start = [rng.randint(0, p - 1) for _ in range(rows * cols)]
    graph = G.matrix_graph(rows, cols, gens, start)
    expect = G.layer_sizes(graph, 1 << 17)
    plan = dict(rng.choice([dict(visited="auto"), dict(visited="bitmap"), dict(visited="hash"),
                            dict(visited="bitmap", dedup="bucket", bucket_min_work=1)]))
    plan["host_loop"] = rng.random() < 0.3
    with NativeGraph(GraphDefinition.matrix(rows, cols, gens, start)) as e:
        info = e.plan(**plan)
        r = e.run()
    assert info["packed"] == 1
    assert r.complete and r.layer_sizes == expect, (rows, cols, gens, start, plan)


@pytest.mark.parametrize("case", range(6))
def test_random_batched_sweep_under_random_shapes(case):
    """64 random instances in one batched run under random tile sizes,
    resident blocks, layer loops, memory budgets (several waves) and
    predicted capacities between a third of and twice each instance's true
    peak layer (under-predictions redo layers inside the launch)."""
    from multigpubfs_b200 import workloads
    from multigpubfs_b200.batch import BatchSweep
    rng = random.Random(SEED * 13 + case)
    graphs, expect = [], []
    while len(graphs) < 64:
        gens, labels = _permutation_case(rng)
        if len(labels) > 9:
            continue
        labels = list(range(len(labels)))  # the batched path takes distinct labels
        graphs.append(workloads.permutation_graph(gens, labels))
        expect.append(P.packed_bfs(gens, labels)[0])
    opts = dict(tile_entries=rng.choice([256, 512, 1024]), blocks_per_sm=rng.choice([0, 2, 3]),
                memory_bytes=rng.choice([None, 64 << 20, 256 << 20]))
    loop = rng.choice(["persistent", "host", "graph"])
    caps = [max(1, int(max(t) * rng.uniform(0.34, 2.0))) for t in expect] if rng.random() < 0.6 else None
    with BatchSweep(graphs, 0) as sweep:
        status = sweep.run(capacities=caps, host_loop=loop == "host", graph_loop=loop == "graph", **opts)
        tables = sweep.layer_tables()
    assert status["complete_instances"] == 64 and not status["fatal"], (opts, loop, status)
    assert tables == expect, (opts, loop)


@pytest.mark.parametrize("case", range(12))
def test_random_graph_split_over_random_ranks(case):
    """The owner-partitioned path (every rank's shard in one process) on
    random graphs of distinct labels, 1 to 9 ranks, random route chunks."""
    from multigpubfs_b200 import GraphDefinition, sharded
    rng = random.Random(SEED * 17 + case)
    gens, labels = _permutation_case(rng)
    labels = list(range(len(labels)))
    expect = P.packed_bfs(gens, labels)[0]
    world = rng.randint(1, 9)
    chunk = rng.choice([32, 1000, 1 << 25])
    got = sharded.run_emulated(GraphDefinition.permutation(gens, labels), world, chunk_parents=chunk)
    assert got == expect, (gens, world, chunk)
