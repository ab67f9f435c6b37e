"""GPU parity: every layer table bit-exact against the reference-pinned oracle.

Runs libmgbfs2 through its C ABI (multigpubfs_b200.engine.NativeGraph) on every
golden case, on LRX S3..S11 (reference packed search), on S13 LRX (the
reference's shipped table) and Coxeter S13 (Mahonian certificate), and on
seeded random generator sets against the C oracle, for each visited-set /
dedup variant that applies.
"""
import math

import pytest

from oracle import graph_oracle as G
from oracle import packed_oracle as P
from tests.conftest import golden

pytestmark = pytest.mark.gpu


def _engine():
    from multigpubfs_b200.engine import NativeGraph
    return NativeGraph


def run(graph_dict, **plan):
    from multigpubfs_b200 import GraphDefinition
    from multigpubfs_b200.native import NativeError
    g = GraphDefinition.from_dict(graph_dict)
    with _engine()(g) as e:
        try:
            info = e.plan(**plan)
        except NativeError as exc:
            if exc.code == 2:  # MGBFS2_UNSUPPORTED for this variant
                return None
            raise
        r = e.run()
        return info, r, e.sample(0, 1000), e.sample(1, 1000)


VARIANTS = {
    "auto": {},
    "bitmap_atomic": dict(visited="bitmap", dedup="atomic"),
    "bitmap_warp": dict(visited="bitmap", dedup="warp"),
    # one-word keys in 32-bit quotient slots where their bits allow, else 64-bit slots
    "hash": dict(visited="hash"),
    "hash_wide": dict(visited="hash", wide_slots=True),
    "hash_load95": dict(visited="hash", hash_load_percent=95),
    "hash3": dict(visited="hash3"),
    # every layer routed through the shard buckets
    "bitmap_bucket": dict(visited="bitmap", dedup="bucket", bucket_min_work=1),
    # no bucket slack: first attempts overflow and are redone with exact counts
    "bitmap_bucket_tight": dict(visited="bitmap", dedup="bucket", bucket_min_work=1, bucket_margin=0),
    # every generator applied, no parent-edge skip
    "bitmap_bucket_noskip": dict(visited="bitmap", dedup="bucket", bucket_min_work=1, parent_skip=False),
    "hash3_noskip": dict(visited="hash3", parent_skip=False),
    # sort-unique tiles of children before the visited test
    "bitmap_sort": dict(visited="bitmap", dedup="sort"),
    "bitmap_sort_noskip": dict(visited="bitmap", dedup="sort", parent_skip=False),
    "hash_sort": dict(visited="hash", dedup="sort"),
    "hash3_sort": dict(visited="hash3", dedup="sort"),
    # claim, then route the winners into a prefix-grouped frontier, every layer
    "bitmap_grouped": dict(visited="bitmap", dedup="grouped", bucket_min_work=1),
    # no group margin: most winners of the first grouped layers go to the spill region
    "bitmap_grouped_tight": dict(visited="bitmap", dedup="grouped", bucket_min_work=1, bucket_margin=0),
    "bitmap_grouped_noskip": dict(visited="bitmap", dedup="grouped", bucket_min_work=1, parent_skip=False),
    # hash with every layer routed to table regions, then inserted per region
    "hash_bucket": dict(visited="hash", dedup="bucket", bucket_min_work=1),
    "hash_bucket_tight": dict(visited="hash", dedup="bucket", bucket_min_work=1, bucket_margin=0),
    # routed layers in parent chunks (as when a layer's buckets exceed the
    # device memory), one chunk at a time; tight: chunks overflow and are redone
    "bitmap_bucket_chunked": dict(visited="bitmap", dedup="bucket", bucket_min_work=1, route_chunk=1 << 14),
    "bitmap_bucket_chunked_tight": dict(visited="bitmap", dedup="bucket", bucket_min_work=1, bucket_margin=0,
                                        route_chunk=1 << 10),
    "hash_bucket_chunked": dict(visited="hash", dedup="bucket", bucket_min_work=1, route_chunk=1 << 12),
    # host-driven layer loop instead of the one-graph device loop
    "bitmap_atomic_hostloop": dict(visited="bitmap", dedup="atomic", host_loop=True),
    "hash_hostloop": dict(visited="hash", host_loop=True),
    "hash_wide_hostloop": dict(visited="hash", wide_slots=True, host_loop=True),
}


def _applicable(case, variant):
    g = case["graph"]
    if variant.startswith("hash3"):
        return case["inverse_closed"]
    if variant.startswith("bitmap"):
        return g["action"]["kind"] == "permutation" and len(set(g["start"])) <= 16 and \
            len(g["start"]) * P.bits_for(len(set(g["start"]))) <= 64 and math.factorial(len(g["start"])) < 1 << 34
    return True


@pytest.mark.parametrize("variant", list(VARIANTS))
def test_golden_cases(exact_cases, variant):
    ran = 0
    for case in exact_cases:
        if not _applicable(case, variant):
            continue
        out = run(case["graph"], **VARIANTS[variant])
        if out is None:
            assert variant != "auto", case["name"]
            continue
        info, r, last, prev = out
        assert r.complete, (case["name"], r)
        assert r.layer_sizes == case["layer_sizes"], (case["name"], info)
        sizes = case["layer_sizes"]
        if case["last_layer"] is not None:
            if sizes[-1] <= 1000:
                assert last == case["last_layer"], case["name"]
            else:
                assert len(last) == 1000 and all(x in case["last_layer"] for x in last)
        if len(sizes) > 1 and sizes[-2] < 1000 and case["previous_layer"] is not None:
            assert prev == case["previous_layer"], case["name"]
        else:
            assert prev == []
        assert r.successors == sum(sizes) * len(case["graph"]["action"]["generators"])
        ran += 1
    assert ran >= 8


@pytest.mark.parametrize("plan", [dict(visited="bitmap", dedup="atomic"), dict(visited="hash")])
def test_device_loop_matches_host_loop(lrx_layers, plan):
    """The device loop and the host loop give the same table, edge counts and
    samples.  The device loop is one persistent cooperative launch for every
    layer (grid barriers between layers) after the seed and the start stamp;
    the host loop launches one kernel per layer."""
    g = G.permutation_graph(G.lrx_generators(10), list(range(10)))
    info, dev, last_d, prev_d = run(g, **plan)
    info_h, host, last_h, prev_h = run(g, **plan, host_loop=True)
    assert dev.layer_sizes == host.layer_sizes == lrx_layers[10]
    assert dev.successors == host.successors and dev.visited_tests == host.visited_tests
    assert last_d == last_h and prev_d == prev_h
    layers = len(lrx_layers[10])
    assert host.kernel_launches == 1 + layers
    assert dev.kernel_launches == 3
    assert len(dev.layer_seconds) == layers - 1 and all(t >= 0 for t in dev.layer_seconds)


def test_parent_skip_accounting(lrx_layers):
    """With parent-edge tags every state but the start skips one of its g
    generators; the layer tables are identical with and without the skip."""
    g = G.permutation_graph(G.lrx_generators(10), list(range(10)))
    info, skip, _, _ = run(g, visited="bitmap", dedup="bucket", bucket_min_work=1)
    info0, noskip, _, _ = run(g, visited="bitmap", dedup="bucket", bucket_min_work=1, parent_skip=False)
    assert info["parent_skip"] == 1 and info0["parent_skip"] == 0
    assert skip.layer_sizes == noskip.layer_sizes == lrx_layers[10]
    n = sum(lrx_layers[10])
    assert skip.successors == noskip.successors == 3 * n
    assert noskip.visited_tests == 3 * n and skip.visited_tests == 3 * n - (n - 1)


@pytest.mark.parametrize("variant", ["auto", "bitmap_atomic", "bitmap_warp", "hash", "hash3", "bitmap_bucket",
                                     "bitmap_bucket_tight", "bitmap_bucket_noskip", "hash3_noskip", "bitmap_sort",
                                     "bitmap_sort_noskip", "hash_sort", "hash3_sort", "bitmap_grouped",
                                     "bitmap_grouped_tight", "bitmap_grouped_noskip", "hash_bucket",
                                     "hash_bucket_tight", "bitmap_bucket_chunked", "bitmap_bucket_chunked_tight",
                                     "hash_bucket_chunked"])
def test_lrx_small(lrx_layers, variant):
    redo = 0
    for n in range(3, 12):
        out = run(G.permutation_graph(G.lrx_generators(n), list(range(n))), **VARIANTS[variant])
        assert out is not None
        assert out[1].layer_sizes == lrx_layers[n], (n, variant)
        redo += out[1].redo_layers
    if variant in ("bitmap_bucket_tight", "hash_bucket_tight", "bitmap_bucket_chunked_tight"):
        assert redo > 0  # the exact redo path ran and changed nothing


def test_s11_hash_plans_quotient_slots(lrx_layers):
    """S11's 44-bit keys fit 32-bit quotient slots: 2^27 slots (512 MB) at the
    default 50 % threshold instead of 2^27 64-bit slots (1 GB); same table."""
    g = G.permutation_graph(G.lrx_generators(11), list(range(11)))
    q = run(g, visited="hash")
    w = run(g, visited="hash", wide_slots=True)
    assert q[0]["table_slot_bytes"] == 4 and q[0]["table_slots"] == 1 << 27 and q[0]["hash_load_percent"] == 50
    assert w[0]["table_slot_bytes"] == 8 and w[0]["table_slots"] == 1 << 27
    assert q[1].layer_sizes == w[1].layer_sizes == lrx_layers[11]
    assert q[2] == w[2] and q[3] == w[3]


@pytest.mark.parametrize("variant", ["bitmap_warp", "bitmap_atomic", "bitmap_bucket_default", "bitmap_grouped_default"])
def test_lrx13_full_table(lrx13, variant):
    defaults = {"bitmap_bucket_default": dict(visited="bitmap", dedup="bucket"),
                "bitmap_grouped_default": dict(visited="bitmap", dedup="grouped")}
    plan = VARIANTS.get(variant) or defaults[variant]
    out = run(G.permutation_graph(G.lrx_generators(13), list(range(13))), **plan)
    info, r, last, prev = out
    assert info["visited"] == "bitmap"
    assert r.layer_sizes == lrx13
    # The deepest layer of S13 LRX is a single state; the one before holds 3.
    assert len(last) == 1 and len(prev) == 3 and len(set(map(tuple, prev))) == 3
    assert sorted(last[0]) == list(range(13))


@pytest.mark.parametrize("n,dedup", [(12, "bucket"), (13, "bucket"), (12, "grouped"), (13, "grouped")])
def test_coxeter_bucketed(n, dedup):
    out = run(G.permutation_graph(G.coxeter_generators(n), list(range(n))), visited="bitmap", dedup=dedup)
    assert out[1].layer_sizes == G.coxeter_layers(n)
    # The deepest Coxeter layer is the single longest element (the reversal).
    assert out[2] == [list(range(n))[::-1]]


@pytest.mark.parametrize("n", [9, 10, 11])
@pytest.mark.parametrize("full_rank", [False, True])
def test_coxeter_grouped_incremental_rank(n, full_rank):
    """Adjacent transpositions: grouped layers derive each child's rank from
    its parent's Lehmer digits (or rank from scratch with full_rank); both give
    the Mahonian layer table, from the first layer on."""
    g = G.permutation_graph(G.coxeter_generators(n), list(range(n)))
    out = run(g, visited="bitmap", dedup="grouped", bucket_min_work=1, full_rank=full_rank)
    assert out[1].layer_sizes == G.coxeter_layers(n)
    assert out[2] == [list(range(n))[::-1]]


@pytest.mark.parametrize("n", [10, 11])
def test_lrx_three_bank_hash(n):
    """S10 / S11 LRX through the three-layer banks against the reference's own
    packed-search tables (fixture)."""
    sizes_ref = golden("lrx_layers.json")["layers"][str(n)]
    out = run(G.permutation_graph(G.lrx_generators(n), list(range(n))), visited="hash3")
    assert out[0]["history_layers"] == 3
    assert out[1].layer_sizes == sizes_ref


@pytest.mark.parametrize("n,variant", [(10, "hash3"), (11, "bitmap_warp"), (13, "bitmap_warp")])
def test_coxeter(n, variant):
    out = run(G.permutation_graph(G.coxeter_generators(n), list(range(n))), **VARIANTS[variant])
    assert out[1].layer_sizes == G.coxeter_layers(n)


@pytest.mark.parametrize("closed", [False, True])
def test_random_sweep_instances(closed):
    for i in range(12):
        g = G.sweep_instance(i, closed)
        n = len(g["start"])
        ref, last_ref, _ = P.packed_bfs(g["action"]["generators"], g["start"], sample=1 << 22)
        for variant in ("auto", "hash", "bitmap_warp", "bitmap_sort", "hash_sort", "bitmap_grouped_tight",
                        "hash_bucket") + \
                (("hash3", "hash3_sort") if closed else ()):
            out = run(g, **VARIANTS[variant])
            assert out[1].layer_sizes == ref, (i, variant, n)
            if ref[-1] <= 1000:
                assert out[2] == last_ref, (i, variant)


def test_layer_limit_deadline_and_cancel():
    import ctypes
    from multigpubfs_b200 import GraphDefinition
    g = GraphDefinition.permutation(G.lrx_generators(9), list(range(9)))
    with _engine()(g) as e:
        e.plan()
        r = e.run(max_layers=5)
        assert not r.complete and r.reason == "PROFILE_LAYER_LIMIT" and len(r.layer_sizes) == 5
        flag = ctypes.c_int32(1)
        r = e.run(cancel_flag=flag)
        assert not r.complete and r.reason == "CANCELLED" and r.layer_sizes == [1]
        r = e.run(on_layer=lambda depth, size, secs: depth >= 3)
        assert r.reason == "CANCELLED" and len(r.layer_sizes) == 4
        r = e.run()
        assert r.complete and sum(r.layer_sizes) == math.factorial(9)


def test_capacity_overflow_is_resource_not_wrong_answer():
    from multigpubfs_b200 import GraphDefinition
    g = GraphDefinition.permutation(G.lrx_generators(8), list(range(8)))
    with _engine()(g) as e:
        e.plan(visited="bitmap", capacity=100)
        r = e.run()
        assert not r.complete and r.reason == "RESOURCE" and "FRONTIER_OVERFLOW" in r.fatal_names
        # every completed layer is still exact
        ref = G.layer_sizes(G.permutation_graph(G.lrx_generators(8), list(range(8))))
        assert r.layer_sizes == ref[:len(r.layer_sizes)]


def test_run_graph_end_to_end(tmp_path, lrx_layers):
    import hashlib
    import json
    from multigpubfs_b200 import GraphDefinition, run_graph
    g = GraphDefinition.permutation(G.lrx_generators(8), list(range(8)))
    report = run_graph(g, tmp_path / "out")
    assert report["status"] == "COMPLETE" and report["reason"] == "FRONTIER_EXHAUSTED"
    assert report["layer_sizes"] == lrx_layers[8]
    assert report["graph_digest"] == g.digest()
    raw = (tmp_path / "out" / "states.json").read_bytes()
    assert hashlib.sha256(raw).hexdigest() == report["states_sha256"]
    states = json.loads(raw)
    assert states["schema"] == 2 and states["state_encoding"] == "signed_int64_vectors"
    exact = G.exact_layers(G.permutation_graph(G.lrx_generators(8), list(range(8))), 1 << 20)
    assert states["current"] == exact[-1]
    assert states["previous_small"] == exact[-2]
    assert len(report["layer_seconds"]) == len(report["layer_sizes"]) - 1


def test_bfs_through_cayleypy_boundary(tmp_path, monkeypatch):
    import sys
    import types
    from types import SimpleNamespace
    import multigpubfs_b200 as mg

    class CayleyGraph:
        def __init__(self, definition):
            self.definition = definition

        def bfs(self, **kwargs):
            raise AssertionError("original bfs must not run")

    module = types.ModuleType("cayleypy")
    module.CayleyGraph = CayleyGraph
    monkeypatch.setitem(sys.modules, "cayleypy", module)
    gens = G.lrx_generators(5)
    graph = CayleyGraph(SimpleNamespace(generators_type=SimpleNamespace(name="PERMUTATION"),
                                        generators_permutations=gens, central_state=list(range(5)), name="lrx-5",
                                        generator_names=["L", "R", "X"]))
    mg.enable_native(mg.NativeOptions(output_root=tmp_path))
    try:
        result = graph.bfs()
    finally:
        mg.disable_native()
    exact = G.exact_layers(G.permutation_graph(gens, list(range(5))), 1000)
    assert result.layer_sizes == [len(x) for x in exact]
    assert result.diameter() == len(exact) - 1
    assert result.last_layer().tolist() == exact[-1]


@pytest.mark.parametrize("ppt", [1, 2, 4])
@pytest.mark.parametrize("plan", [dict(visited="bitmap", dedup="atomic"), dict(visited="bitmap", dedup="warp"),
                                  dict(visited="hash"), dict(visited="hash", wide_slots=True),
                                  dict(visited="bitmap", dedup="atomic", host_loop=True)])
def test_every_parents_per_thread_shape_is_exact(ppt, plan):
    """The fused kernels' tile shapes (1, 2 or 4 parents per thread), device
    and host loops, on LRX S10 and Coxeter S9 against the reference's tables."""
    from multigpubfs_b200 import GraphDefinition
    from multigpubfs_b200.engine import NativeGraph
    for gens, n, expect in ((G.lrx_generators(10), 10, golden("lrx_layers.json")["layers"]["10"]),
                            (G.coxeter_generators(9), 9, G.coxeter_layers(9))):
        with NativeGraph(GraphDefinition.permutation(gens, list(range(n)))) as e:
            info = e.plan(parents_per_thread=ppt, **plan)
            assert info["parents_per_thread"] == ppt
            assert e.run().layer_sizes == expect, (n, ppt, plan)


@pytest.mark.parametrize("shape", [dict(group_chunk=256), dict(group_chunk=1 << 20), dict(group_chunk=2048, blocks_per_sm=4),
                                   dict(blocks_per_sm=8), dict(bucket_margin=0)])
def test_grouped_shapes_are_exact(shape):
    """Every grouped layer (bucket_min_work 1) under the tuner's shapes, on
    S11 LRX against the reference's table."""
    from multigpubfs_b200 import GraphDefinition
    from multigpubfs_b200.engine import NativeGraph
    with NativeGraph(GraphDefinition.permutation(G.lrx_generators(11), list(range(11)))) as e:
        info = e.plan(visited="bitmap", dedup="grouped", bucket_min_work=1, **shape)
        assert info["dedup"] == "grouped"
        assert e.run().layer_sizes == golden("lrx_layers.json")["layers"]["11"]


@pytest.mark.parametrize("blocks", [1, 2, 8, 16])
def test_fused_blocks_per_sm_are_exact(blocks):
    """Resident-block shapes of the fused bitmap and hash kernels on S10
    Coxeter against the Mahonian layer sizes."""
    from multigpubfs_b200 import GraphDefinition
    from multigpubfs_b200.engine import NativeGraph
    for plan in (dict(visited="bitmap", dedup="atomic"), dict(visited="hash")):
        with NativeGraph(GraphDefinition.permutation(G.coxeter_generators(10), list(range(10)))) as e:
            e.plan(blocks_per_sm=blocks, **plan)
            assert e.run().layer_sizes == G.coxeter_layers(10), plan


def test_route_chunk_must_be_a_multiple_of_1024():
    from multigpubfs_b200 import GraphDefinition
    from multigpubfs_b200.native import NativeError
    g = GraphDefinition.from_dict(G.permutation_graph(G.lrx_generators(8), list(range(8))))
    with _engine()(g) as e:
        with pytest.raises(NativeError) as exc:
            e.plan(visited="bitmap", dedup="bucket", route_chunk=1000)
        assert exc.value.code == 1
        e.plan(visited="bitmap", dedup="bucket", bucket_min_work=1, route_chunk=2048)
        assert e.run().layer_sizes == G.layer_sizes(G.permutation_graph(G.lrx_generators(8), list(range(8))))


@pytest.mark.parametrize("dedup", ["grouped", "bucket"])
def test_s14_lrx_first_layers_match_the_oracle(dedup):
    """Degree 14, every layer from the first through the large-bitmap layers:
    grouped with 4-symbol groups (24,024 regions of 10! bits), or owner-routed
    in 65,536-parent chunks; the first 24 layers equal the oracle's."""
    from multigpubfs_b200 import GraphDefinition
    n = 14
    gens = G.lrx_generators(n)
    expect, _, _ = P.packed_bfs(gens, list(range(n)), use_bitmap=False, max_layers=24, partial=True,
                                max_states=1 << 27)
    g = GraphDefinition.from_dict(G.permutation_graph(gens, list(range(n))))
    plan = dict(visited="bitmap", dedup=dedup, bucket_min_work=1)
    if dedup == "bucket":
        plan["route_chunk"] = 1 << 16
    with _engine()(g) as e:
        info = e.plan(**plan)
        r = e.run(max_layers=24)
    assert info["shards"] == (24024 if dedup == "grouped" else 182)
    assert len(expect) == 24 and r.layer_sizes == expect


_S14_CHILD = """
import json, sys
sys.path.insert(0, sys.argv[1])
from multigpubfs_b200 import GraphDefinition
from multigpubfs_b200.engine import NativeGraph
n = 14
left = [(i + 1) % n for i in range(n)]
right = [(i - 1) % n for i in range(n)]
x = list(range(n)); x[0], x[1] = 1, 0
g = GraphDefinition.permutation([left, right, x], list(range(n)))
out = {}
for dedup in ("auto", "bucket"):
    print("dedup", dedup, file=sys.stderr, flush=True)
    with NativeGraph(g, 0) as e:
        info = e.plan(visited="bitmap", dedup=dedup)
        r = e.run()
    out[dedup] = [info["dedup"], r.layer_sizes]
print(json.dumps(out))
"""


def test_s14_lrx_full_bfs_on_one_gpu():
    """The whole S14 LRX BFS (14! = 87,178,291,200 states, 4.6e9 in the peak
    layer) under the default plan (grouped layers with 24,024 prefix groups and
    a memory-bounded spill) and owner-routed in parent chunks sized by the free
    memory: both settle 14! states, agree layer by layer, and start with the
    reference's first 24 layers.  It needs about 130 GB of the device, so it
    runs in a fresh process, beside none of the earlier tests' buffers."""
    import json
    import subprocess
    import sys
    from pathlib import Path

    import torch
    from multigpubfs_b200 import native
    n = 14
    fx = golden("lrx14_prefix.json")
    root = str(Path(__file__).resolve().parents[1])
    # This process's cached buffers and tensors go back to the device first.
    native.trim_memory(0)
    torch.cuda.empty_cache()
    free, total = torch.cuda.mem_get_info()
    child = subprocess.run([sys.executable, "-c", _S14_CHILD, root], capture_output=True, text=True, timeout=600)
    assert child.returncode == 0, f"free before: {free / 2**30:.1f} of {total / 2**30:.1f} GiB\n" + child.stderr[-2000:]
    tables = json.loads(child.stdout.strip().splitlines()[-1])
    assert tables["auto"][0] == "grouped" and tables["bucket"][0] == "bucket"
    sizes = tables["auto"][1]
    assert sum(sizes) == math.factorial(n) and sizes[:24] == fx["layers"]
    assert tables["bucket"][1] == sizes


def test_routed_layers_under_a_memory_budget_keep_the_table():
    """S12 Coxeter (11 generators, the certified Mahonian table) routed on a
    device budget of 1.2 GB: its peak layer's buckets alone would need about
    2.6 GB. Its routed layers therefore go in parent chunks sized by the free
    memory. That takes more route/accept launches than the same BFS
    unbounded, and gives the certified table."""
    import torch
    from multigpubfs_b200 import GraphDefinition, native
    n = 12
    g = GraphDefinition.from_dict(G.permutation_graph(G.coxeter_generators(n), list(range(n))))
    expect = G.coxeter_layers(n)
    native.trim_memory(0)
    torch.cuda.empty_cache()
    with _engine()(g) as e:
        e.plan(visited="bitmap", dedup="bucket")
        free = e.run()
    native.trim_memory(0)
    free_bytes, _ = torch.cuda.mem_get_info()
    with _engine()(g) as e:
        e.plan(visited="bitmap", dedup="bucket", reserve_bytes=free_bytes - (1200 << 20))
        bounded = e.run()
    assert free.layer_sizes == expect and bounded.layer_sizes == expect
    assert bounded.kernel_launches > free.kernel_launches
