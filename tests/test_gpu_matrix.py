"""Int64 matrix groups on the wide-key path at sizes where one state is often
claimed by several threads in the same layer: SL(2, p) on 2x2 matrices,
against the reference's own exact_layers tables (tests/golden/matrix_groups.json)
on repeated runs, and the group order p(p^2 - 1) beyond the fixtures."""
import pytest

from tests.conftest import golden

pytestmark = pytest.mark.gpu


def _sl2(p):
    from multigpubfs_b200 import GraphDefinition
    gens = [([1, 1, 0, 1], p), ([1, 0, 1, 1], p), ([1, p - 1, 0, 1], p), ([1, 0, p - 1, 1], p)]
    return GraphDefinition.matrix(2, 2, gens, [1, 0, 0, 1])


@pytest.mark.parametrize("case", ["sl2_mod31", "sl2_mod101"])
def test_sl2_tables_match_the_reference_on_every_run(case):
    from multigpubfs_b200 import GraphDefinition
    from multigpubfs_b200.engine import NativeGraph
    fx = golden("matrix_groups.json")["cases"][case]
    g = GraphDefinition.from_dict(fx["graph"])
    with NativeGraph(g) as e:
        e.plan()
        for _ in range(6):
            r = e.run()
            assert r.complete and r.layer_sizes == fx["layers"]


@pytest.mark.parametrize("p", [211, 251])
def test_sl2_orbit_is_the_group_order(p):
    from multigpubfs_b200.engine import NativeGraph
    with NativeGraph(_sl2(p)) as e:
        e.plan()
        for _ in range(3):
            r = e.run()
            assert r.complete and r.states == p * (p * p - 1)


def _gl2(p):
    from multigpubfs_b200 import GraphDefinition
    from multigpubfs_b200.workloads import gl2_graph
    return GraphDefinition.from_dict(gl2_graph(p))


@pytest.mark.parametrize("visited", ["bitmap", "hash", "hash3", "auto"])
def test_packed_matrices_match_the_reference_on_every_visited_set(visited):
    from multigpubfs_b200 import GraphDefinition
    from multigpubfs_b200.engine import NativeGraph
    from oracle import graph_oracle as G
    fx = golden("matrix_groups.json")["cases"]["sl2_mod31"]
    g = GraphDefinition.from_dict(fx["graph"])
    with NativeGraph(g) as e:
        info = e.plan(visited=visited)
        r = e.run()
        last = e.sample(0, 1000)
    assert info["packed"] == 1 and info["bits_per_symbol"] == 5 and info["parent_skip"] == 1
    if info["visited"] == "bitmap":
        assert info["bitmap_bits"] == 31 ** 4
    assert r.layer_sizes == fx["layers"]
    expect_last = sorted(tuple(s) for s in G.exact_layers(fx["graph"], 1 << 20)[-1])
    assert [tuple(s) for s in last] == expect_last


@pytest.mark.parametrize("p", [31, 101])
def test_gl2_orbit_is_the_group_order(p):
    from multigpubfs_b200.engine import NativeGraph
    with NativeGraph(_gl2(p)) as e:
        info = e.plan()
        r = e.run()
    assert info["packed"] == 1 and info["visited"] == "bitmap"
    assert r.complete and r.states == (p * p - 1) * (p * p - p)


def test_unpackable_matrices_stay_on_the_wide_path():
    """Coefficients whose products could leave int64 are not packed; the wide
    path keeps the reference's wrap-then-modulus."""
    from multigpubfs_b200 import GraphDefinition
    from multigpubfs_b200.engine import NativeGraph
    from oracle import graph_oracle as G
    big = 1 << 45
    gens = [([1, big, 0, 1], 1 << 20), ([1, 0, 1, 1], 1 << 20)]
    g = GraphDefinition.matrix(2, 1, gens, [1, 2])
    with NativeGraph(g) as e:
        info = e.plan()
        r = e.run(max_layers=6)
    assert info["packed"] == 0
    graph = G.matrix_graph(2, 1, gens, [1, 2])
    seen, layer, expect = {(1, 2)}, [(1, 2)], [1]
    while len(expect) < 6:
        nxt = []
        for s in layer:
            for k in range(len(gens)):
                c = tuple(G.successor(graph, list(s), k))
                if c not in seen:
                    seen.add(c)
                    nxt.append(c)
        layer = nxt
        expect.append(len(nxt))
    assert r.layer_sizes == expect


@pytest.mark.parametrize("case", ["sl2_mod31", "sl2_mod101"])
@pytest.mark.parametrize("route_chunk", [None, 1024])
def test_routed_radix_layers_match_the_reference(case, route_chunk):
    """Every layer routed by the top entry (m shards of the radix bitmap),
    then claimed shard by shard; whole layers, or 1024 parents per pass."""
    from multigpubfs_b200 import GraphDefinition
    from multigpubfs_b200.engine import NativeGraph
    fx = golden("matrix_groups.json")["cases"][case]
    with NativeGraph(GraphDefinition.from_dict(fx["graph"])) as e:
        info = e.plan(visited="bitmap", dedup="bucket", bucket_min_work=1, route_chunk=route_chunk)
        for _ in range(3):
            assert e.run().layer_sizes == fx["layers"]
    assert info["dedup"] == "bucket" and info["shards"] == int(case.split("mod")[1])


def test_large_radix_bitmaps_route_by_default():
    """GL(2,211): 1.97e9 states, a 236 MB radix bitmap (above 64 MiB, so the
    planner routes its large layers by the top entry)."""
    from multigpubfs_b200.engine import NativeGraph
    p = 211
    with NativeGraph(_gl2(p)) as e:
        info = e.plan()
        r = e.run()
    assert info["visited"] == "bitmap" and info["dedup"] == "bucket" and info["shards"] == p
    assert r.complete and r.states == (p * p - 1) * (p * p - p)


def test_packed_matrix_checkpoint_resumes_exactly(tmp_path):
    """A radix-bitmap BFS stopped at a layer limit, checkpointed and resumed in
    a fresh handle ends with the reference's table."""
    from multigpubfs_b200 import GraphDefinition, archive
    from multigpubfs_b200.engine import NativeGraph
    fx = golden("matrix_groups.json")["cases"]["sl2_mod101"]
    g = GraphDefinition.from_dict(fx["graph"])
    with NativeGraph(g) as e:
        e.plan(visited="bitmap")
        part = e.run(max_layers=12)
        assert part.layer_sizes == fx["layers"][:12]
        archive.save_checkpoint(e, tmp_path / "ck", part)
    with NativeGraph(g) as e:
        e.plan(visited="bitmap")
        archive.load_checkpoint(e, tmp_path / "ck")
        assert e.run().layer_sizes == fx["layers"]
