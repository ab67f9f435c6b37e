"""Layer archive and checkpoint/resume through the C ABI: archived layers
partition the orbit and match the oracle's table; a BFS stopped at a layer
limit, checkpointed and resumed in a fresh handle ends with the table and
samples of an uninterrupted run; a checkpoint of another graph, or a corrupted
one, is refused."""
import math

import pytest

from oracle import graph_oracle as G
from oracle import packed_oracle as P
from tests.conftest import golden

pytestmark = pytest.mark.gpu


def _graph(gens, start):
    from multigpubfs_b200 import GraphDefinition
    return GraphDefinition.from_dict(G.permutation_graph(gens, start))


def test_archived_layers_partition_the_orbit(tmp_path):
    from multigpubfs_b200 import archive
    g = _graph(G.lrx_generators(8), list(range(8)))
    result, manifest = archive.run_archived(g, tmp_path / "a")
    expect = golden("lrx_layers.json")["layers"]["8"]
    assert result.complete and result.layer_sizes == expect
    assert manifest["status"] == "COMPLETE" and manifest["last_completed_layer"] == len(expect) - 1
    assert [f["states"] for f in manifest["files"]] == expect
    seen = set()
    for d in range(len(expect)):
        rows = archive.decode(archive.read_layer(tmp_path / "a", d), manifest["packing"], 8)
        assert len(rows) == expect[d]
        seen.update(tuple(r) for r in rows)
    assert len(seen) == math.factorial(8)


def test_archive_retention_policies(tmp_path):
    from multigpubfs_b200 import archive
    g = _graph(G.lrx_generators(8), list(range(8)))
    expect = golden("lrx_layers.json")["layers"]["8"]
    _, fixed = archive.run_archived(g, tmp_path / "fixed", retained_layers=3)
    assert [f["depth"] for f in fixed["files"]] == [len(expect) - 3, len(expect) - 2, len(expect) - 1]
    assert sorted(p.name for p in (tmp_path / "fixed").glob("layer-*.bin")) == [f["path"] for f in fixed["files"]]
    _, compact = archive.run_archived(g, tmp_path / "compact", policy=archive.COMPACT_POLICY)
    kept = [f["depth"] for f in compact["files"]]
    assert kept == [d for d, s in enumerate(expect) if s <= 1000 or d == len(expect) - 1]
    with pytest.raises(KeyError):
        archive.read_layer(tmp_path / "compact", max(range(len(expect)), key=lambda d: expect[d]))


CASES = {
    "bitmap_device_loop": (G.lrx_generators(11), list(range(11)), dict(visited="bitmap", dedup="atomic"), 25),
    "hash_quotient": (G.lrx_generators(11), list(range(11)), dict(visited="hash"), 30),
    "bitmap_grouped": (G.lrx_generators(10), list(range(10)), dict(visited="bitmap", dedup="grouped",
                                                                   bucket_min_work=1), 20),
    "bitmap_bucket": (G.coxeter_generators(9), list(range(9)), dict(visited="bitmap", dedup="bucket",
                                                                    bucket_min_work=1), 12),
    "product_domain": ([[1, 2, 3, 4, 5, 0, 6, 7, 8, 9], [5, 0, 1, 2, 3, 4, 6, 7, 8, 9],
                        [0, 1, 2, 3, 4, 5, 7, 6, 9, 8], [0, 1, 2, 3, 4, 5, 8, 9, 6, 7]],
                       [0, 0, 1, 1, 2, 3, 4, 4, 5, 6], dict(visited="bitmap"), 3),
}


@pytest.mark.parametrize("case", sorted(CASES))
def test_checkpoint_resume_matches_an_uninterrupted_run(tmp_path, case):
    from multigpubfs_b200 import archive
    from multigpubfs_b200.engine import NativeGraph
    gens, start, plan, stop = CASES[case]
    g = _graph(gens, start)
    with NativeGraph(g) as e:
        e.plan(**plan)
        full = e.run()
        last, prev = e.sample(0, 1000), e.sample(1, 1000)
    assert full.complete
    with NativeGraph(g) as e:
        e.plan(**plan)
        part = e.run(max_layers=stop)
        assert not part.complete and len(part.layer_sizes) == stop
        manifest = archive.save_checkpoint(e, tmp_path / case, part)
    assert manifest["layer_sizes"] == full.layer_sizes[:stop]
    with NativeGraph(g) as e:
        info = e.plan(**plan)
        archive.load_checkpoint(e, tmp_path / case)
        rest = e.run()
        assert rest.complete and rest.layer_sizes == full.layer_sizes
        assert e.sample(0, 1000) == last and e.sample(1, 1000) == prev
    if case == "product_domain":
        assert info["rank_components"] > 1


def test_checkpoint_of_another_graph_or_corrupted_is_refused(tmp_path):
    from multigpubfs_b200 import archive
    from multigpubfs_b200.engine import NativeGraph
    from multigpubfs_b200.native import NativeError
    g = _graph(G.lrx_generators(9), list(range(9)))
    with NativeGraph(g) as e:
        e.plan(visited="bitmap")
        part = e.run(max_layers=10)
        archive.save_checkpoint(e, tmp_path / "ck", part)
        e.checkpoint(tmp_path / "raw.bin")
    other = _graph(G.coxeter_generators(9), list(range(9)))
    with NativeGraph(other) as e:
        e.plan(visited="bitmap")
        with pytest.raises(ValueError, match="CHECKPOINT_GRAPH_MISMATCH"):
            archive.load_checkpoint(e, tmp_path / "ck")
        with pytest.raises(NativeError) as info:  # the library checks the generators itself
            e.resume(tmp_path / "raw.bin")
        assert info.value.code == 1
    data = bytearray((tmp_path / "ck" / "checkpoint.bin").read_bytes())
    data[-1] ^= 0xFF
    (tmp_path / "ck" / "checkpoint.bin").write_bytes(bytes(data))
    with NativeGraph(g) as e:
        e.plan(visited="bitmap")
        with pytest.raises(ValueError, match="CHECKPOINT_CHECKSUM"):
            archive.load_checkpoint(e, tmp_path / "ck")
