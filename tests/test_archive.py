"""Layer archive host logic on CPU (multigpubfs_b200.archive): packing and
decoding of archived words, the manifest written after every layer, the two
retention policies of the reference's tail archive
(scripts/bfs_tail_archive.py) and checksum verification of a read."""
import json

import numpy as np
import pytest

from multigpubfs_b200 import archive
from multigpubfs_b200.graph_definition import GraphDefinition
from oracle import graph_oracle as G


def _graph(n=6):
    return GraphDefinition.permutation(G.lrx_generators(n), list(range(n)))


def _layers(n=6):
    return G.exact_layers(G.permutation_graph(G.lrx_generators(n), list(range(n))), 1 << 20)


def _words(layer, pack):
    out = []
    for s in layer:
        w = 0
        for i, v in enumerate(s):
            w |= pack["labels"].index(v) << (pack["bits_per_symbol"] * i)
        out.append(w)
    return np.array(out, dtype=np.uint64)


def test_packing_round_trips_states():
    g = GraphDefinition.permutation(G.lrx_generators(5), [40, 10, 30, 20, 50])
    pack = archive.packing(g)
    assert pack["labels"] == [10, 20, 30, 40, 50] and pack["bits_per_symbol"] == 4
    states = [[40, 10, 30, 20, 50], [10, 20, 30, 40, 50], [50, 40, 30, 20, 10]]
    assert archive.decode(_words(states, pack), pack, 5) == states


def test_every_layer_is_archived_with_its_checksum(tmp_path):
    g, layers = _graph(), _layers()
    a = archive.LayerArchive(tmp_path / "a", g)
    pack = archive.packing(g)
    for d, layer in enumerate(layers):
        a.layer(d, _words(layer, pack), 0.001 * d)
        manifest = json.loads((tmp_path / "a" / "manifest.json").read_text())
        assert manifest["last_completed_layer"] == d and manifest["status"] == "INCOMPLETE"
    done = a.close(True, "FRONTIER_EXHAUSTED")
    assert done["status"] == "COMPLETE" and [f["states"] for f in done["files"]] == [len(x) for x in layers]
    for d, layer in enumerate(layers):
        got = archive.decode(archive.read_layer(tmp_path / "a", d), pack, 6)
        assert sorted(map(tuple, got)) == sorted(map(tuple, layer))
    with pytest.raises(ValueError, match="ARCHIVE_NONCONTIGUOUS_DEPTH"):
        a.layer(len(layers) + 1, np.zeros(1, dtype=np.uint64), 0.0)


def test_retention_policies_keep_the_reference_layers(tmp_path):
    g, layers = _graph(7), _layers(7)
    pack = archive.packing(g)
    fixed = archive.LayerArchive(tmp_path / "fixed", g, retained_layers=2)
    compact = archive.LayerArchive(tmp_path / "compact", g, policy=archive.COMPACT_POLICY)
    for d, layer in enumerate(layers):
        fixed.layer(d, _words(layer, pack), 0.0)
        compact.layer(d, _words(layer, pack), 0.0)
    last = len(layers) - 1
    assert [f["depth"] for f in fixed.files] == [last - 1, last]
    assert sorted(p.name for p in (tmp_path / "fixed").glob("layer-*.bin")) == [f["path"] for f in fixed.files]
    assert [f["depth"] for f in compact.files] == [d for d, x in enumerate(layers) if len(x) <= 1000 or d == last]


def test_corrupted_layer_is_refused(tmp_path):
    g, layers = _graph(), _layers()
    pack = archive.packing(g)
    a = archive.LayerArchive(tmp_path / "a", g)
    for d, layer in enumerate(layers):
        a.layer(d, _words(layer, pack), 0.0)
    path = tmp_path / "a" / "layer-000003.bin"
    data = bytearray(path.read_bytes())
    data[0] ^= 1
    path.write_bytes(bytes(data))
    with pytest.raises(ValueError, match="ARCHIVE_CHECKSUM"):
        archive.read_layer(tmp_path / "a", 3)


def test_archive_arguments_are_checked(tmp_path):
    with pytest.raises(ValueError, match="ARCHIVE_RETENTION"):
        archive.LayerArchive(tmp_path / "x", _graph(), retained_layers=0)
    with pytest.raises(ValueError, match="ARCHIVE_POLICY"):
        archive.LayerArchive(tmp_path / "y", _graph(), policy="keep_everything_twice")
    m = GraphDefinition.matrix(1, 1, [([2], 7)], [3])
    with pytest.raises(ValueError, match="ARCHIVE_REQUIRES_PACKED_STATES"):
        archive.LayerArchive(tmp_path / "z", m)
    archive.LayerArchive(tmp_path / "w", _graph())
    with pytest.raises(FileExistsError):
        archive.LayerArchive(tmp_path / "w", _graph())
