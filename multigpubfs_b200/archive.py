"""Layer archive and checkpoint/resume of a single-graph BFS.

Layer archive (the role of the reference's tail archive,
scripts/bfs_tail_archive.py): every completed layer is written as one file of
packed states (little-endian uint64 words, symbol i in bits 4i.. of its dense
code, parent-edge tags removed) with its SHA-256 in manifest.json, which is
replaced atomically after each layer, so a reader always sees whole layers.
Retention: all layers, the last `retained_layers`, or the reference's
"last_complete_small_1000" policy (the deepest layer plus every layer of at
most 1000 states).

Checkpoint / resume (beyond the reference, whose archive restarts a search
from scratch): `save_checkpoint` writes the engine's state between layers
(mgbfs2_checkpoint_write) with a manifest holding the graph digest, the layer
table and the file's SHA-256; `load_checkpoint` verifies both before handing
the file to mgbfs2_checkpoint_resume, and the next run() goes on from there.
"""
from __future__ import annotations

import hashlib
import json
import os
from pathlib import Path

from .engine import NativeGraph
from .graph_definition import GraphDefinition

ARCHIVE_SCHEMA = 1
CHECKPOINT_SCHEMA = 1
COMPACT_POLICY = "last_complete_small_1000"


def _atomic_json(path: Path, value) -> None:
    tmp = path.with_suffix(".tmp")
    with tmp.open("w", encoding="utf-8") as f:
        json.dump(value, f, indent=1, sort_keys=True)
        f.write("\n")
        f.flush()
        os.fsync(f.fileno())
    os.replace(tmp, path)


def _sha256_file(path: Path) -> str:
    h = hashlib.sha256()
    with path.open("rb") as f:
        for chunk in iter(lambda: f.read(8 << 20), b""):
            h.update(chunk)
    return h.hexdigest()


def packing(graph: GraphDefinition) -> dict:
    """How archived words decode: the dense code of the label at position i
    sits in bits [b*i, b*i + b); codes number the distinct start labels in
    ascending order."""
    labels = sorted(set(graph.start))
    bits = 4
    while bits < 32 and (1 << bits) < len(labels):
        bits *= 2
    return {"bits_per_symbol": bits, "bytes_per_state": 8, "byte_order": "little",
            "symbol_order": "symbol i in bits [bits_per_symbol*i, bits_per_symbol*(i+1))", "labels": labels}


def decode(words, pack: dict, n: int):
    """Archived words -> label rows."""
    b, labels = pack["bits_per_symbol"], pack["labels"]
    mask = (1 << b) - 1
    return [[labels[(int(w) >> (b * i)) & mask] for i in range(n)] for w in words]


class LayerArchive:
    """Writes the layers of one BFS under `root` (which must not exist)."""

    def __init__(self, root, graph: GraphDefinition, *, retained_layers: int | None = None,
                 policy: str | None = None):
        if graph.action["kind"] != "permutation":
            raise ValueError("ARCHIVE_REQUIRES_PACKED_STATES")
        if retained_layers is not None and (type(retained_layers) is not int or retained_layers < 1):
            raise ValueError("ARCHIVE_RETENTION")
        if policy not in (None, COMPACT_POLICY):
            raise ValueError("ARCHIVE_POLICY")
        self.root = Path(root)
        self.root.mkdir(parents=True, exist_ok=False)
        self.retained_layers, self.policy = retained_layers, policy
        self.files = []
        self.manifest = {"schema": ARCHIVE_SCHEMA, "status": "INCOMPLETE", "stop_reason": "running",
                         "last_completed_layer": -1, "graph_digest": graph.digest(), "graph": graph.to_dict(),
                         "packing": packing(graph), "layers": [], "files": []}
        if policy:
            self.manifest["retention"] = {"policy": policy}
        elif retained_layers:
            self.manifest["retention"] = {"policy": "fixed_whole_layers", "layers": retained_layers}
        _atomic_json(self.root / "manifest.json", self.manifest)

    def layer(self, depth: int, words, seconds: float) -> None:
        """Commits layer `depth` (its packed words, a numpy uint64 array)."""
        if depth != len(self.manifest["layers"]):
            raise ValueError("ARCHIVE_NONCONTIGUOUS_DEPTH")
        path = self.root / f"layer-{depth:06d}.bin"
        tmp = path.with_suffix(".tmp")
        data = words.astype("<u8").tobytes()
        with tmp.open("wb") as f:
            f.write(data)
            f.flush()
            os.fsync(f.fileno())
        os.replace(tmp, path)
        self.files.append({"depth": depth, "states": len(words), "bytes": len(data),
                           "sha256": hashlib.sha256(data).hexdigest(), "path": path.name})
        self.manifest["layers"].append({"depth": depth, "states": len(words), "seconds": float(seconds)})
        self.manifest["last_completed_layer"] = depth
        self._retain()
        self.manifest["files"] = list(self.files)
        _atomic_json(self.root / "manifest.json", self.manifest)

    def _retain(self) -> None:
        if self.policy == COMPACT_POLICY:
            deepest = self.files[-1]["depth"]
            keep = [f for f in self.files if f["depth"] == deepest or f["states"] <= 1000]
        elif self.retained_layers:
            keep = self.files[-self.retained_layers:]
        else:
            return
        for f in self.files:
            if f not in keep:
                (self.root / f["path"]).unlink()
        self.files = keep

    def close(self, complete: bool, reason: str) -> dict:
        self.manifest["status"] = "COMPLETE" if complete else "INCOMPLETE"
        self.manifest["stop_reason"] = reason
        _atomic_json(self.root / "manifest.json", self.manifest)
        return self.manifest


def run_archived(graph: GraphDefinition, root, device: int = 0, *, retained_layers=None, policy=None,
                 max_layers=None, **plan) -> tuple:
    """Exact BFS of `graph` with every completed layer archived under `root`.
    Returns (RunResult, manifest).  The layers come from the engine's layer
    callback (the host-driven loop) through mgbfs2_frontier_words."""
    archive = LayerArchive(root, graph, retained_layers=retained_layers, policy=policy)
    with NativeGraph(graph, device) as engine:
        engine.plan(**plan)
        pack = packing(graph)
        start = 0
        for i, v in enumerate(graph.start):
            start |= pack["labels"].index(v) << (pack["bits_per_symbol"] * i)
        import numpy as np
        archive.layer(0, np.array([start], dtype=np.uint64), 0.0)
        failures = []

        def on_layer(depth, size, seconds):
            try:
                words = engine.frontier_words()
                if len(words) != size:
                    raise RuntimeError("ARCHIVE_LAYER_SIZE")
                archive.layer(depth, words, seconds)
                return False
            except Exception as exc:  # noqa: BLE001 - stop the run, re-raised below
                failures.append(exc)
                return True
        result = engine.run(on_layer=on_layer, max_layers=max_layers)
    if failures:
        archive.close(False, "ARCHIVE_WRITE_FAILED")
        raise failures[0]
    return result, archive.close(result.complete, result.reason)


def read_layer(root, depth: int):
    """The archived words of one layer, verified against the manifest."""
    import numpy as np
    root = Path(root)
    manifest = json.loads((root / "manifest.json").read_text())
    entry = next((f for f in manifest["files"] if f["depth"] == depth), None)
    if entry is None:
        raise KeyError(f"layer {depth} not retained")
    data = (root / entry["path"]).read_bytes()
    if len(data) != entry["bytes"] or hashlib.sha256(data).hexdigest() != entry["sha256"]:
        raise ValueError("ARCHIVE_CHECKSUM")
    return np.frombuffer(data, dtype="<u8")


def save_checkpoint(engine: NativeGraph, root, result) -> dict:
    """Writes the engine's state after `result = engine.run(...)` to `root`
    (checkpoint.bin and checkpoint.json) and returns the manifest."""
    root = Path(root)
    root.mkdir(parents=True, exist_ok=True)
    path = root / "checkpoint.bin"
    engine.checkpoint(path)
    manifest = {"schema": CHECKPOINT_SCHEMA, "graph_digest": engine.graph.digest(),
                "layer_sizes": list(result.layer_sizes), "complete": bool(result.complete),
                "reason": result.reason, "plan": engine.plan_info, "bytes": path.stat().st_size,
                "sha256": _sha256_file(path), "path": path.name}
    _atomic_json(root / "checkpoint.json", manifest)
    return manifest


def load_checkpoint(engine: NativeGraph, root) -> dict:
    """Verifies `root`'s checkpoint against the engine's graph and the file's
    checksum, then loads it (the engine must be planned with the same visited
    structure); the next engine.run() goes on from its depth."""
    root = Path(root)
    manifest = json.loads((root / "checkpoint.json").read_text())
    if manifest.get("schema") != CHECKPOINT_SCHEMA:
        raise ValueError("CHECKPOINT_SCHEMA")
    if manifest["graph_digest"] != engine.graph.digest():
        raise ValueError("CHECKPOINT_GRAPH_MISMATCH")
    path = root / manifest["path"]
    if path.stat().st_size != manifest["bytes"] or _sha256_file(path) != manifest["sha256"]:
        raise ValueError("CHECKPOINT_CHECKSUM")
    engine.resume(path)
    return manifest
