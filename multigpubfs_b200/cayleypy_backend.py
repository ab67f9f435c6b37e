"""Explicit, reversible CayleyPy ``graph.bfs()`` integration.

Same public surface and semantics as multigpubfs/cayleypy_backend.py:14-206
(NativeOptions, NativeBfsResult, bfs, enable_native, disable_native): the
patch is installed only by ``enable_native``; ``backend='torch'`` calls the
original; unsupported keyword values raise NotImplementedError (or call the
original under ``backend='auto'``); exactly one decoded start state; native
failures propagate and are never restarted on the CPU; a foreign replacement
of ``CayleyGraph.bfs`` raises RuntimeError.  ``run_graph`` is this package's
single-GPU engine (launch.py).
"""
from __future__ import annotations

import json
import os
import tempfile
import threading
from dataclasses import dataclass, field
from functools import wraps
from pathlib import Path

from .graph_definition import GraphDefinition, _flatten, from_cayleypy
from .launch import _normalize_segment_strategy, run_graph


@dataclass(frozen=True)
class NativeOptions:
    output_root: str | Path | None = None
    devices: tuple[int, ...] | None = None
    max_seconds: int | None = None
    autotune: bool = True
    memory_backend: str = "legacy"
    memory_preset: str = "balanced"
    segment_rows: int = 1 << 32
    segment_strategy: str = field(default_factory=lambda: os.environ.get("MGBFS_SEGMENT_STRATEGY", "atomic"))
    bitmap_owner_page: int | None = None
    planner: str = "plain"

    def __post_init__(self):
        _normalize_segment_strategy(self.segment_strategy)
        if self.memory_preset not in ("balanced", "max_capacity"):
            raise ValueError("INVALID_MEMORY_PRESET")
        if type(self.segment_rows) is not int or not 1 <= self.segment_rows <= 1 << 32:
            raise ValueError("INVALID_SEGMENT_ROWS")
        page = self.bitmap_owner_page
        if page is not None and (type(page) is not int or page < 0 or page > 1 << 20 or (page and page & (page - 1))):
            raise ValueError("INVALID_BITMAP_OWNER_PAGE")
        if page and self.memory_backend != "permutation_bitmap":
            raise ValueError("BITMAP_OWNER_PAGE_REQUIRES_BITMAP")
        if self.planner not in ("plain", "learned"):
            raise ValueError("INVALID_PLANNER")


@dataclass(frozen=True)
class NativeBfsResult:
    """Exact layer counts with compact state samples (not CayleyPy's full
    BfsResult: no retained small layers, edges, hashes or paths)."""
    bfs_completed: bool
    layer_sizes: list[int]
    graph: object
    report: dict
    output: Path
    layers: dict = field(default_factory=dict)
    layer_samples: dict = field(default_factory=dict)
    backend: str = field(default="native", init=False)

    def num_vertices(self):
        return sum(self.layer_sizes)

    def diameter(self):
        if not self.bfs_completed:
            raise RuntimeError("BFS_INCOMPLETE: only completed_depth is known")
        return self.completed_depth

    @property
    def completed_depth(self):
        return len(self.layer_sizes) - 1

    def get_layer(self, layer_id):
        if layer_id not in self.layers:
            raise KeyError("Full layer not retained; use layer_samples for compact samples")
        return self.layers[layer_id].cpu().numpy()

    def last_layer(self):
        return self.get_layer(self.completed_depth)


_LOCK = threading.RLock()
_ORIGINAL = _INSTALLED = None
_DEFAULTS = dict(max_layer_size_to_store=1000, max_layer_size_to_explore=10 ** 12, max_diameter=1000000,
                 return_all_edges=False, return_all_hashes=False, stop_condition=None, disable_batching=False)


def _unsupported(kwargs):
    for key, value in kwargs.items():
        if key == "start_states":
            continue
        if key not in _DEFAULTS or value != _DEFAULTS[key]:
            return key
    return None


def _search(original, graph, backend, options, output, kwargs):
    if backend not in ("native", "torch", "auto"):
        raise ValueError("backend must be native, torch or auto")
    if not isinstance(options, NativeOptions):
        raise TypeError("native_options must be NativeOptions")
    if backend == "torch":
        if output is not None:
            raise ValueError("output belongs to the native backend")
        return original(graph, **kwargs)
    unsupported = _unsupported(kwargs)
    if unsupported:
        if backend == "auto" and output is None:
            return original(graph, **kwargs)
        raise NotImplementedError(f"Native BFS does not support {unsupported}; use backend='torch'")
    definition = from_cayleypy(graph)
    if kwargs.get("start_states") is not None:
        start = _flatten(kwargs["start_states"])
        if len(start) != len(definition.start):
            if backend == "auto" and output is None:
                return original(graph, **kwargs)
            raise NotImplementedError("Native BFS supports a single decoded start state")
        value = json.loads(definition.to_json())
        value["start"] = start
        definition = GraphDefinition.from_dict(value)
    if output is None:
        root = Path(options.output_root or Path.cwd() / "bfs-results")
        root.mkdir(parents=True, exist_ok=True)
        output = Path(tempfile.mkdtemp(prefix="run-", dir=root)) / "result"
    output = Path(output).absolute()
    report = run_graph(definition, output, devices=options.devices, max_seconds=options.max_seconds,
                       autotune=options.autotune, memory_backend=options.memory_backend,
                       segment_rows=options.segment_rows, memory_preset=options.memory_preset,
                       segment_strategy=options.segment_strategy, bitmap_owner_page=options.bitmap_owner_page,
                       **({"planner": options.planner} if options.planner != "plain" else {}))
    import torch
    snapshot = json.loads((output / "states.json").read_text())
    sizes = report["layer_sizes"]
    samples, layers = {}, {}
    for depth, name in ((len(sizes) - 1, "current"), (len(sizes) - 2, "previous_small")):
        rows = snapshot.get(name, [])
        if depth < 0 or not rows:
            continue
        tensor = torch.tensor(rows, dtype=torch.int64)
        if definition.action["kind"] == "matrix":
            tensor = tensor.reshape(-1, definition.action["rows"], definition.action["cols"])
        samples[depth] = tensor
        if len(rows) == sizes[depth]:
            layers[depth] = tensor
    return NativeBfsResult(report["status"] == "COMPLETE", sizes, getattr(graph, "definition", graph), report,
                           output, layers, samples)


def _cayley_graph_class():
    from cayleypy import CayleyGraph
    return CayleyGraph


def bfs(graph, *, backend="native", native_options=None, output=None, **kwargs):
    """Dispatch once without modifying CayleyPy."""
    cls = _cayley_graph_class()
    with _LOCK:
        original = _ORIGINAL or cls.bfs
    return _search(original, graph, backend, native_options or NativeOptions(), output, kwargs)


def enable_native(options=None, *, default_backend="native", recovery=True):
    """Route CayleyGraph.bfs() to the native engine; importing this package has
    no side effects.  ``recovery`` is accepted for signature compatibility (the
    in-process engine leaves no native processes behind to recover)."""
    global _ORIGINAL, _INSTALLED
    cls = _cayley_graph_class()
    if default_backend not in ("native", "auto", "torch"):
        raise ValueError("Invalid default_backend")
    selected = options or NativeOptions()
    if not isinstance(selected, NativeOptions):
        raise TypeError("options must be NativeOptions")
    with _LOCK:
        if _ORIGINAL is not None and cls.bfs is not _INSTALLED:
            raise RuntimeError("CayleyGraph.bfs was replaced by another integration")
        original = _ORIGINAL or cls.bfs

        @wraps(original)
        def installed(graph, **kwargs):
            return _search(original, graph, kwargs.pop("backend", default_backend),
                           kwargs.pop("native_options", selected), kwargs.pop("output", None), kwargs)

        _ORIGINAL, _INSTALLED = original, installed
        cls.bfs = installed


def disable_native():
    """Restore the original method without overwriting another integration."""
    global _ORIGINAL, _INSTALLED
    cls = _cayley_graph_class()
    with _LOCK:
        if _ORIGINAL is not None:
            if cls.bfs is not _INSTALLED:
                raise RuntimeError("CayleyGraph.bfs was replaced by another integration")
            cls.bfs = _ORIGINAL
            _ORIGINAL = _INSTALLED = None
