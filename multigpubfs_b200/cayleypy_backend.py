"""Explicit, reversible CayleyPy ``graph.bfs()`` integration.

Public surface of multigpubfs/cayleypy_backend.py:14-206 (NativeOptions,
NativeBfsResult, bfs, enable_native, disable_native) and its contract:

* importing the package patches nothing; ``enable_native`` installs one
  replacement of ``CayleyGraph.bfs`` and ``disable_native`` removes it;
* ``backend='torch'`` calls CayleyPy's own method with the caller's keywords;
* a keyword the native engine cannot honour (anything but CayleyPy's defaults,
  or more than one start state) raises NotImplementedError before any device
  work -- or, under ``backend='auto'`` with no ``output``, goes to CayleyPy;
* a native failure propagates: nothing is ever restarted on the CPU;
* a replacement of ``CayleyGraph.bfs`` made by someone else is never
  overwritten or removed (RuntimeError).

The engine behind it is ``run_graph`` (launch.py), one GPU through the C ABI.
"""
from __future__ import annotations

import json
import os
import tempfile
import threading
from dataclasses import dataclass, field
from functools import update_wrapper
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

    def engine_keywords(self) -> dict:
        """The run_graph keywords these options select."""
        chosen = dict(devices=self.devices, max_seconds=self.max_seconds, autotune=self.autotune,
                      memory_backend=self.memory_backend, segment_rows=self.segment_rows,
                      memory_preset=self.memory_preset, segment_strategy=self.segment_strategy,
                      bitmap_owner_page=self.bitmap_owner_page)
        if self.planner != "plain":
            chosen["planner"] = self.planner
        return chosen


@dataclass(frozen=True)
class NativeBfsResult:
    """Exact layer counts with compact state samples.  Unlike CayleyPy's
    BfsResult it keeps no full small layers, edges, hashes or paths: only the
    deepest layer and the one before it, and those in full only when the
    sample holds the whole layer."""
    bfs_completed: bool
    layer_sizes: list[int]
    graph: object
    report: dict
    output: Path
    layers: dict = field(default_factory=dict)
    layer_samples: dict = field(default_factory=dict)
    backend: str = field(default="native", init=False)

    @property
    def completed_depth(self):
        """Depth of the deepest layer reached (depth 0 is the start)."""
        return len(self.layer_sizes) - 1

    def num_vertices(self):
        total = 0
        for size in self.layer_sizes:
            total += size
        return total

    def diameter(self):
        if self.bfs_completed:
            return self.completed_depth
        raise RuntimeError("BFS_INCOMPLETE: only completed_depth is known")

    def get_layer(self, layer_id):
        try:
            layer = self.layers[layer_id]
        except KeyError:
            raise KeyError("Full layer not retained; use layer_samples for compact samples") from None
        return layer.cpu().numpy()

    def last_layer(self):
        return self.get_layer(self.completed_depth)


# CayleyPy's bfs() keywords and the only values the native engine honours.
_HONOURED = {"max_layer_size_to_store": 1000, "max_layer_size_to_explore": 10 ** 12, "max_diameter": 1000000,
             "return_all_edges": False, "return_all_hashes": False, "stop_condition": None,
             "disable_batching": False}
_BACKENDS = ("native", "torch", "auto")


def _blocking_keyword(kwargs):
    """First keyword whose value the engine cannot honour, else None
    (``start_states`` is judged separately, by its shape)."""
    return next((key for key, value in kwargs.items()
                 if key != "start_states" and (key not in _HONOURED or value != _HONOURED[key])), None)


def _definition_for(graph, start_states):
    """The graph's contract, with its start replaced by ``start_states`` when
    that is exactly one decoded state; None when it is not."""
    definition = from_cayleypy(graph)
    if start_states is None:
        return definition
    state = _flatten(start_states)
    if len(state) != definition.state_elements:
        return None
    return definition.with_start(state)


def _result_folder(options, output) -> Path:
    if output is not None:
        return Path(output).absolute()
    root = Path(options.output_root) if options.output_root else Path.cwd() / "bfs-results"
    root.mkdir(parents=True, exist_ok=True)
    # A fresh parent per call keeps receipts apart; run_graph makes the child.
    return (Path(tempfile.mkdtemp(prefix="run-", dir=root)) / "result").absolute()


def _samples(definition, report, folder):
    """Compact samples of the deepest layer ("current") and of the layer
    before it ("previous_small"), keyed by depth, as int64 tensors (matrix
    states reshaped to rows x cols); a sample that holds its whole layer is
    also a retained layer."""
    import torch
    stored = json.loads((folder / "states.json").read_text())
    sizes = report["layer_sizes"]
    action = definition.action
    samples, full = {}, {}
    for offset, key in enumerate(("current", "previous_small")):
        depth = len(sizes) - 1 - offset
        rows = stored.get(key) or []
        if depth < 0 or not rows:
            continue
        states = torch.tensor(rows, dtype=torch.int64)
        if action["kind"] == "matrix":
            states = states.reshape(-1, action["rows"], action["cols"])
        samples[depth] = states
        if len(rows) == sizes[depth]:
            full[depth] = states
    return samples, full


def _dispatch(original, graph, backend, options, output, kwargs):
    """Routes one bfs() call: CayleyPy's own method, or the native engine."""
    if backend not in _BACKENDS:
        raise ValueError("backend must be native, torch or auto")
    if not isinstance(options, NativeOptions):
        raise TypeError("native_options must be NativeOptions")
    if backend == "torch":
        if output is not None:
            raise ValueError("output belongs to the native backend")
        return original(graph, **kwargs)
    may_fall_back = backend == "auto" and output is None
    blocker = _blocking_keyword(kwargs)
    if blocker is not None:
        if may_fall_back:
            return original(graph, **kwargs)
        raise NotImplementedError(f"Native BFS does not support {blocker}; use backend='torch'")
    definition = _definition_for(graph, kwargs.get("start_states"))
    if definition is None:
        if may_fall_back:
            return original(graph, **kwargs)
        raise NotImplementedError("Native BFS supports a single decoded start state")
    folder = _result_folder(options, output)
    report = run_graph(definition, folder, **options.engine_keywords())
    samples, full = _samples(definition, report, folder)
    return NativeBfsResult(report["status"] == "COMPLETE", report["layer_sizes"],
                           getattr(graph, "definition", graph), report, folder, full, samples)


class _Installer:
    """Owns at most one replacement of ``CayleyGraph.bfs``.

    ``saved`` is the method that was on the class when the replacement went
    in, ``mine`` the replacement itself; both are None while nothing is
    installed.  A class attribute that is neither means another integration
    replaced ours, and then this installer touches nothing.
    """

    def __init__(self):
        self.lock = threading.RLock()
        self.saved = None
        self.mine = None

    def original(self, cls):
        with self.lock:
            return self.saved if self.saved is not None else cls.bfs

    def _assert_owned(self, cls):
        if self.saved is not None and cls.bfs is not self.mine:
            raise RuntimeError("CayleyGraph.bfs was replaced by another integration")

    def install(self, cls, default_backend, options):
        with self.lock:
            self._assert_owned(cls)
            original = self.original(cls)

            def replacement(graph, **kwargs):
                backend = kwargs.pop("backend", default_backend)
                chosen = kwargs.pop("native_options", options)
                output = kwargs.pop("output", None)
                return _dispatch(original, graph, backend, chosen, output, kwargs)

            update_wrapper(replacement, original)
            self.saved, self.mine = original, replacement
            cls.bfs = replacement

    def remove(self, cls):
        with self.lock:
            if self.saved is None:
                return
            self._assert_owned(cls)
            cls.bfs = self.saved
            self.saved = self.mine = None


_INSTALLER = _Installer()


def _cayley_graph_class():
    from cayleypy import CayleyGraph
    return CayleyGraph


def bfs(graph, *, backend="native", native_options=None, output=None, **kwargs):
    """One native (or CayleyPy) search without patching CayleyPy."""
    original = _INSTALLER.original(_cayley_graph_class())
    return _dispatch(original, graph, backend, native_options or NativeOptions(), output, kwargs)


def enable_native(options=None, *, default_backend="native", recovery=True):
    """Route ``CayleyGraph.bfs()`` to the native engine until
    ``disable_native()``.  Enabling twice replaces the previous defaults.
    ``recovery`` is accepted for signature compatibility: the in-process engine
    leaves no native worker processes behind to recover."""
    if default_backend not in _BACKENDS:
        raise ValueError("Invalid default_backend")
    selected = NativeOptions() if options is None else options
    if not isinstance(selected, NativeOptions):
        raise TypeError("options must be NativeOptions")
    _INSTALLER.install(_cayley_graph_class(), default_backend, selected)


def disable_native():
    """Put CayleyPy's own method back, unless another integration replaced ours."""
    _INSTALLER.remove(_cayley_graph_class())
