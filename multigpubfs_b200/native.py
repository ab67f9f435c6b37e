"""ctypes binding of libmgbfs2.so (the C ABI declared in include/mgbfs2.h).

There is no CPU fallback: if the shared library is missing or no CUDA device
is present, every entry point raises ``NativeUnavailable``.
"""
from __future__ import annotations

import ctypes as C
import os
import threading
from pathlib import Path

from .build import LIBRARY

_LOCK = threading.Lock()
_LIB = None

DEVICE_STATUS = 5  # MGBFS2_DEVICE_STATUS
VISITED = {"auto": 0, "bitmap": 1, "hash": 2, "hash3": 3}
VISITED_NAMES = {v: k for k, v in VISITED.items()}
DEDUP = {"auto": 0, "atomic": 1, "warp": 2, "sort": 3, "bucket": 4, "grouped": 5}
DEDUP_NAMES = {v: k for k, v in DEDUP.items()}
PLANNER = {"plain": 0, "learned": 1}
REASONS = {0: "FRONTIER_EXHAUSTED", 1: "DEADLINE", 2: "CANCELLED", 3: "RESOURCE", 4: "PROFILE_LAYER_LIMIT"}
ERROR_BITS = {1: "FRONTIER_OVERFLOW", 2: "TABLE_FULL", 4: "RANK_RANGE", 8: "BUCKET_OVERFLOW", 16: "WAIT_LIMIT",
              32: "ARENA_OVERFLOW", 64: "BAD_STATE", 128: "BAD_REFERENCE"}


class NativeUnavailable(RuntimeError):
    """libmgbfs2 could not be loaded or no CUDA device is usable."""


class NativeError(RuntimeError):
    def __init__(self, code: int, where: str, message: str = ""):
        self.code = code
        text = f"{where}: MGBFS2_STATUS_{code} ({status_string(code)})"
        if message:
            text += f": {message}"
        super().__init__(text)


class GraphDesc(C.Structure):
    _fields_ = [("kind", C.c_uint32), ("elements", C.c_uint32), ("rows", C.c_uint32), ("cols", C.c_uint32),
                ("generators", C.c_uint32), ("permutations", C.POINTER(C.c_uint32)),
                ("matrices", C.POINTER(C.c_int64)), ("moduli", C.POINTER(C.c_uint32)),
                ("start", C.POINTER(C.c_int64)), ("orbit_bound", C.c_uint64)]


class PlanRequest(C.Structure):
    _fields_ = [("visited", C.c_uint32), ("dedup", C.c_uint32), ("capacity", C.c_uint64),
                ("reserve_bytes", C.c_uint64), ("shards", C.c_uint32), ("block", C.c_uint32),
                ("planner", C.c_uint32), ("bucket_margin", C.c_uint32), ("bucket_min_work", C.c_uint64),
                ("options", C.c_uint32), ("hash_load_percent", C.c_uint32), ("predicted_states", C.c_uint64),
                ("predicted_peak", C.c_uint64), ("group_chunk", C.c_uint32), ("blocks_per_sm", C.c_uint32),
                ("parents_per_thread", C.c_uint32), ("route_chunk", C.c_uint32)]


OPTION_NO_PARENT_SKIP = 1
OPTION_HOST_LOOP = 2
OPTION_FULL_RANK = 4
OPTION_WIDE_SLOTS = 8


class PlanInfo(C.Structure):
    _fields_ = [("visited", C.c_uint32), ("dedup", C.c_uint32), ("packed", C.c_uint32),
                ("bits_per_symbol", C.c_uint32), ("key_words", C.c_uint32), ("history_layers", C.c_uint32),
                ("capacity", C.c_uint64), ("table_slots", C.c_uint64), ("bitmap_bits", C.c_uint64),
                ("device_bytes", C.c_uint64), ("state_bound", C.c_uint64), ("shards", C.c_uint32),
                ("block", C.c_uint32), ("inverse_closed", C.c_uint32), ("planner", C.c_uint32),
                ("parent_skip", C.c_uint32), ("bucket_prefix", C.c_uint32), ("table_slot_bytes", C.c_uint32),
                ("hash_load_percent", C.c_uint32), ("group_chunk", C.c_uint32), ("blocks_per_sm", C.c_uint32),
                ("rank_components", C.c_uint32), ("parents_per_thread", C.c_uint32)]

    def to_dict(self):
        d = {name: getattr(self, name) for name, _ in self._fields_}
        d["visited"] = VISITED_NAMES.get(self.visited, self.visited)
        d["dedup"] = DEDUP_NAMES.get(self.dedup, self.dedup)
        d["planner"] = {0: "plain", 1: "learned"}.get(self.planner, self.planner)
        return d


class RunLimits(C.Structure):
    _fields_ = [("max_seconds", C.c_double), ("max_layers", C.c_uint32), ("reserved", C.c_uint32),
                ("cancel", C.POINTER(C.c_int32))]


class RunStatus(C.Structure):
    _fields_ = [("complete", C.c_uint32), ("reason", C.c_uint32), ("fatal", C.c_uint32), ("layers", C.c_uint32),
                ("states", C.c_uint64), ("successors", C.c_uint64), ("bfs_seconds", C.c_double),
                ("redo_layers", C.c_uint32), ("kernel_launches", C.c_uint32), ("peak_device_bytes", C.c_uint64),
                ("device_seconds", C.c_double), ("kernel_seconds", C.c_double), ("visited_tests", C.c_uint64)]


class BatchOptions(C.Structure):
    _fields_ = [("max_depth", C.c_uint32), ("blocks_per_sm", C.c_uint32), ("host_loop", C.c_uint32),
                ("tile_entries", C.c_uint32), ("memory_bytes", C.c_uint64), ("reserve_bytes", C.c_uint64),
                ("predicted_capacity", C.POINTER(C.c_uint64))]


class BatchStatus(C.Structure):
    _fields_ = [("instances", C.c_uint32), ("complete_instances", C.c_uint32), ("waves", C.c_uint32),
                ("redo_instances", C.c_uint32), ("graph_launches", C.c_uint32), ("kernel_launches", C.c_uint32),
                ("layer_steps", C.c_uint32), ("fatal", C.c_uint32), ("states", C.c_uint64),
                ("successors", C.c_uint64), ("seconds", C.c_double), ("device_seconds", C.c_double),
                ("redo_layers", C.c_uint32), ("reserved", C.c_uint32)]

    def to_dict(self):
        return {name: getattr(self, name) for name, _ in self._fields_ if name != "reserved"}


LAYER_CALLBACK = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_uint32, C.c_uint64, C.c_double)

_SIGNATURES = {
    "mgbfs2_graph_create": (C.c_int, [C.POINTER(GraphDesc), C.c_int, C.POINTER(C.c_void_p), C.c_char_p, C.c_size_t]),
    "mgbfs2_plan": (C.c_int, [C.c_void_p, C.POINTER(PlanRequest), C.POINTER(PlanInfo)]),
    "mgbfs2_run": (C.c_int, [C.c_void_p, C.POINTER(RunLimits), LAYER_CALLBACK, C.c_void_p, C.POINTER(RunStatus)]),
    "mgbfs2_layer_table": (C.c_int, [C.c_void_p, C.POINTER(C.c_uint64), C.POINTER(C.c_double), C.c_size_t,
                                     C.POINTER(C.c_size_t)]),
    "mgbfs2_sample": (C.c_int, [C.c_void_p, C.c_uint32, C.POINTER(C.c_int64), C.c_size_t, C.POINTER(C.c_size_t)]),
    "mgbfs2_status_string": (C.c_char_p, [C.c_int]),
    "mgbfs2_destroy": (None, [C.c_void_p]),
    "mgbfs2_trim_memory": (C.c_int, [C.c_int]),
    "mgbfs2_table_probes": (C.c_int, [C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_uint64)]),
    "mgbfs2_checkpoint_write": (C.c_int, [C.c_void_p, C.c_char_p]),
    "mgbfs2_checkpoint_resume": (C.c_int, [C.c_void_p, C.c_char_p]),
    "mgbfs2_frontier_words": (C.c_int, [C.c_void_p, C.c_void_p, C.c_size_t, C.POINTER(C.c_size_t)]),
    "mgbfs2_trace_range_push": (None, [C.c_char_p]),
    "mgbfs2_trace_range_pop": (None, []),
    "mgbfs2_rank_components": (C.c_int, [C.c_uint32, C.c_uint32, C.c_uint32, C.POINTER(C.c_uint32), C.c_uint32,
                                         C.POINTER(C.c_uint32), C.c_void_p, C.c_uint64, C.c_void_p,
                                         C.POINTER(C.c_uint64), C.c_void_p, C.c_void_p]),
    "mgbfs2_batch_layer_tables": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint64, C.c_void_p]),
    "mgbfs2_successors_i64": (C.c_int, [C.c_uint32] * 5 + [C.c_void_p, C.c_uint64, C.c_void_p, C.c_void_p,
                                                           C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "mgbfs2_successors_packed": (C.c_int, [C.c_uint32, C.c_uint32, C.c_uint32, C.POINTER(C.c_uint32), C.c_void_p,
                                           C.c_uint64, C.c_void_p, C.c_void_p]),
    "mgbfs2_rank_packed": (C.c_int, [C.c_uint32, C.c_uint32, C.c_uint32, C.POINTER(C.c_uint32), C.c_void_p,
                                     C.c_uint64, C.c_void_p, C.c_void_p, C.c_void_p]),
    "mgbfs2_bitmap_claim": (C.c_int, [C.c_void_p, C.c_uint64, C.c_void_p, C.c_uint64, C.c_void_p, C.c_uint32,
                                      C.c_void_p, C.c_void_p]),
    "mgbfs2_hash_insert": (C.c_int, [C.c_void_p, C.c_uint64, C.c_void_p, C.c_uint64, C.c_void_p, C.c_void_p,
                                     C.c_void_p]),
    "mgbfs2_sort_unique_tiles": (C.c_int, [C.c_void_p, C.c_uint64, C.c_uint32, C.c_uint32, C.c_void_p, C.c_void_p,
                                           C.c_void_p]),
    "mgbfs2_bucket_keys": (C.c_int, [C.c_void_p, C.c_uint64, C.c_uint32, C.c_uint32, C.c_void_p, C.c_uint64,
                                     C.c_void_p, C.c_void_p, C.c_void_p]),
    "mgbfs2_expand_layer_bitmap": (C.c_int, [C.c_uint32, C.c_uint32, C.POINTER(C.c_uint32), C.c_void_p, C.c_uint64,
                                             C.c_void_p, C.c_void_p, C.c_uint64, C.c_void_p, C.c_void_p,
                                             C.c_void_p, C.c_uint64, C.c_void_p]),
    "mgbfs2_expand_layer_scratch_bytes": (C.c_uint64, [C.c_uint32, C.c_uint32, C.c_uint64]),
    "mgbfs2_expand_layer_bitmap_static": (C.c_int, [C.c_uint32, C.c_uint32, C.POINTER(C.c_uint32), C.c_void_p,
                                                    C.c_uint64, C.c_void_p, C.c_void_p, C.c_uint64, C.c_void_p,
                                                    C.c_void_p, C.c_void_p]),
    "mgbfs2_shard_geometry": (C.c_int, [C.c_uint32, C.c_uint32, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32),
                                        C.POINTER(C.c_uint64)]),
    "mgbfs2_shard_scratch_bytes": (C.c_uint64, []),
    "mgbfs2_shard_route": (C.c_int, [C.c_uint32, C.c_uint32, C.POINTER(C.c_uint32), C.c_void_p, C.c_uint64,
                                     C.c_uint32, C.c_void_p, C.c_uint64, C.c_void_p, C.c_void_p, C.c_void_p,
                                     C.c_uint64, C.c_void_p]),
    "mgbfs2_shard_accept": (C.c_int, [C.c_uint32, C.c_uint32, C.c_uint32, C.c_void_p, C.c_void_p, C.c_void_p,
                                      C.c_void_p, C.c_uint64, C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint64,
                                      C.c_void_p]),
    "mgbfs2_batch_create": (C.c_int, [C.POINTER(GraphDesc), C.c_uint32, C.c_int, C.POINTER(C.c_void_p), C.c_char_p,
                                      C.c_size_t]),
    "mgbfs2_batch_run": (C.c_int, [C.c_void_p, C.POINTER(BatchOptions), C.POINTER(BatchStatus)]),
    "mgbfs2_batch_layer_table": (C.c_int, [C.c_void_p, C.c_uint32, C.POINTER(C.c_uint64), C.c_size_t,
                                           C.POINTER(C.c_size_t)]),
    "mgbfs2_batch_layer_seconds": (C.c_int, [C.c_void_p, C.c_uint32, C.POINTER(C.c_double), C.c_size_t,
                                             C.POINTER(C.c_size_t)]),
    "mgbfs2_batch_destroy": (None, [C.c_void_p]),
    "mgbfs2_mlp_param_count": (C.c_uint32, [C.c_uint32]),
    "mgbfs2_mlp_forward": (C.c_int, [C.c_uint32, C.c_void_p, C.c_void_p, C.c_uint64, C.c_void_p, C.c_void_p]),
    "mgbfs2_mlp_loss_grad": (C.c_int, [C.c_uint32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_float, C.c_float,
                                       C.c_uint64, C.c_void_p, C.c_void_p, C.c_void_p]),
    "mgbfs2_mlp_adam": (C.c_int, [C.c_uint32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_float, C.c_float,
                                  C.c_float, C.c_float, C.c_uint32, C.c_void_p]),
    "mgbfs2_mlp_to_bf16": (C.c_int, [C.c_uint32, C.c_void_p, C.c_void_p, C.c_void_p]),
    "mgbfs2_mlp_infer_bf16": (C.c_int, [C.c_uint32, C.c_void_p, C.c_void_p, C.c_uint64, C.c_void_p, C.c_void_p]),
    "mgbfs2_mlp_rollout_bf16": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32,
                                          C.c_uint32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "mgbfs2_group_order": (C.c_int, [C.POINTER(C.c_uint32), C.c_uint32, C.c_uint32, C.POINTER(C.c_uint64)]),
    "mgbfs2_graph_statics": (C.c_int, [C.c_uint32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32,
                                       C.c_void_p, C.c_void_p]),
}


def group_order(generators) -> int:
    """Order of the permutation group the generators generate (host
    Schreier-Sims in libmgbfs2; no device needed)."""
    gens = [list(g) for g in generators]
    n = len(gens[0]) if gens else 1
    flat = (C.c_uint32 * max(1, n * len(gens)))(*[x for g in gens for x in g])
    out = C.c_uint64()
    check(load().mgbfs2_group_order(flat, n, len(gens), C.byref(out)), "mgbfs2_group_order")
    return int(out.value)


def graph_statics(graphs, threads: int = 0):
    """Planner statics of many permutation graphs in one host call
    (mgbfs2_graph_statics): a (count, 8) float32 array in the device rollout's
    layout and a uint64 array of settled-state counts (|G| for distinct
    labels, else the multinomial bound).  `graphs` are (generators, start)
    pairs."""
    import numpy as np
    degree, gens, perms, labels = [], [], [], []
    for generators, start in graphs:
        ids = {}
        labels.extend(ids.setdefault(v, len(ids)) for v in start)
        degree.append(len(start))
        gens.append(len(generators))
        for g in generators:
            perms.extend(g)
    count = len(degree)
    statics = np.zeros((count, 8), dtype=np.float32)
    states = np.zeros(count, dtype=np.uint64)
    if not count:
        return statics, states
    d = np.asarray(degree, dtype=np.uint32)
    k = np.asarray(gens, dtype=np.uint32)
    p = np.asarray(perms, dtype=np.uint32)
    lab = np.asarray(labels, dtype=np.uint32)
    check(load().mgbfs2_graph_statics(count, d.ctypes.data, k.ctypes.data, p.ctypes.data, lab.ctypes.data, threads,
                                      statics.ctypes.data, states.ctypes.data), "mgbfs2_graph_statics")
    return statics, states


def exported_symbols():
    """Names declared by include/mgbfs2.h that the library must export."""
    return sorted(_SIGNATURES)


def load(path: str | Path | None = None):
    """Load libmgbfs2 (no device check).  Raises NativeUnavailable if absent."""
    global _LIB
    with _LOCK:
        if _LIB is not None and path is None:
            return _LIB
        target = Path(path) if path else Path(os.environ.get("MGBFS2_LIBRARY", LIBRARY))
        if not target.exists():
            raise NativeUnavailable(f"libmgbfs2 not built: {target} (run python -m multigpubfs_b200.build)")
        try:
            lib = C.CDLL(str(target))
        except OSError as exc:
            raise NativeUnavailable(f"libmgbfs2 failed to load: {exc}") from exc
        for name, (restype, argtypes) in _SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = restype
            fn.argtypes = argtypes
        if path is None:
            _LIB = lib
        return lib


def status_string(code: int) -> str:
    try:
        return load().mgbfs2_status_string(code).decode()
    except NativeUnavailable:
        return "UNKNOWN"


def require_device():
    """Load the library and require a CUDA device (no CPU fallback)."""
    lib = load()
    import torch
    if not torch.cuda.is_available():
        raise NativeUnavailable("no CUDA device: the native BFS has no CPU fallback")
    return lib


def trim_memory(device: int = 0):
    """Give the library's cached device buffers and the pool's unused memory
    back to the device (mgbfs2_trim_memory)."""
    check(require_device().mgbfs2_trim_memory(device), "mgbfs2_trim_memory")


def check(code: int, where: str):
    if code:
        raise NativeError(code, where)


def stream_handle(stream=None) -> int | None:
    """cudaStream_t of a torch stream (None -> torch's current stream)."""
    import torch
    s = stream if stream is not None else torch.cuda.current_stream()
    return s.cuda_stream


def ptr(tensor) -> int:
    return tensor.data_ptr()
