"""Python handle over one libmgbfs2 graph: create -> plan -> run -> table/sample.

This is the in-process replacement of the reference's ``mgbfs graph`` process
(crates/mgbfs-runtime/src/generic_run.rs): same plan, layer loop and report
fields, called through the C ABI instead of a subprocess.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

from . import native
from .graph_definition import GraphDefinition


@dataclass
class RunResult:
    complete: bool
    reason: str
    fatal: int
    layer_sizes: list
    layer_seconds: list
    states: int
    successors: int
    bfs_seconds: float
    kernel_launches: int
    redo_layers: int
    peak_device_bytes: int
    device_seconds: float = 0.0
    kernel_seconds: float = 0.0
    visited_tests: int = 0
    fatal_names: list = field(default_factory=list)


class NativeGraph:
    """Owns one mgbfs2_graph handle on one device."""

    def __init__(self, graph: GraphDefinition, device: int = 0):
        self.lib = native.require_device()
        self.graph = graph
        self.device = device
        a = graph.action
        start = graph.start
        self._keep = []
        desc = native.GraphDesc()
        desc.elements = len(start)
        desc.generators = graph.generator_count
        st = (C.c_int64 * len(start))(*start)
        self._keep.append(st)
        desc.start = C.cast(st, C.POINTER(C.c_int64))
        bound = graph.expected_max_unique_states
        desc.orbit_bound = 0 if bound is None else bound
        if a["kind"] == "permutation":
            desc.kind = 0
            desc.rows, desc.cols = len(start), 1
            flat = (C.c_uint32 * (len(start) * desc.generators))(*[x for g in a["generators"] for x in g])
            self._keep.append(flat)
            desc.permutations = C.cast(flat, C.POINTER(C.c_uint32))
        else:
            desc.kind = 1
            desc.rows, desc.cols = a["rows"], a["cols"]
            mats = (C.c_int64 * (a["rows"] * a["rows"] * desc.generators))(
                *[x for g in a["generators"] for x in g["matrix"]])
            mods = (C.c_uint32 * desc.generators)(*[g["modulo"] for g in a["generators"]])
            self._keep += [mats, mods]
            desc.matrices = C.cast(mats, C.POINTER(C.c_int64))
            desc.moduli = C.cast(mods, C.POINTER(C.c_uint32))
        handle = C.c_void_p()
        err = C.create_string_buffer(512)
        rc = self.lib.mgbfs2_graph_create(C.byref(desc), device, C.byref(handle), err, len(err))
        if rc:
            raise native.NativeError(rc, "mgbfs2_graph_create", err.value.decode(errors="replace"))
        self.handle = handle
        self.plan_info = None

    def close(self):
        if getattr(self, "handle", None):
            self.lib.mgbfs2_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def plan(self, *, visited="auto", dedup="auto", capacity=None, reserve_bytes=None, shards=None,
             planner="plain", bucket_margin=None, bucket_min_work=None, parent_skip=True, host_loop=False,
             full_rank=False, wide_slots=False, hash_load_percent=None, predicted_states=None,
             predicted_peak=None, group_chunk=None, blocks_per_sm=None, parents_per_thread=None,
             route_chunk=None) -> dict:
        """Plans the run (mgbfs2_plan).  planner="learned" needs
        `predicted_states` (and optionally `predicted_peak`), e.g. from
        planner.predict_graph."""
        req = native.PlanRequest()
        req.predicted_states = int(predicted_states or 0)
        req.predicted_peak = int(predicted_peak or 0)
        req.group_chunk = int(group_chunk or 0)
        req.blocks_per_sm = int(blocks_per_sm or 0)
        req.parents_per_thread = int(parents_per_thread or 0)
        req.route_chunk = int(route_chunk or 0)
        req.options = ((0 if parent_skip else native.OPTION_NO_PARENT_SKIP) |
                       (native.OPTION_HOST_LOOP if host_loop else 0) | (native.OPTION_FULL_RANK if full_rank else 0) |
                       (native.OPTION_WIDE_SLOTS if wide_slots else 0))
        req.hash_load_percent = hash_load_percent or 0
        req.bucket_margin = 0 if bucket_margin is None else (0xFFFFFFFF if bucket_margin == 0 else bucket_margin)
        req.bucket_min_work = bucket_min_work or 0
        req.visited = native.VISITED[visited]
        req.dedup = native.DEDUP[dedup]
        req.capacity = capacity or 0
        req.reserve_bytes = reserve_bytes or 0
        req.shards = shards or 0
        req.planner = native.PLANNER[planner]
        info = native.PlanInfo()
        native.check(self.lib.mgbfs2_plan(self.handle, C.byref(req), C.byref(info)), "mgbfs2_plan")
        self.plan_info = info.to_dict()
        return self.plan_info

    def run(self, *, max_seconds=None, max_layers=None, cancel_flag=None, on_layer=None) -> RunResult:
        limits = native.RunLimits()
        limits.max_seconds = float(max_seconds or 0)
        limits.max_layers = max_layers or 0
        if cancel_flag is not None:
            limits.cancel = C.cast(C.addressof(cancel_flag), C.POINTER(C.c_int32))
        status = native.RunStatus()

        def trampoline(user, depth, size, seconds):
            try:
                return 1 if on_layer(depth, size, seconds) else 0
            except Exception:
                return 1

        cb = native.LAYER_CALLBACK(trampoline) if on_layer else native.LAYER_CALLBACK()
        native.check(self.lib.mgbfs2_run(self.handle, C.byref(limits), cb, None, C.byref(status)), "mgbfs2_run")
        sizes, seconds = self.layer_table()
        names = [name for bit, name in native.ERROR_BITS.items() if status.fatal & bit]
        return RunResult(bool(status.complete), native.REASONS.get(status.reason, str(status.reason)), status.fatal,
                         sizes, seconds, status.states, status.successors, status.bfs_seconds,
                         status.kernel_launches, status.redo_layers, status.peak_device_bytes,
                         status.device_seconds, status.kernel_seconds, status.visited_tests, names)

    def table_probes(self):
        """(mean probes per stored key, keys) of the all-visited hash after a run."""
        mean, keys = C.c_double(), C.c_uint64()
        native.check(self.lib.mgbfs2_table_probes(self.handle, C.byref(mean), C.byref(keys)), "mgbfs2_table_probes")
        return float(mean.value), int(keys.value)

    def checkpoint(self, path):
        """Writes the BFS state after run() (mgbfs2_checkpoint_write)."""
        native.check(self.lib.mgbfs2_checkpoint_write(self.handle, str(path).encode()), "mgbfs2_checkpoint_write")

    def resume(self, path):
        """Loads a checkpoint into this planned handle; the next run() goes on
        from its depth (mgbfs2_checkpoint_resume)."""
        native.check(self.lib.mgbfs2_checkpoint_resume(self.handle, str(path).encode()), "mgbfs2_checkpoint_resume")

    def frontier_words(self):
        """The deepest layer's packed states (numpy uint64), tags removed."""
        import numpy as np
        count = C.c_size_t()
        native.check(self.lib.mgbfs2_frontier_words(self.handle, None, 0, C.byref(count)), "mgbfs2_frontier_words")
        out = np.zeros(max(count.value, 1), dtype=np.uint64)
        native.check(self.lib.mgbfs2_frontier_words(self.handle, out.ctypes.data, out.size, C.byref(count)),
                     "mgbfs2_frontier_words")
        return out[:count.value]

    def layer_table(self):
        count = C.c_size_t()
        native.check(self.lib.mgbfs2_layer_table(self.handle, None, None, 0, C.byref(count)), "mgbfs2_layer_table")
        n = count.value
        sizes = (C.c_uint64 * max(n, 1))()
        secs = (C.c_double * max(n, 1))()
        native.check(self.lib.mgbfs2_layer_table(self.handle, sizes, secs, n, C.byref(count)), "mgbfs2_layer_table")
        return [int(sizes[i]) for i in range(n)], [float(secs[i]) for i in range(1, n)]

    def sample(self, which: int, limit: int = 1000):
        """which=0: up to `limit` states of the deepest layer; which=1: the layer
        before it if it holds fewer than 1000 states.  Sorted int64 rows."""
        width = self.graph.state_elements
        out = (C.c_int64 * max(1, limit * width))()
        rows = C.c_size_t()
        native.check(self.lib.mgbfs2_sample(self.handle, which, out, limit, C.byref(rows)), "mgbfs2_sample")
        return [[int(out[r * width + e]) for e in range(width)] for r in range(rows.value)]
