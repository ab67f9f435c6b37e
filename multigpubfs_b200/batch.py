"""Batched sweep: many BFS instances in one device-driven CUDA-graph loop.

    with BatchSweep(graphs) as sweep:
        status = sweep.run()                 # plain planner: orbit-bound capacities
        tables = sweep.layer_tables()
        status = sweep.run(capacities=[...]) # learned planner: predicted capacities, exact overflow rerun

The reference runs such sweeps one graph at a time through a resident worker
pool (multigpubfs/generic_session.py:139, docs/RESIDENT_SWEEP.md); here one
mgbfs2_batch_run advances every instance together, a whole wave per graph
launch.
"""
from __future__ import annotations

import ctypes as C

from . import native
from .graph_definition import GraphDefinition


class BatchSweep:
    def __init__(self, graphs, device: int = 0):
        self.lib = native.require_device()
        self.graphs = [g if isinstance(g, GraphDefinition) else GraphDefinition.from_dict(g) for g in graphs]
        n = len(self.graphs)
        descs = (native.GraphDesc * n)()
        self._keep = []
        for k, g in enumerate(self.graphs):
            a = g.action
            if a["kind"] != "permutation":
                raise ValueError("BATCH_REQUIRES_PERMUTATION_ACTION")
            start = g.start
            st = (C.c_int64 * len(start))(*start)
            flat = (C.c_uint32 * (len(start) * g.generator_count))(*[x for gen in a["generators"] for x in gen])
            self._keep += [st, flat]
            d = descs[k]
            d.kind = 0
            d.elements = d.rows = len(start)
            d.cols = 1
            d.generators = g.generator_count
            d.permutations = C.cast(flat, C.POINTER(C.c_uint32))
            d.start = C.cast(st, C.POINTER(C.c_int64))
        handle = C.c_void_p()
        err = C.create_string_buffer(512)
        rc = self.lib.mgbfs2_batch_create(descs, n, device, C.byref(handle), err, len(err))
        if rc:
            raise native.NativeError(rc, "mgbfs2_batch_create", err.value.decode(errors="replace"))
        self.handle = handle
        self.count = n

    def close(self):
        if getattr(self, "handle", None):
            self.lib.mgbfs2_batch_destroy(self.handle)
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

    def run(self, *, capacities=None, memory_bytes=None, max_depth=None, host_loop=False, graph_loop=False,
            blocks_per_sm=None) -> dict:
        """Runs every instance to completion.  Each wave is one persistent
        cooperative launch by default; `host_loop` launches every layer step
        from the host (one sync per layer, e.g. for a profiler) and
        `graph_loop` runs the steps as a CUDA-graph WHILE loop."""
        if host_loop and graph_loop:
            raise ValueError("host_loop and graph_loop are exclusive")
        opts = native.BatchOptions()
        opts.max_depth = max_depth or 0
        opts.host_loop = 1 if host_loop else (2 if graph_loop else 0)
        opts.memory_bytes = memory_bytes or 0
        opts.blocks_per_sm = blocks_per_sm or 0
        keep = None
        if capacities is not None:
            if len(capacities) != self.count:
                raise ValueError("capacities: one per instance")
            keep = (C.c_uint64 * self.count)(*[max(0, int(c)) for c in capacities])
            opts.predicted_capacity = C.cast(keep, C.POINTER(C.c_uint64))
        status = native.BatchStatus()
        native.check(self.lib.mgbfs2_batch_run(self.handle, C.byref(opts), C.byref(status)), "mgbfs2_batch_run")
        return status.to_dict()

    def layer_table(self, instance: int):
        count = C.c_size_t()
        native.check(self.lib.mgbfs2_batch_layer_table(self.handle, instance, None, 0, C.byref(count)),
                     "mgbfs2_batch_layer_table")
        sizes = (C.c_uint64 * max(count.value, 1))()
        native.check(self.lib.mgbfs2_batch_layer_table(self.handle, instance, sizes, count.value, C.byref(count)),
                     "mgbfs2_batch_layer_table")
        return [int(sizes[i]) for i in range(count.value)]

    def layer_tables(self):
        return [self.layer_table(i) for i in range(self.count)]
