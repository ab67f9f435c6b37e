"""Batched sweep: many BFS instances, each wave one persistent launch.

    with BatchSweep(graphs) as sweep:
        status = sweep.run()                 # plain planner: orbit-bound capacities
        tables = sweep.layer_tables()
        status = sweep.run(capacities=[...]) # learned planner: predicted capacities, exact overflow rerun
        sweep.write_results("out/")          # results.csv, layers.csv, checksums.json

The reference runs such sweeps one graph at a time through a resident worker
pool (multigpubfs/generic_session.py:139, docs/RESIDENT_SWEEP.md); here one
mgbfs2_batch_run advances every instance together, a whole wave per launch.
"""
from __future__ import annotations

import csv
import ctypes as C
import hashlib
import json
from itertools import chain
from pathlib import Path

import numpy as np

from . import native
from .graph_definition import GraphDefinition


_DESC_DTYPE = np.dtype({
    "names": [name for name, _ in native.GraphDesc._fields_],
    "formats": [np.uint64 if issubclass(t, C._Pointer) or t is C.c_uint64 else np.uint32
                for _, t in native.GraphDesc._fields_],
    "offsets": [getattr(native.GraphDesc, name).offset for name, _ in native.GraphDesc._fields_],
    "itemsize": C.sizeof(native.GraphDesc)})


class BatchSweep:
    def __init__(self, graphs, device: int = 0):
        """`graphs`: schema-2 dicts or GraphDefinitions of permutation graphs.
        Their generators and starts are packed into two flat arrays that the
        descriptors point into; mgbfs2_batch_create validates them (generator
        permutations, distinct labels, degree and generator limits)."""
        self.lib = native.require_device()
        self.graphs = [g.to_dict() if isinstance(g, GraphDefinition) else g for g in graphs]
        n = len(self.graphs)
        if not n:
            raise ValueError("BATCH_ARGUMENT: no instances")
        if any(g["action"]["kind"] != "permutation" for g in self.graphs):
            raise ValueError("BATCH_REQUIRES_PERMUTATION_ACTION")
        degree = np.fromiter((len(g["start"]) for g in self.graphs), dtype=np.int64, count=n)
        gens = np.fromiter((len(g["action"]["generators"]) for g in self.graphs), dtype=np.int64, count=n)
        starts = np.fromiter(chain.from_iterable(g["start"] for g in self.graphs), dtype=np.int64,
                             count=int(degree.sum()))
        perms = np.fromiter(chain.from_iterable(chain.from_iterable(g["action"]["generators"]) for g in self.graphs),
                            dtype=np.int64, count=int((degree * gens).sum()))
        if perms.size and (perms.min() < 0 or perms.max() > 0xFFFFFFFF):
            raise ValueError("GRAPH_PERMUTATION_GENERATOR")
        perms = perms.astype(np.uint32)
        self._keep = [starts, perms]
        # The descriptor array is filled column-wise through a numpy view with
        # the ctypes structure's field offsets.
        descs = (native.GraphDesc * n)()
        view = np.frombuffer(descs, dtype=_DESC_DTYPE, count=n)
        view["elements"] = view["rows"] = degree
        view["cols"] = 1
        view["generators"] = gens
        view["permutations"] = perms.ctypes.data + 4 * (np.cumsum(degree * gens) - degree * gens)
        view["start"] = starts.ctypes.data + 8 * (np.cumsum(degree) - degree)
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
            blocks_per_sm=None, tile_entries=None) -> dict:
        """Runs every instance to completion.  Each wave is one persistent
        cooperative launch by default; `host_loop` launches every layer step
        from the host (one sync per layer, e.g. for a profiler) and
        `graph_loop` runs the steps as a CUDA-graph WHILE loop.
        `blocks_per_sm` and `tile_entries` (256, 512 or 1024 frontier entries
        per tile) are speed-only shapes; autotune.choose_sweep_shape picks them."""
        if host_loop and graph_loop:
            raise ValueError("host_loop and graph_loop are exclusive")
        opts = native.BatchOptions()
        opts.max_depth = max_depth or 0
        opts.host_loop = 1 if host_loop else (2 if graph_loop else 0)
        opts.memory_bytes = memory_bytes or 0
        opts.blocks_per_sm = blocks_per_sm or 0
        opts.tile_entries = tile_entries or 0
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
        """Every instance's layer table, from one native call."""
        offsets = np.zeros(self.count + 1, dtype=np.uint64)
        native.check(self.lib.mgbfs2_batch_layer_tables(self.handle, None, 0, offsets.ctypes.data),
                     "mgbfs2_batch_layer_tables")
        total = int(offsets[-1])
        flat = np.zeros(max(total, 1), dtype=np.uint64)
        native.check(self.lib.mgbfs2_batch_layer_tables(self.handle, flat.ctypes.data, total, offsets.ctypes.data),
                     "mgbfs2_batch_layer_tables")
        values = flat.tolist()
        cuts = offsets.tolist()
        return [values[cuts[i]:cuts[i + 1]] for i in range(self.count)]

    def layer_seconds(self, instance: int):
        """Per-layer expansion seconds of one instance, aligned with its layer
        table (entry 0, the start, is 0; entry d is its wave's step that
        produced layer d)."""
        count = C.c_size_t()
        native.check(self.lib.mgbfs2_batch_layer_seconds(self.handle, instance, None, 0, C.byref(count)),
                     "mgbfs2_batch_layer_seconds")
        out = (C.c_double * max(count.value, 1))()
        native.check(self.lib.mgbfs2_batch_layer_seconds(self.handle, instance, out, count.value, C.byref(count)),
                     "mgbfs2_batch_layer_seconds")
        return [float(out[i]) for i in range(count.value)]

    def write_results(self, output):
        """The sweep tables of the last run: see `write_sweep_results`."""
        names = [g.get("name") or f"instance-{i}" for i, g in enumerate(self.graphs)]
        degrees = [len(g["start"]) for g in self.graphs]
        return write_sweep_results(output, names, degrees, self.layer_tables(),
                                   [self.layer_seconds(i) for i in range(self.count)])


def write_sweep_results(output, names, degrees, tables, seconds):
    """Writes a sweep's tables in the layout of the reference's sweep outputs
    (docs/reproduce-pair-sweeps.md:17-23), one row per instance instead of per
    (n, r) pair:

    - results.csv: instance, name, n, status (COMPLETE / INCOMPLETE), the
      start's eccentricity when complete, completed depth, visited states,
      BFS seconds;
    - layers.csv: instance, depth, state count, cumulative count, expansion
      seconds (empty for depth zero, which is not expanded);
    - checksums.json: SHA256 of both files.

    An instance without a table (not completed) is INCOMPLETE with no layers.
    Returns the checksums."""
    out = Path(output)
    out.mkdir(parents=True, exist_ok=True)
    with open(out / "results.csv", "w", newline="", encoding="utf-8") as f:
        w = csv.writer(f, lineterminator="\n")
        w.writerow(["instance", "name", "n", "status", "eccentricity", "completed_depth", "visited", "bfs_seconds"])
        for i, (name, n, table, secs) in enumerate(zip(names, degrees, tables, seconds)):
            done = bool(table)
            w.writerow([i, name, n, "COMPLETE" if done else "INCOMPLETE", len(table) - 1 if done else "",
                        len(table) - 1 if done else "", sum(table), f"{sum(secs):.9f}"])
    with open(out / "layers.csv", "w", newline="", encoding="utf-8") as f:
        w = csv.writer(f, lineterminator="\n")
        w.writerow(["instance", "depth", "count", "cumulative", "seconds"])
        for i, (table, secs) in enumerate(zip(tables, seconds)):
            total = 0
            for d, count in enumerate(table):
                total += count
                w.writerow([i, d, count, total, "" if d == 0 else f"{secs[d]:.9f}"])
    sums = {name: hashlib.sha256((out / name).read_bytes()).hexdigest() for name in ("results.csv", "layers.csv")}
    (out / "checksums.json").write_text(json.dumps(sums, indent=1, sort_keys=True) + "\n", encoding="utf-8")
    return sums
