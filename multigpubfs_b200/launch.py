"""run_graph: plan + exact BFS on one GPU + the schema-2 report/states files.

Mirrors ``multigpubfs.launch.run_graph`` (multigpubfs/launch.py:151): same
keyword surface and validation codes, same output folder contract
(``report.json`` + ``states.json``, receipt-checked as in launch.py:77-82).
The reference spawns a native CLI per GPU; here the engine is called
in-process through the C ABI on one device.
"""
from __future__ import annotations

import hashlib
import json
import os
import time
from pathlib import Path

from .engine import NativeGraph
from .graph_definition import GraphDefinition, from_cayleypy

_BACKEND_NAMES = {"bitmap": "B200_PERMUTATION_BITMAP", "hash": "B200_EXACT_ALL_VISITED_HASH",
                  "hash3": "B200_THREE_LAYER_BANK_HASH"}
_STRATEGY_TO_DEDUP = {"atomic": "atomic", "warp": "warp", "batch": "sort", "bucket": "bucket"}


def _normalize_memory_backend(name):
    if name in ("segmented", "segmented32", "segmented24"):
        return "segmented24"
    if name in ("legacy", "permutation_bitmap"):
        return name
    raise ValueError("INVALID_MEMORY_BACKEND")


def _normalize_segment_strategy(name):
    if name not in ("atomic", "warp", "batch", "bucket"):
        raise ValueError("INVALID_SEGMENT_STRATEGY")
    return name


def _receipt(output: Path, digest: str) -> dict:
    """The receipt checks of launch.py:77-82."""
    report = json.loads((output / "report.json").read_text(encoding="utf-8"))
    if report["graph_digest"] != digest:
        raise RuntimeError("GRAPH_RECEIPT_IDENTITY_MISMATCH")
    if report["status"] not in ("COMPLETE", "INCOMPLETE"):
        raise RuntimeError("GRAPH_RECEIPT_STATUS")
    if hashlib.sha256((output / "states.json").read_bytes()).hexdigest() != report["states_sha256"]:
        raise RuntimeError("GRAPH_RECEIPT_CHECKSUM")
    return report


def select_visited(memory_backend: str, graph: GraphDefinition) -> str:
    """memory_backend -> visited set: legacy lets the planner choose; segmented24
    keeps an exact hash (three-layer banks when inverse-closed);
    permutation_bitmap is the exact rank bitmap."""
    if memory_backend == "permutation_bitmap":
        return "bitmap"
    if memory_backend == "segmented24":
        return "hash3" if graph.inverse_closed() else "hash"
    return "auto"


def run_graph(graph, output, *, device=None, devices=None, capacity=None, max_seconds=None, executable=None,
              shards=None, autotune=True, backend="auto", memory_backend="legacy", segment_rows=None,
              memory_preset="balanced", segment_strategy=None, peer_transport="auto", transport="auto",
              candidate_order="auto", bitmap_owner_page=None, planner="plain", visited=None, dedup=None,
              max_layers=None, cancel_flag=None):
    """Exact BFS of ``graph`` on one GPU; writes ``output``/report.json and
    states.json and returns the report dict.  Failures raise; there is no CPU
    restart."""
    if not isinstance(graph, GraphDefinition):
        graph = from_cayleypy(graph)
    if device is not None and devices is not None:
        raise ValueError("DEVICE_SELECTION_CONFLICT")
    if device is not None:
        if type(device) is not int or device < 0:
            raise ValueError("INVALID_DEVICE")
        devices = [device]
    if devices is not None and (not isinstance(devices, (list, tuple)) or not devices
                                or any(type(v) is not int or v < 0 for v in devices)
                                or len(set(devices)) != len(devices)):
        raise ValueError("INVALID_DEVICES")
    if devices is not None and len(devices) > 1:
        raise ValueError("MULTI_DEVICE_NOT_BUILT: this engine runs one BFS per GPU")
    if max_seconds is not None and (type(max_seconds) is not int or max_seconds < 1):
        raise ValueError("INVALID_MAX_SECONDS")
    if shards is not None and (type(shards) is not int or not 1 <= shards <= 4096):
        raise ValueError("INVALID_SHARDS")
    if type(autotune) is not bool:
        raise ValueError("INVALID_AUTOTUNE")
    if segment_rows is not None and (type(segment_rows) is not int or not 1 <= segment_rows <= 1 << 32):
        raise ValueError("INVALID_SEGMENT_ROWS")
    if bitmap_owner_page is not None and (type(bitmap_owner_page) is not int or bitmap_owner_page < 0
                                          or bitmap_owner_page > 1 << 20
                                          or (bitmap_owner_page and bitmap_owner_page & (bitmap_owner_page - 1))):
        raise ValueError("INVALID_BITMAP_OWNER_PAGE")
    if backend not in ("auto", "generic", "shard_ab_hash", "shard_ab_sort_merge"):
        raise ValueError("INVALID_BACKEND")
    memory_backend = _normalize_memory_backend(memory_backend)
    if bitmap_owner_page and memory_backend != "permutation_bitmap":
        raise ValueError("BITMAP_OWNER_PAGE_REQUIRES_BITMAP")
    if segment_strategy is None:
        segment_strategy = os.environ.get("MGBFS_SEGMENT_STRATEGY", "atomic")
    segment_strategy = _normalize_segment_strategy(segment_strategy)
    if memory_backend == "legacy" and segment_strategy != "atomic":
        raise ValueError("SEGMENT_STRATEGY_REQUIRES_SEGMENTED_BACKEND")
    if memory_preset not in ("balanced", "max_capacity"):
        raise ValueError("INVALID_MEMORY_PRESET")
    if memory_backend == "permutation_bitmap":
        if graph.action["kind"] != "permutation":
            raise ValueError("BITMAP_REQUIRES_PERMUTATION_ACTION")
        if not 1 <= len(graph.start) <= 64:
            raise ValueError("BITMAP_UNSUPPORTED_DEGREE")
    if peer_transport not in ("auto", "host", "lsa"):
        raise ValueError("INVALID_PEER_TRANSPORT")
    if transport not in ("auto", "full", "parent"):
        raise ValueError("INVALID_TRANSPORT")
    if candidate_order not in ("auto", "none", "radix"):
        raise ValueError("INVALID_CANDIDATE_ORDER")
    if capacity is not None and (type(capacity) is not int or capacity < 1):
        raise ValueError("INVALID_CAPACITY")
    if planner not in ("plain", "learned"):
        raise ValueError("INVALID_PLANNER")
    output = Path(output).absolute()
    if output.exists():
        raise FileExistsError(output)
    if visited is None:
        visited = select_visited(memory_backend, graph)
    if dedup is None:
        dedup = "auto" if memory_backend == "legacy" else _STRATEGY_TO_DEDUP[segment_strategy]
        if dedup == "atomic" and memory_backend == "legacy":
            dedup = "auto"
    dev = devices[0] if devices else 0
    digest = graph.digest()
    setup_started = time.perf_counter()
    tuned = {"enabled": autotune, "source": None}
    shapes = {}
    if autotune and visited == "auto" and dedup == "auto" and shards is None:
        # Only a plan the caller left open is tuned, within min(60, max_seconds // 3)
        # seconds that come off the run's deadline (multigpubfs/launch.py:277-290).
        from . import autotune as tuner
        budget = 60 if max_seconds is None else min(60, max(1, max_seconds // 3))
        t0 = time.perf_counter()
        prof = tuner.choose_profile(graph, dev, budget_seconds=budget)
        if max_seconds is not None:
            max_seconds = max(1, int(max_seconds - (time.perf_counter() - t0)))
        tuned = {"enabled": True, "source": prof["source"], "plan": prof["plan"]}
        visited = prof["plan"].get("visited", visited)
        dedup = prof["plan"].get("dedup", dedup)
        shards = prof["plan"].get("shards", shards)
        shapes = {k: prof["plan"][k] for k in ("group_chunk", "blocks_per_sm", "bucket_margin", "hash_load_percent")
                  if k in prof["plan"]}
    learned = {}
    if planner == "learned":
        # The prediction sizes and chooses; mgbfs2_plan rejects the learned
        # planner without one.
        from .planner import choose_path
        learned = choose_path(graph.to_dict(), device=dev)
    with NativeGraph(graph, dev) as engine:
        plan = engine.plan(visited=visited, dedup=dedup, capacity=capacity, shards=shards, **shapes,
                           **(learned or {"planner": planner}))
        setup_seconds = time.perf_counter() - setup_started
        result = engine.run(max_seconds=max_seconds, max_layers=max_layers, cancel_flag=cancel_flag)
        current = engine.sample(0, 1000)
        previous = engine.sample(1, 1000)
    status = "COMPLETE" if result.complete else "INCOMPLETE"
    reason = result.reason
    if reason == "RESOURCE":
        reason = f"RESOURCE_{result.fatal}"
    states = {"schema": 2, "state_encoding": "signed_int64_vectors", "current": current,
              "previous_small": previous, "current_sample_limit": 1000}
    state_bytes = json.dumps(states, sort_keys=True, separators=(",", ":")).encode()
    bfs = max(result.bfs_seconds, 1e-12)
    report = {
        "schema": 2, "status": status, "reason": reason,
        "backend": _BACKEND_NAMES[plan["visited"]], "device": dev, "world": 1, "devices": [dev],
        "graph_digest": digest, "layer_sizes": result.layer_sizes, "layer_seconds": result.layer_seconds,
        "setup_seconds": setup_seconds, "bfs_seconds": result.bfs_seconds, "capacity": plan["capacity"],
        "arena_bytes": result.peak_device_bytes, "plan": plan, "state_bytes": 8 * plan["key_words"],
        "states_sha256": hashlib.sha256(state_bytes).hexdigest(),
        "retention": "current sample <=1000 and previous layer only if <1000",
        "scope": "single-device exact BFS, libmgbfs2 (sm_100a)",
        "successors": result.successors, "successors_per_second": result.successors / bfs,
        "states_per_second": result.states / bfs, "kernel_launches": result.kernel_launches,
        "redo_layers": result.redo_layers, "fatal_bits": result.fatal_names,
        "memory_backend": memory_backend, "segment_strategy": segment_strategy, "autotune": tuned,
        "planner": {"name": planner, **({k: learned[k] for k in ("predicted_states", "predicted_peak")}
                                        if learned else {})},
    }
    output.mkdir(parents=True)
    (output / "states.json").write_bytes(state_bytes)
    tmp = output / "report.json.tmp"
    tmp.write_text(json.dumps(report, indent=2))
    tmp.replace(output / "report.json")
    return _receipt(output, digest)
