"""Pilot-run autotuner: picks the visited-set path of one graph, then the
shapes of that path, by timing candidate plans on the graph's own first
layers, and caches the choice.

Mirrors the reference's tuning layer in what it decides and how (re-designed
for this engine's plans, not ported):

* size profiles (multigpubfs/size_profiles.py:40-56): graphs below
  ``PILOT_MIN_STATES`` states are not piloted; they take the fixed default plan;
* timed trials with a keep-the-default rule (generic_distributed_native.rs:186-266,
  multigpubfs/autotune.py:276): every candidate expands the same layer prefix,
  is timed on the device, and replaces the default plan only if it is at
  least ``MIN_GAIN`` (10 %) faster (autotune.py:263);
* a profile cache (multigpubfs/profile_cache.py) keyed by graph digest, device
  name and library build, so a graph is piloted once per machine.

Stage 1 candidates are the engine's exact paths for the graph: the plain
bitmap with per-lane or warp-merged atomics, owner-routed bucket layers with
one- or two-symbol shard prefixes, grouped claim-then-route layers, the
open-addressing hash and, for inverse-closed graphs, the three-bank hash.
Stage 2 varies the shapes of the path stage 1 kept (`shape_candidates`): the
work-item size and resident blocks per SM of grouped layers, the bucket
margin of routed layers, the growth threshold of the hash table, and the
resident blocks of the fused kernels; the stage-1 plan with default shapes is
the default trial.  Results never depend on the choice: every path and shape
is exact and only changes speed.

A batched sweep is tuned the same way (`choose_sweep_shape`): its tile size and
resident blocks per SM are timed on a spread sample of the sweep's instances,
every trial's layer tables must equal the default's, and the keep-the-default
rule and the cache apply.
"""
from __future__ import annotations

import json
import math
import os
import time
from pathlib import Path

from .graph_definition import GraphDefinition

PILOT_MIN_STATES = 1 << 24     # smaller graphs take the default plan
PILOT_WORK = 1 << 27           # successors expanded by each pilot (a layer prefix)
MIN_GAIN = 0.10                # a candidate must beat the default by this much
DEFAULT = {"visited": "auto", "dedup": "auto"}


def cache_path() -> Path:
    env = os.environ.get("MGBFS2_AUTOTUNE_CACHE")
    if env:
        return Path(env)
    return Path(os.environ.get("XDG_CACHE_HOME", Path.home() / ".cache")) / "multigpubfs_b200" / "autotune.json"


def _state_bound(graph: GraphDefinition) -> int:
    start = graph.start
    counts = {}
    for v in start:
        counts[v] = counts.get(v, 0) + 1
    return math.factorial(len(start)) // math.prod(math.factorial(c) for c in counts.values())


def candidate_plans(graph: GraphDefinition) -> list[dict]:
    """The plans the pilot compares, default first."""
    out = [dict(DEFAULT)]
    if graph.action["kind"] == "permutation":
        n = len(graph.start)
        distinct = len(set(graph.start)) == n
        out += [{"visited": "bitmap", "dedup": "atomic"}, {"visited": "bitmap", "dedup": "warp"}]
        if distinct and 2 <= n <= 16:
            out.append({"visited": "bitmap", "dedup": "bucket", "shards": 1})       # one-symbol prefix
            if n * (n - 1) <= 256:
                out.append({"visited": "bitmap", "dedup": "bucket", "shards": 256})  # two-symbol prefix
            out.append({"visited": "bitmap", "dedup": "grouped"})
    out.append({"visited": "hash", "dedup": "atomic"})
    if graph.inverse_closed():
        out.append({"visited": "hash3", "dedup": "atomic"})
    return out


def shape_candidates(plan: dict, resolved: dict) -> list[dict]:
    """Stage 2: shape variations of the plan stage 1 kept, default first.
    `resolved` is the plan info mgbfs2_plan returned for it (the path it
    resolved to when the request said auto)."""
    out = [dict(plan)]
    dedup, visited = resolved.get("dedup"), resolved.get("visited")
    if dedup == "grouped":
        for chunk in (2048, 4096, 8192):
            for blocks in (6, 8):
                if (chunk, blocks) != (4096, 8):
                    out.append(dict(plan, group_chunk=chunk, blocks_per_sm=blocks))
    elif dedup == "bucket":
        out += [dict(plan, bucket_margin=m) for m in (1024, 16384)]
    elif visited == "hash":
        out += [dict(plan, hash_load_percent=f) for f in (35, 70)]
        out.append(dict(plan, parents_per_thread=2 if resolved.get("parents_per_thread", 4) in (1, 4) else 1))
        out += [dict(plan, blocks_per_sm=b) for b in (4, 8)]
    elif visited == "bitmap":
        out += [dict(plan, blocks_per_sm=b) for b in (3, 6)]
        out.append(dict(plan, parents_per_thread=2 if resolved.get("parents_per_thread", 4) == 4 else 4))
    return out


def cache_key(graph: GraphDefinition, device_name: str, build: str) -> str:
    return f"{graph.digest()}|{device_name}|{build}"


def load_cache(path: Path) -> dict:
    try:
        return json.loads(path.read_text())
    except (OSError, ValueError):
        return {}


def store_cache(path: Path, cache: dict) -> None:
    path.parent.mkdir(parents=True, exist_ok=True)
    tmp = path.with_suffix(".tmp")
    tmp.write_text(json.dumps(cache, indent=1, sort_keys=True))
    tmp.replace(path)


def pick(trials: list[dict], min_gain: float = MIN_GAIN) -> dict:
    """Keep-the-default rule over timed trials ({"plan", "seconds"}; the first
    trial is the default; failed trials have seconds None)."""
    default = trials[0]
    ok = [t for t in trials if t["seconds"] is not None]
    if not ok:
        return default["plan"]
    best = min(ok, key=lambda t: t["seconds"])
    if default["seconds"] is None or best["seconds"] <= default["seconds"] * (1.0 - min_gain):
        return best["plan"]
    return default["plan"]


def pilot_depth(layer_sizes: list[int], gens: int, work: int = PILOT_WORK) -> int:
    """Layers a pilot expands: the shortest prefix whose successors reach
    `work` (all layers if the search is smaller)."""
    total = 0
    for d, s in enumerate(layer_sizes):
        total += s * gens
        if total >= work:
            return d + 1
    return len(layer_sizes)


def _run_pilot(graph, plan, device, max_layers, max_seconds, info=None):
    from .engine import NativeGraph
    from . import native
    try:
        with NativeGraph(graph, device) as eng:
            resolved = eng.plan(**plan)
            if info is not None:
                info.update(resolved)
            eng.run(max_layers=max_layers, max_seconds=max_seconds)   # warm: pool memory, module load
            r = eng.run(max_layers=max_layers, max_seconds=max_seconds)
            return r
    except native.NativeError:
        return None


def _trials(graph, plans, device, depth, per_trial, first, started, budget_seconds):
    trials = []
    for plan in plans:
        if time.perf_counter() - started > budget_seconds:
            break
        r = _run_pilot(graph, plan, device, depth, per_trial)
        ok = r is not None and r.layer_sizes[:depth] == first.layer_sizes[:depth] and len(r.layer_sizes) >= depth
        trials.append({"plan": plan, "seconds": r.device_seconds if ok else None})
    return trials


def choose_profile(graph: GraphDefinition, device: int = 0, *, budget_seconds: float = 60.0,
                   cache: Path | None = None, use_cache: bool = True) -> dict:
    """The plan for `graph` on `device`: from the cache, or by pilot runs.

    Returns {"plan": {...}, "source": "size"|"cache"|"pilot", "trials": [...]}."""
    if _state_bound(graph) < PILOT_MIN_STATES:
        return {"plan": dict(DEFAULT), "source": "size", "trials": []}
    import torch
    from . import native
    device_name = torch.cuda.get_device_name(device)
    stamp = Path(native.LIBRARY).with_suffix(".stamp")
    build = stamp.read_text().strip()[:16] if stamp.exists() else "unbuilt"
    path = cache or cache_path()
    key = cache_key(graph, device_name, build)
    entries = load_cache(path) if use_cache else {}
    if key in entries:
        return {"plan": entries[key]["plan"], "source": "cache", "trials": entries[key].get("trials", [])}
    started = time.perf_counter()
    plans = candidate_plans(graph)
    per_trial = max(1.0, budget_seconds / (2 * len(plans)))
    # The default plan's pilot fixes the layer prefix every candidate expands.
    first = _run_pilot(graph, plans[0], device, None, per_trial)
    if first is None:
        return {"plan": dict(DEFAULT), "source": "pilot", "trials": []}
    depth = pilot_depth(first.layer_sizes, graph.generator_count)
    trials = _trials(graph, plans, device, depth, per_trial, first, started, budget_seconds)
    choice = pick(trials)
    # Stage 2: the shapes of the kept path, with the same rule.
    resolved = {}
    if _run_pilot(graph, choice, device, 1, per_trial, info=resolved) is not None:
        shapes = shape_candidates(choice, resolved)
        if len(shapes) > 1:
            shape_trials = _trials(graph, shapes, device, depth, per_trial, first, started, budget_seconds)
            choice = pick(shape_trials)
            trials += shape_trials
    if use_cache:
        entries = load_cache(path)
        entries[key] = {"plan": choice, "trials": trials, "pilot_layers": depth}
        store_cache(path, entries)
    return {"plan": choice, "source": "pilot", "trials": trials, "pilot_layers": depth}


SWEEP_SAMPLE = 64                  # instances a sweep pilot runs
SWEEP_SHAPES = [{}, {"tile_entries": 512}, {"tile_entries": 256}, {"blocks_per_sm": 3}, {"blocks_per_sm": 2}]


def sweep_sample(count: int, sample: int = SWEEP_SAMPLE) -> list[int]:
    """Indices of the instances a sweep pilot runs: `sample` of them spread
    evenly over the sweep (all of them for smaller sweeps)."""
    if count <= sample:
        return list(range(count))
    return sorted({(k * count) // sample for k in range(sample)})


def sweep_cache_key(graphs, device_name: str, build: str) -> str:
    import hashlib
    h = hashlib.sha256()
    for g in graphs:
        h.update(GraphDefinition.from_dict(g).digest().encode() if isinstance(g, dict) else g.digest().encode())
    return f"sweep:{h.hexdigest()[:32]}|{device_name}|{build}"


def choose_sweep_shape(graphs, device: int = 0, *, sample: int = SWEEP_SAMPLE, budget_seconds: float = 30.0,
                       cache: Path | None = None, use_cache: bool = True) -> dict:
    """The batched sweep's shape (keyword arguments of BatchSweep.run) for
    `graphs` on `device`: from the cache, or by timing SWEEP_SHAPES on a
    sample of the instances (each trial runs the sample twice and keeps the
    second device time; a trial whose tables differ from the default's is
    discarded).  Returns {"shape", "source", "trials", "sample"}."""
    import torch
    from . import native
    from .batch import BatchSweep
    graphs = list(graphs)
    device_name = torch.cuda.get_device_name(device)
    stamp = Path(native.LIBRARY).with_suffix(".stamp")
    build = stamp.read_text().strip()[:16] if stamp.exists() else "unbuilt"
    path = cache or cache_path()
    key = sweep_cache_key(graphs, device_name, build)
    entries = load_cache(path) if use_cache else {}
    if key in entries:
        return {"shape": entries[key]["shape"], "source": "cache", "trials": entries[key].get("trials", []),
                "sample": entries[key].get("sample", [])}
    picked = sweep_sample(len(graphs), sample)
    started = time.perf_counter()
    trials, expect = [], None
    with BatchSweep([graphs[i] for i in picked], device) as sweep:
        for shape in SWEEP_SHAPES:
            if trials and time.perf_counter() - started > budget_seconds:
                break
            try:
                sweep.run(**shape)
                status = sweep.run(**shape)
                tables = sweep.layer_tables()
            except native.NativeError:
                trials.append({"plan": shape, "seconds": None})
                continue
            if expect is None:
                expect = tables
            ok = status["complete_instances"] == status["instances"] and not status["fatal"] and tables == expect
            trials.append({"plan": shape, "seconds": status["device_seconds"] if ok else None})
    choice = pick(trials) if trials else {}
    if use_cache:
        entries = load_cache(path)
        entries[key] = {"shape": choice, "trials": trials, "sample": picked}
        store_cache(path, entries)
    return {"shape": choice, "source": "pilot", "trials": trials, "sample": picked}
