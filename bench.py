#!/usr/bin/env python
"""Benchmark of the exact BFS engine on B200s.  Prints ONE JSON line (rank 0).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl native|reference] [--workload NAME]

Workloads (one step = one pass of the workload):

* ``s13-lrx`` (default, the headline): the Cayley graph of S13 under L (cyclic
  left shift), R (cyclic right shift) and X (swap of positions 0, 1), full BFS
  from the identity: 13! = 6,227,020,800 states, 79 layers, 18,681,062,400
  successors, exact Lehmer-rank bitmap.  Every BFS's table is checked against
  the reference's shipped table.
* ``s14-lrx``: the same graph on 14 symbols, 14! = 87,178,291,200 states in 92
  layers (peak 4,595,217,203), on one GPU: grouped layers of 24,024 prefix
  groups; checked by its total and the reference's first 24 layers.
* ``s13-coxeter``: S13 under the adjacent transpositions s1..s12 (inverse-closed),
  checked against the Mahonian layer certificate.
* ``s11-lrx-hash``: S11 LRX through the exact-key open-addressing hash of all
  visited states, checked against the reference's packed-search table.
* ``sweep512``: 512 seeded instances (n in {7..10}, 2-3 random generators,
  directed and inverse-closed variants) in one batched run, every table
  checked against the oracle's fixture.  With N GPUs the instances are split
  between the ranks by exact work (g |G| per instance) and rank 0 checks the
  gathered tables.
* ``planner-s12``: learned vs plain planner on 128 S12 instances and on the
  held-out sweep; tables checked against the oracle's fixtures.
* ``s13-lrx-sharded``: the S13 LRX BFS split over the ranks by state ownership
  (an NCCL all-to-all of routed children per layer chunk; strong scaling),
  checked against the reference's table.

Keys of the line: ``value`` is successors/s with inputs resident, timed with
CUDA events on the launching stream over the K steps; ``e2e`` is the same
metric through the C ABI from host buffers (create -> plan -> run -> tables ->
destroy, every step, wall clock); ``roofline`` divides algorithmic bytes
B_alg = 16 N + 32 E p by the summed duration of the layer-expansion launches;
``cpu_baseline`` is the C oracle (a CPU restatement of the reference's exact
BFS) on all host cores over a bounded sample of the same workload.
``--impl reference`` times that CPU implementation alone (rank 0).
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

HBM_FALLBACK_GBS = 6650.0
SWEEP_SEED = 20261203
HELDOUT_SEED = SWEEP_SEED + 4096


def lrx(n):
    left = [(i + 1) % n for i in range(n)]
    right = [(i - 1) % n for i in range(n)]
    x = list(range(n))
    x[0], x[1] = x[1], x[0]
    return [left, right, x]


def coxeter(n):
    out = []
    for i in range(n - 1):
        g = list(range(n))
        g[i], g[i + 1] = g[i + 1], g[i]
        out.append(g)
    return out


WORKLOADS = {
    "s13-lrx": dict(n=13, gens=lrx(13), visited="bitmap", dedup="grouped",
                    desc="S13 LRX full BFS (L, R, X from identity; 6,227,020,800 states), exact Lehmer-rank bitmap"),
    "s14-lrx": dict(n=14, gens=lrx(14), visited="bitmap", dedup="auto",
                    desc="S14 LRX full BFS (87,178,291,200 states, 4.6e9 in the peak layer), exact Lehmer-rank "
                         "bitmap, grouped layers with 24,024 prefix groups and a memory-bounded spill"),
    "s13-coxeter": dict(n=13, gens=coxeter(13), visited="bitmap", dedup="grouped",
                        desc="S13 adjacent transpositions s1..s12 full BFS (6,227,020,800 states), exact bitmap"),
    "s11-lrx-hash": dict(n=11, gens=lrx(11), visited="hash", dedup="atomic",
                         desc="S11 LRX full BFS (39,916,800 states), exact-key open-addressing hash of all visited states"),
    "s10-coxeter": dict(n=10, gens=coxeter(10), visited="bitmap", dedup="auto",
                        desc="S10 adjacent transpositions full BFS (3,628,800 states), Lehmer bitmap; beside it the "
                             "reference's own GPU BFS of the same graph (gpu/cayley_bfs.cu) on the same B200"),
    "gl2-211-matrix": dict(matrix_p=211, visited="bitmap", dedup="auto",
                           desc="GL(2,211) on 2x2 int64 matrices mod 211 from the identity, 6 generators: "
                                "1,972,681,200 states, 99.5 % of the certified entry-space bound 211^4; packed "
                                "8-bit entries, mixed-radix bitmap"),
}
BATCHED = ("sweep512", "planner-s12", "s13-lrx-sharded")

# Bounded CPU samples (about 10-30 s of C-oracle work on a 16-core host): the
# layers run of each workload's sample; s11-lrx-hash runs whole, and sweep512
# runs its first 128 instances whole.
CPU_SAMPLE_LAYERS = {"s13-lrx": 32, "s13-coxeter": 20, "planner-s12": 17, "s14-lrx": 32}
# Past 13 symbols the oracle's bitmap (n!/8 bytes of host memory) gives way to
# its exact hash, sized for the sample.
CPU_SAMPLE_HASH_STATES = {"s14-lrx": 1 << 27}


def measured_peak():
    try:
        d = json.loads((ROOT / "MEASURED_PEAKS.json").read_text())
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return HBM_FALLBACK_GBS, "fallback"


def golden(name):
    return json.loads((ROOT / "tests" / "golden" / name).read_text())


def expected_layers(name, n):
    if name == "s13-lrx":
        return golden("lrx13_layers.json")["layers"]
    if name in ("s13-coxeter", "s10-coxeter"):
        sizes = [1]
        for i in range(1, n + 1):
            out, window = [], 0
            for j in range(len(sizes) + i - 1):
                if j < len(sizes):
                    window += sizes[j]
                if j >= i:
                    window -= sizes[j - i]
                out.append(window)
            sizes = out
        return sizes
    if name == "s11-lrx-hash":
        return golden("lrx_layers.json")["layers"]["11"]
    return None


def workload_graph(name):
    from multigpubfs_b200 import GraphDefinition
    w = WORKLOADS[name]
    if "matrix_p" in w:
        from multigpubfs_b200.workloads import gl2_graph
        return GraphDefinition.from_dict(gl2_graph(w["matrix_p"]))
    return GraphDefinition.permutation(w["gens"], list(range(w["n"])))


def matrix_sample(p, states=300_000):
    """The oracle's level BFS of GL(2, p) (oracle.graph_oracle.successor, one
    core) until the settled states pass `states`: (layer sizes, seconds)."""
    from oracle import graph_oracle as G
    from multigpubfs_b200.workloads import gl2_graph
    graph = gl2_graph(p)
    gens = len(graph["action"]["generators"])
    t = time.perf_counter()
    start = (1, 0, 0, 1)
    seen, layer, sizes = {start}, [start], [1]
    while layer and sum(sizes) < states:
        nxt = []
        for s in layer:
            for k in range(gens):
                c = tuple(G.successor(graph, list(s), k))
                if c not in seen:
                    seen.add(c)
                    nxt.append(c)
        layer = nxt
        if nxt:
            sizes.append(len(nxt))
    return sizes, time.perf_counter() - t


def generator_digest(graph):
    import hashlib
    text = json.dumps(graph["action"]["generators"], separators=(",", ":"))
    return hashlib.sha256(text.encode()).hexdigest()


def sweep_fixture(key, graphs):
    """The oracle's tables for `graphs` (tests/golden/sweep_tables.json), after
    checking that the seeded generators are the ones the fixture was made from."""
    fx = golden("sweep_tables.json")[key]
    digests = [generator_digest(g) for g in graphs]
    if digests != fx["generators_sha256"][:len(graphs)]:
        raise RuntimeError(f"{key}: generated instances differ from the fixture's")
    return fx["tables"]


class ClockSampler:
    """nvidia-smi clock / throttle-reason sampling during the timed region."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: str):
        self.gpu = gpu_index
        self.proc = None
        self.path = Path(os.environ.get("TMPDIR", "/tmp")) / f"mgbfs2-clocks-{os.getpid()}.csv"

    def __enter__(self):
        try:
            self.out = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.out,
                                         stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
        try:
            self.out.close()
        except Exception:
            pass

    def summary(self):
        try:
            rows = [r.split(",") for r in self.path.read_text().splitlines() if r.strip()]
            self.path.unlink()
        except Exception:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[1]))
                mx = float(r[2])
                for name, v in zip(names, r[5:9]):
                    if v.strip() == "Active":
                        reasons.add(name)
            except (ValueError, IndexError):
                continue
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


# ---------------------------------------------------------------------------
# CPU baseline: the C oracle on a bounded sample of the same workload.

def cpu_sample(name, threads=None):
    from oracle import packed_oracle as P
    from multigpubfs_b200 import workloads
    threads = threads or P.default_threads()
    P.library()
    if name == "s13-lrx-sharded":
        name = "s13-lrx"  # the same BFS, split or not
    t = time.perf_counter()
    succ = states = 0
    engine = "C oracle (restated reference exact BFS)"
    if name in WORKLOADS and "matrix_p" in WORKLOADS[name]:
        p = WORKLOADS[name]["matrix_p"]
        sizes, _ = matrix_sample(p)
        threads = 1
        states, succ = sum(sizes), 6 * sum(sizes)
        what = f"GL(2,{p}) layers 0-{len(sizes) - 1}"
        engine = "Python oracle level BFS (restated reference exact_layers, one core)"
    elif name in WORKLOADS:
        w = WORKLOADS[name]
        layers = CPU_SAMPLE_LAYERS.get(name)
        bitmap = w["visited"] == "bitmap" and name not in CPU_SAMPLE_HASH_STATES
        sizes, _, _ = P.packed_bfs(w["gens"], list(range(w["n"])), use_bitmap=bitmap, threads=threads,
                                   max_layers=layers or (1 << 16), partial=bool(layers),
                                   max_states=CPU_SAMPLE_HASH_STATES.get(name))
        states, succ = sum(sizes), len(w["gens"]) * sum(sizes)
        what = (f"{name} layers 0-{len(sizes) - 1}" if layers else f"{name} full BFS") + \
               f" ({'Lehmer bitmap' if bitmap else 'exact hash set'})"
    elif name == "sweep512":
        graphs = workloads.sweep(512)[:128]
        for g in graphs:
            sizes, _, _ = P.packed_bfs(g["action"]["generators"], g["start"], use_bitmap=True, threads=threads)
            states += sum(sizes)
            succ += len(g["action"]["generators"]) * sum(sizes)
        what = "the first 128 of the 512 sweep instances, full BFS each (Lehmer bitmap)"
    else:
        g = workloads.planner_instance(0)
        layers = CPU_SAMPLE_LAYERS[name]
        sizes, _, _ = P.packed_bfs(g["action"]["generators"], g["start"], use_bitmap=True, threads=threads,
                                   max_layers=layers, partial=True)
        states, succ = sum(sizes), len(g["action"]["generators"]) * sum(sizes)
        what = f"S12 planner instance 0, layers 0-{len(sizes) - 1} (Lehmer bitmap)"
    dt = time.perf_counter() - t
    return {"value": succ / dt, "unit": "successors/s", "cores": threads, "kind": "port",
            "sample": f"{what}: {states:,} states, {succ:,} successors, {engine}, {dt:.2f} s"}


def workload_desc(name):
    if name in WORKLOADS:
        return WORKLOADS[name]["desc"]
    if name == "sweep512":
        return ("batched sweep: 512 instances (256 seeds x directed / inverse-closed), n in {7,8,9,10}, 2-3 seeded "
                "random generators, exact per-instance Lehmer bitmaps")
    if name == "s13-lrx-sharded":
        return "S13 LRX full BFS (6,227,020,800 states) split over the ranks by state ownership"
    return "learned vs plain planner: 128 S12 instances (2-4 random generators plus inverses), whole device"


def reference_arm(args, rank):
    if rank != 0:
        return 0
    for _ in range(args.warmup):
        cpu_sample(args.workload)
    runs = [cpu_sample(args.workload) for _ in range(args.steps)]
    value = statistics.median(r["value"] for r in runs)
    line = {"metric": "successors/s", "value": value, "unit": "successors/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": None, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u64", "data": "synthetic",
            "config": {"workload": workload_desc(args.workload)},
            "impl": "reference",
            "cpu_baseline": {"value": value, "unit": "successors/s", "cores": runs[0]["cores"], "kind": "port",
                             "sample": runs[0]["sample"]},
            "e2e": {"value": value, "unit": "successors/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def gpu_index(local):
    visible = os.environ.get("CUDA_VISIBLE_DEVICES", "").split(",")
    return visible[local] if visible and visible[0] else str(local)


def roofline(b_alg, seconds, kernel, traffic=None, traffic_source=None, **extra):
    peak, peak_kind = measured_peak()
    achieved = b_alg / seconds / 1e9
    out = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
           "traffic": traffic, "peak_kind": peak_kind, "b_alg_bytes": b_alg, "kernel": kernel}
    if traffic_source:
        out["traffic_source"] = traffic_source
    out.update(extra)
    return out


# ---------------------------------------------------------------------------
# Batched sweep.

def bench_sweep(args, rank, world, local):
    """512 instances; with N ranks each runs a work-balanced share as its own
    waves (no collective on the data path) and rank 0 checks the gathered
    tables against the oracle's fixture."""
    import torch
    import torch.distributed as dist
    from datetime import timedelta
    from multigpubfs_b200 import native, replicas, workloads
    from multigpubfs_b200.batch import BatchSweep
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        dist.init_process_group("nccl", timeout=timedelta(seconds=300), device_id=dev)
    graphs = workloads.sweep(512)
    expect = sweep_fixture("sweep512", graphs)
    _, order = native.graph_statics([(g["action"]["generators"], g["start"]) for g in graphs])
    work = [len(g["action"]["generators"]) * int(s) for g, s in zip(graphs, order)]
    owner = replicas.partition_instances(work, world)
    ids = [i for i in range(len(graphs)) if owner[i] == rank]
    mine = [graphs[i] for i in ids]
    mine_expect = [expect[i] for i in ids]

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    with BatchSweep(mine, local) as sweep:
        for _ in range(args.warmup):
            sweep.run(host_loop=args.host_loop)
        assert sweep.layer_tables() == mine_expect, "sweep tables differ from the oracle fixture (warm-up)"
        barrier()
        with ClockSampler(gpu_index(local)) as clocks:
            runs = [sweep.run(host_loop=args.host_loop) for _ in range(args.steps)]
        barrier()
        tables = sweep.layer_tables()
    assert tables == mine_expect, "sweep tables differ from the oracle fixture (timed runs)"
    dev_s = sum(r["device_seconds"] for r in runs)
    succ = runs[0]["successors"]
    states = runs[0]["states"]
    launches = sum(r["kernel_launches"] for r in runs)

    # e2e: a fresh batch from host graph descriptions every step.
    e2e = []
    h2d = sum(8 * len(g["start"]) + 4 * len(g["start"]) * len(g["action"]["generators"]) for g in mine)
    d2h = 0
    for i in range(args.steps + 1):
        barrier()
        t0 = time.perf_counter()
        with BatchSweep(mine, local) as sweep:
            sweep.run(host_loop=args.host_loop)
            got = sweep.layer_tables()
        torch.cuda.synchronize()
        if i:
            e2e.append(time.perf_counter() - t0)
        assert got == mine_expect
        d2h = 8 * sum(len(t) for t in got)
    e2e_s = sum(e2e) / len(e2e)

    total_succ, dev_max, e2e_max = succ, dev_s, e2e_s
    if world > 1:
        # The job's time is the slowest rank's; its work is every rank's.
        t = torch.tensor([dev_s, e2e_s], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        n = torch.tensor([succ], dtype=torch.int64, device=dev)
        dist.all_reduce(n, op=dist.ReduceOp.SUM)
        dev_max, e2e_max, total_succ = float(t[0].item()), float(t[1].item()), int(n.item())
        gathered = replicas.gather_tables(ids, tables, len(graphs), device=dev)
        if rank == 0:
            assert gathered == expect, "gathered sweep tables differ from the oracle fixture"
    if rank == 0:
        all_states = sum(map(sum, expect))
        line = {"metric": "successors/s", "value": total_succ * args.steps / dev_max, "unit": "successors/s",
                "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": dev_max / args.steps * 1e3, "higher_is_better": True,
                "scaling": "strong" if world > 1 else "weak", "vs_baseline": None, "dtype": "u64",
                "data": "synthetic",
                "config": {"workload": workload_desc("sweep512"), "instances": len(graphs),
                           "states_per_step": all_states, "successors_per_step": total_succ,
                           "parallelism": f"instances split over {world} rank(s) by g|G|" if world > 1 else "1 GPU",
                           "l2": "per-instance bitmaps and frontiers together exceed L2 (about 0.3 GB per step)"},
                "settled_states_per_s": all_states * args.steps / dev_max,
                "wall_ms_per_step": sum(r["seconds"] for r in runs) / len(runs) * 1e3,
                "e2e": {"value": total_succ / e2e_max, "unit": "successors/s", "h2d_bytes_per_step": h2d,
                        "d2h_bytes_per_step": d2h},
                "roofline": roofline(16 * states + 32 * succ, dev_s / args.steps,
                                     "batch_wave (one persistent cooperative launch per wave)", traffic=None),
                "waves": runs[0]["waves"], "layer_steps": runs[0]["layer_steps"],
                "gpu_launches": launches, "clocks": clocks.summary()}
        if world == 1 and not args.no_cpu_baseline:
            line["cpu_baseline"] = cpu_sample("sweep512")
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def bench_planner(args, local):
    """Learned vs plain planner on batched sweeps.  The network is fitted by
    the library's kernels on 4/5 of the layer tables of the 512-instance sweep
    plus 32 S11 / S12 instances on other seeds, and its capacity margin is
    calibrated on the other 1/5.  The plain run reserves each instance's orbit
    bound n!, the learned run its predicted peak times the margin (a layer
    that outgrows it is redone in a larger segment); both must give the
    oracle's tables.  Scenarios: 128 S12 instances with the whole device, and
    the held-out 512-instance sweep under 1 GiB and 256 MiB budgets.  The
    learned wall time includes the prediction."""
    import torch
    from multigpubfs_b200 import native, workloads
    from multigpubfs_b200.batch import BatchSweep
    from multigpubfs_b200.planner import (PlannerNet, calibrate_margin, predicted_capacities, rollout_device,
                                          training_set)
    torch.cuda.set_device(local)
    t0 = time.perf_counter()
    train = workloads.sweep(512) + [workloads.planner_instance(i, n=n, seed_base=20261204 + 50000 + 100 * n)
                                    for n in (11, 12) for i in range(16)]
    with BatchSweep(train, local) as sw:
        sw.run()
        tables = sw.layer_tables()
    assert tables[:512] == sweep_fixture("sweep512", train[:512]), "training tables differ from the oracle fixture"
    fit_ids = [i for i in range(len(train)) if i % 5]
    cal_ids = [i for i in range(len(train)) if i % 5 == 0]
    X, T = training_set([train[i] for i in fit_ids], [tables[i] for i in fit_ids])
    net = PlannerNet(local, seed=0)
    hist = net.fit(X, T, steps=2000, lr=3e-3)
    margin = calibrate_margin(net, [train[i] for i in cal_ids], [tables[i] for i in cal_ids])
    train_s = time.perf_counter() - t0
    s12 = [workloads.planner_instance(i) for i in range(args.instances)]
    heldout = workloads.sweep(512, seed_base=HELDOUT_SEED)
    s12_fixture = golden("sweep_tables.json")["planner_s12"]
    scenarios = [
        ("s12", f"{args.instances} S12 instances, 2-4 seeded random generators plus inverses, whole device", s12,
         None),
        ("sweep_heldout_1gib", "512-instance sweep on held-out seeds, n in {7,8,9,10}, 1 GiB memory budget",
         heldout, 1 << 30),
        ("sweep_heldout_256mib", "512-instance sweep on held-out seeds, n in {7,8,9,10}, 256 MiB memory budget",
         heldout, 1 << 28),
    ]

    def check(name, graphs, got):
        # Every table against the oracle: the fixture where it has one, and
        # the exact state count |G| (host Schreier-Sims) for every instance.
        if name == "s12":
            for k, i in enumerate(s12_fixture["indices"]):
                if i < len(graphs):
                    assert generator_digest(graphs[i]) == s12_fixture["generators_sha256"][k]
                    assert got[i] == s12_fixture["tables"][k], f"S12 instance {i} differs from the oracle fixture"
            _, states = native.graph_statics([(g["action"]["generators"], g["start"]) for g in graphs])
            assert [sum(t) for t in got] == [int(s) for s in states], "S12 state counts differ from |G|"
        else:
            assert got == sweep_fixture("sweep512_heldout", graphs), f"{name}: tables differ from the oracle fixture"

    keys = ("seconds", "device_seconds", "waves", "redo_layers", "redo_instances", "states", "successors")
    report, same_all = {}, True
    for name, desc, graphs, budget in scenarios:
        t1 = time.perf_counter()
        caps = predicted_capacities(net, graphs, margin=margin)
        predict_s = time.perf_counter() - t1
        with BatchSweep(graphs, local) as sw:
            sw.run(memory_bytes=budget)  # warm-up: pool memory, module load
            runs = {"plain": [], "learned": []}
            for _ in range(max(1, args.steps)):
                for arm, capacities in (("plain", None), ("learned", caps)):
                    st = sw.run(capacities=capacities, memory_bytes=budget)
                    st["layer_tables"] = sw.layer_tables()
                    runs[arm].append(st)
        out = {}
        for arm, rs in runs.items():
            assert all(r["layer_tables"] == rs[0]["layer_tables"] for r in rs)
            check(name, graphs, rs[0]["layer_tables"])
            out[arm] = sorted(rs, key=lambda r: r["seconds"])[len(rs) // 2]
        same = out["plain"]["layer_tables"] == out["learned"]["layer_tables"]
        same_all &= same
        peaks = [max(t) for t in out["plain"]["layer_tables"]]
        peaks_pred, _, _ = rollout_device(net, graphs)
        logr = sorted(math.log(q / max(1.0, p)) for p, q in zip(peaks_pred, peaks))
        learned_wall = out["learned"]["seconds"] + predict_s
        report[name] = {
            "workload": desc, "instances": len(graphs), "memory_budget_bytes": budget, "identical_tables": same,
            "oracle_checked": True,
            "plain": {k: out["plain"][k] for k in keys},
            "learned": dict({k: out["learned"][k] for k in keys}, predict_seconds=predict_s,
                            wall_with_prediction=learned_wall),
            "speedup_wall": out["plain"]["seconds"] / learned_wall,
            "reserved_frontier_words": {"plain": sum(math.factorial(len(g["start"])) for g in graphs),
                                        "learned": sum(caps)},
            "peak_log_true_over_predicted": {"median_abs": sorted(abs(x) for x in logr)[len(logr) // 2],
                                             "min": logr[0], "max": logr[-1]}}
    main_s = report["s12"]
    learned = main_s["learned"]
    line = {"metric": "successors/s", "value": learned["successors"] / learned["device_seconds"],
            "unit": "successors/s", "n_gpus": 1, "steps": max(1, args.steps), "warmup": 1,
            "ms_per_step": learned["device_seconds"] * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u64", "data": "synthetic",
            "config": {"workload": "learned vs plain planner on batched sweeps (value: S12 scenario, learned, "
                                   "device time; e2e: its wall time with the prediction)"},
            "e2e": {"value": learned["successors"] / learned["wall_with_prediction"], "unit": "successors/s",
                    "h2d_bytes_per_step": sum(8 * 12 + 4 * 12 * len(g["action"]["generators"]) for g in s12),
                    "d2h_bytes_per_step": 8 * sum(len(t) for t in s12_fixture["tables"])},
            "roofline": roofline(16 * learned["states"] + 32 * learned["successors"], learned["device_seconds"],
                                 "batch_wave (S12 scenario, learned capacities)"),
            "identical_tables": same_all, "scenarios": report,
            "predictor": {"train_rows": int(len(X)), "loss_first": hist[0], "loss_last": hist[-1],
                          "train_seconds": train_s, "margin": margin}}
    if not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_sample("planner-s12")
    print(json.dumps(line), flush=True)
    return 0 if same_all else 1


# ---------------------------------------------------------------------------
# Single-graph workloads.

def bench_single(args, rank, world, local):
    import torch
    import torch.distributed as dist
    from datetime import timedelta
    from multigpubfs_b200 import GraphDefinition
    from multigpubfs_b200.engine import NativeGraph

    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=timedelta(seconds=300), device_id=torch.device("cuda", local))
    w = WORKLOADS[args.workload]
    visited = args.visited or w["visited"]
    dedup = args.dedup or w["dedup"]
    graph = workload_graph(args.workload)
    expect = expected_layers(args.workload, w.get("n"))
    if args.workload == "s14-lrx":
        # No whole S14 table ships with the reference: 14! states in all, and
        # the first 24 layers of the reference's own CPU search.
        prefix = golden("lrx14_prefix.json")["layers"]

        def table_ok(sizes):
            return sum(sizes) == math.factorial(14) and sizes[:len(prefix)] == prefix
    elif expect is None:
        # GL(2, p): the group order, and the oracle's first layers.
        p = w["matrix_p"]
        order = (p * p - 1) * (p * p - p)
        prefix, _ = matrix_sample(p, 50_000)

        def table_ok(sizes):
            return sum(sizes) == order and sizes[:len(prefix) - 1] == prefix[:-1]
    else:
        def table_ok(sizes):
            return sizes == expect

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    # ---- value: resident engine, K whole BFS runs ------------------------------------
    eng = NativeGraph(graph, local)
    plan = eng.plan(visited=visited, dedup=dedup, host_loop=args.host_loop)
    for _ in range(args.warmup):
        r = eng.run()
        assert table_ok(r.layer_sizes), "layer table mismatch in warm-up"
    results = []
    barrier()
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(gpu_index(local)) as clocks:
        start.record()
        wall0 = time.perf_counter()
        for _ in range(args.steps):
            results.append(eng.run())
        stop.record()
        barrier()
        wall = time.perf_counter() - wall0
    device_s = start.elapsed_time(stop) * 1e-3
    # The engine runs on its own stream and each run() returns after its
    # stream is done, so the torch events bracket the whole K runs; the
    # engine's own CUDA-event time of each run is summed beside it.
    engine_s = sum(r.device_seconds for r in results)
    for r in results:
        assert r.complete and table_ok(r.layer_sizes), "layer table mismatch in a timed run"
    device_max = device_s
    if world > 1:
        # Replicas: every rank must hold the same table; the job time is the slowest rank's.
        from multigpubfs_b200 import replicas
        view = replicas.exchange(results[0].layer_sizes, device_s, results[0].successors * args.steps,
                                 device=torch.device("cuda", local))
        device_max = view["device_seconds_max"]
    succ = results[0].successors
    states = results[0].states
    tests = results[0].visited_tests
    kernel_s = sum(r.kernel_seconds for r in results) / len(results)
    launches = sum(r.kernel_launches for r in results)
    # The hash's probes per visited test, measured on the final table: every
    # stored key's distance from its home slot plus one (mgbfs2_table_probes).
    probes = eng.table_probes()[0] if plan["visited"] == "hash" else 1.0
    eng.close()

    # ---- e2e: C-ABI handle from host buffers, every step ------------------------------
    e2e_times = []
    if "matrix_p" in w:
        h2d = 8 * 4 + 6 * (8 * 4 + 4) + 8
    else:
        h2d = 8 * w["n"] + 4 * w["n"] * len(w["gens"]) + 8
    d2h = 0
    for i in range(args.steps + 1):
        barrier()
        t0 = time.perf_counter()
        with NativeGraph(graph, local) as e:
            e.plan(visited=visited, dedup=dedup, host_loop=args.host_loop)
            r = e.run()
            sizes, _ = e.layer_table()
            cur = e.sample(0, 1000)
            prev = e.sample(1, 1000)
        torch.cuda.synchronize()
        if i:
            e2e_times.append(time.perf_counter() - t0)
        assert table_ok(sizes)
        d2h = 24 * len(sizes) + 16 * len(sizes) + 8 * len(graph.start) * (len(cur) + len(prev))
    e2e_t = torch.tensor([sum(e2e_times) / len(e2e_times)], dtype=torch.float64, device="cuda")
    if world > 1:
        dist.all_reduce(e2e_t, op=dist.ReduceOp.MAX)

    if rank == 0:
        b_alg = int(16 * states + 32 * succ * probes)
        traffic, source = None, None
        prof = ROOT / "profiles" / f"traffic_{args.workload}.json"
        if prof.exists():
            try:
                traffic = json.loads(prof.read_text()).get(plan["dedup"], {}).get("dram_bytes_per_bfs")
                source = f"ncu capture summarised in profiles/{prof.name}, not measured in this run"
            except Exception:
                traffic = None
        kernel_names = {"grouped": "expand_grouped (grouped layers; small layers expand_packed)",
                        "bucket": "route_lehmer + accept_lehmer (bucketed layers; small layers expand_packed)"}
        line = {
            "metric": "successors/s",
            "value": world * succ * args.steps / device_max,
            "unit": "successors/s",
            "n_gpus": world,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": device_max / args.steps * 1e3,
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "u64",
            "data": "synthetic",
            "config": {"workload": w["desc"], "visited": plan["visited"], "dedup": plan["dedup"],
                       "planner": plan["planner"], "parallelism": f"replicas{world}" + (
                           " (each GPU runs the whole BFS; the BFS itself is not split)" if world > 1 else ""),
                       "states_per_bfs": states, "successors_per_bfs": succ, "visited_tests_per_bfs": tests,
                       "l2": "working set larger than L2 (%s)" % (
                           "bitmap %d MB, frontiers up to several GB" % (plan["bitmap_bits"] // 8 // (1 << 20))
                           if plan["visited"] == "bitmap" else
                           "table of %d slots = %d MB" % (plan["table_slots"],
                                                          plan["table_slots"] * plan["table_slot_bytes"] >> 20))},
            "settled_states_per_s": world * states * args.steps / device_max,
            "wall_ms_per_step": wall / args.steps * 1e3,
            "engine_ms_per_step": engine_s / args.steps * 1e3,
            "kernel_ms_per_step": kernel_s * 1e3,
            "e2e": {"value": world * succ / float(e2e_t.item()), "unit": "successors/s",
                    "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
            "roofline": roofline(b_alg, kernel_s,
                                 kernel_names.get(plan["dedup"], "expand_packed (fused layer expansion)"),
                                 traffic=traffic, traffic_source=source,
                                 **({"probes_per_test": round(probes, 4),
                                     "probes_source": "mean over the final table's keys (mgbfs2_table_probes)",
                                     "table_slot_bytes": plan["table_slot_bytes"]}
                                    if plan["visited"] == "hash" else {})),
            "gpu_launches": launches,
            "clocks": clocks.summary(),
        }
        if world == 1 and not args.no_cpu_baseline:
            line["cpu_baseline"] = cpu_sample(args.workload)
        if args.workload == "s10-coxeter":
            line["same_box_reference_gpu"] = reference_gpu_leg(w["n"], expect, succ, args)
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def reference_gpu_leg(n, expect, succ, args):
    """The reference's own GPU BFS of S_n under adjacent transpositions
    (gpu/cayley_bfs.cu, built into oracle/_ref), timed on this B200: its
    warp-aggregated variant, one host-driven step per layer, tables checked."""
    from oracle import ref_gpu
    if not ref_gpu.available():
        return {"unavailable": "oracle/_ref/libmgbfs_ref_gpu.so not built (reference sources absent at build)"}
    with ref_gpu.CayleyBfs(n) as ref:
        for _ in range(args.warmup):
            sizes, _, _ = ref.run(1, 0)
            assert sizes == expect, "reference GPU table differs"
        runs = [ref.run(1, 0) for _ in range(args.steps)]
    assert all(r[0] == expect for r in runs)
    kernel_s = sum(r[1] for r in runs) / len(runs) * 1e-3
    wall_s = sum(r[2] for r in runs) / len(runs)
    return {"value": succ / wall_s, "unit": "successors/s", "kernel_only_value": succ / kernel_s,
            "ms_per_bfs": wall_s * 1e3, "kernel_ms_per_bfs": kernel_s * 1e3,
            "code": "reference gpu/cayley_bfs.cu expand_kernel (warp-aggregated variant, one step per layer), "
                    "compiled for sm_100a from the reference sources"}


def bench_sharded(args, rank, world, local):
    """One S13 LRX BFS split over the ranks by state ownership
    (multigpubfs_b200.sharded): each rank owns a slice of the bitmap, children
    are routed to their owners and exchanged with an NCCL all-to-all per layer
    chunk.  One rank (no torchrun) runs the same loop over a one-rank NCCL
    group.  Strong scaling: the total work is one BFS whatever N is."""
    import socket
    import torch
    import torch.distributed as dist
    from datetime import timedelta
    from multigpubfs_b200 import GraphDefinition, sharded
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world == 1 and "MASTER_ADDR" not in os.environ:
        with socket.socket() as sock:
            sock.bind(("127.0.0.1", 0))
            port = sock.getsockname()[1]
        os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK="0", WORLD_SIZE="1")
    dist.init_process_group("nccl", timeout=timedelta(seconds=300), device_id=dev)
    n, gens = 13, lrx(13)
    graph = GraphDefinition.permutation(gens, list(range(n)))
    expect = expected_layers("s13-lrx", n)
    chunk = 1 << 26

    def barrier():
        dist.barrier()
        torch.cuda.synchronize()

    shard = sharded.DeviceShard(graph, rank, world, dev, chunk_parents=chunk)
    bfs = sharded.ShardedBfs([shard], sharded.DistExchange(None, dev))
    for _ in range(args.warmup):
        shard.reset()
        assert bfs.run() == expect, "layer table mismatch in warm-up"
    barrier()
    shard.launches = 0
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    tables = []
    with ClockSampler(gpu_index(local)) as clocks:
        start.record()
        for _ in range(args.steps):
            shard.reset()
            tables.append(bfs.run())
        stop.record()
        barrier()
    device_s = start.elapsed_time(stop) * 1e-3
    launches = shard.launches
    assert all(t == expect for t in tables), "layer table mismatch in a timed run"
    del bfs, shard
    torch.cuda.empty_cache()

    # e2e: shards built from the host graph every step.
    e2e = []
    for i in range(args.steps + 1):
        barrier()
        t0 = time.perf_counter()
        s = sharded.DeviceShard(graph, rank, world, dev, chunk_parents=chunk)
        got = sharded.ShardedBfs([s], sharded.DistExchange(None, dev)).run()
        del s
        torch.cuda.synchronize()
        if i:
            e2e.append(time.perf_counter() - t0)
        assert got == expect
    t = torch.tensor([device_s, sum(e2e) / len(e2e)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    device_max, e2e_max = float(t[0].item()), float(t[1].item())
    if rank == 0:
        states = sum(expect)
        succ = len(gens) * states
        geo = sharded.geometry(n, world)
        line = {
            "metric": "successors/s", "value": succ * args.steps / device_max, "unit": "successors/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": device_max / args.steps * 1e3, "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None, "dtype": "u64", "data": "synthetic",
            "config": {"workload": "S13 LRX full BFS (6,227,020,800 states) split over the ranks by state "
                                   "ownership: prefix blocks of two Lehmer digits, block s on rank s mod N",
                       "parallelism": f"owner-partitioned bitmap over {world} rank(s), NCCL all-to-all per chunk",
                       "slice_bits_per_rank": geo.slice_bits, "chunk_parents": chunk,
                       "states_per_bfs": states, "successors_per_bfs": succ,
                       "l2": "bitmap slices and frontiers larger than L2 at N <= 4"},
            "settled_states_per_s": states * args.steps / device_max,
            "e2e": {"value": succ / e2e_max, "unit": "successors/s", "h2d_bytes_per_step": 8 * n + 4 * n * 3,
                    "d2h_bytes_per_step": 8 * len(expect)},
            "roofline": roofline(16 * states + 32 * succ, device_max / args.steps,
                                 "count_lehmer + route_lehmer + accept_lehmer (owner-partitioned), timed as the "
                                 "whole step including the exchange"),
            "gpu_launches": launches,
            "clocks": clocks.summary(),
        }
        if world == 1 and not args.no_cpu_baseline:
            line["cpu_baseline"] = cpu_sample("s13-lrx")
        print(json.dumps(line), flush=True)
    dist.barrier()
    dist.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["native", "reference"], default="native")
    ap.add_argument("--workload", choices=sorted(WORKLOADS) + list(BATCHED), default="s13-lrx")
    ap.add_argument("--host-loop", action="store_true",
                    help="layers as separate kernel launches with a host round trip each (for a profiler); "
                         "by default a wave of the sweep, or a fused BFS, is one persistent launch")
    ap.add_argument("--instances", type=int, default=128, help="planner-s12: number of S12 instances")
    ap.add_argument("--dedup", default=None)
    ap.add_argument("--visited", default=None)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return reference_arm(args, rank)
    if args.workload == "sweep512":
        return bench_sweep(args, rank, world, local)
    if args.workload == "planner-s12":
        if world > 1 and rank != 0:
            return 0
        return bench_planner(args, local)
    if args.workload == "s13-lrx-sharded":
        return bench_sharded(args, rank, world, local)
    return bench_single(args, rank, world, local)


if __name__ == "__main__":
    sys.exit(main())
