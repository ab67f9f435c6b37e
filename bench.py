#!/usr/bin/env python
"""Benchmark: exact full BFS of S13 LRX on one B200 (one step = one whole BFS).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl native|reference] [--workload NAME]

Prints ONE JSON line (rank 0).  Workload (default ``s13-lrx``): the Cayley
graph of S13 under L (cyclic left shift), R (cyclic right shift) and X (swap
positions 0,1), from the identity: 13! = 6,227,020,800 states, 79 layers,
18,681,062,400 successors per BFS, exact Lehmer-rank bitmap visited set.  Every
timed BFS's layer table is checked against the reference's shipped table.

* ``value``: successors/s over the K timed BFS runs, device-timed with CUDA
  events bracketing the K runs (synchronised before and after), inputs
  resident; with N GPUs (torchrun) each rank runs its own replica (the BFS does
  not shard on one node in this build) and value = N * E / max-over-ranks time.
* ``e2e``: the same metric through the C-ABI handle from host buffers:
  create -> plan -> run -> layer table -> samples -> destroy, every step.
* ``roofline``: algorithmic bytes B_alg = 16*N + 32*E (8-byte packed states
  written once and read once; one 32-byte DRAM sector per visited test) over
  the summed duration of the layer-expansion kernel launches, against the
  measured HBM copy bandwidth.
* ``cpu_baseline``: the C oracle (a CPU restatement of the reference's exact
  BFS) on all host cores, over a bounded sample (the first 32 BFS layers of the
  same graph).
``--impl reference`` times that CPU implementation alone (rank 0).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

HBM_FALLBACK_GBS = 6650.0
CPU_SAMPLE_LAYERS = 32


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
    "s13-coxeter": dict(n=13, gens=coxeter(13), visited="bitmap", dedup="grouped",
                        desc="S13 adjacent transpositions s1..s12 full BFS (6,227,020,800 states), exact bitmap"),
    "s11-lrx-hash": dict(n=11, gens=lrx(11), visited="hash", dedup="atomic",
                         desc="S11 LRX full BFS (39,916,800 states), exact-key open-addressing hash of all visited states"),
}


def measured_peak():
    path = ROOT / "MEASURED_PEAKS.json"
    try:
        d = json.loads(path.read_text())
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return HBM_FALLBACK_GBS, "fallback"


def expected_layers(name, n):
    if name == "s13-lrx":
        return json.loads((ROOT / "tests/golden/lrx13_layers.json").read_text())["layers"]
    if name == "s13-coxeter":
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
        return json.loads((ROOT / "tests/golden/lrx_layers.json").read_text())["layers"]["11"]
    return None


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


def cpu_baseline(threads=None):
    """The C oracle on the first CPU_SAMPLE_LAYERS layers of S13 LRX, all host cores."""
    from oracle import packed_oracle as P
    threads = threads or P.default_threads()
    P.library()
    t = time.perf_counter()
    sizes, _, _ = P.packed_bfs(lrx(13), list(range(13)), use_bitmap=True, threads=threads,
                               max_layers=CPU_SAMPLE_LAYERS, partial=True)
    dt = time.perf_counter() - t
    succ = 3 * sum(sizes)
    return {"value": succ / dt, "unit": "successors/s", "cores": threads, "kind": "port",
            "sample": f"S13 LRX layers 0-{CPU_SAMPLE_LAYERS - 1} ({sum(sizes):,} states, {succ:,} successors), "
                      f"C oracle (restated reference exact BFS), {dt:.2f} s"}


def reference_arm(args, rank):
    if rank != 0:
        return 0
    name = args.workload
    for _ in range(args.warmup):
        cpu_baseline()
    runs = [cpu_baseline() for _ in range(args.steps)]
    value = statistics.median(r["value"] for r in runs)
    line = {"metric": "successors/s", "value": value, "unit": "successors/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": None, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u64", "data": "synthetic",
            "config": {"workload": WORKLOADS.get(name, WORKLOADS["s13-lrx"])["desc"],
                       "sample_layers": CPU_SAMPLE_LAYERS},
            "impl": "reference",
            "cpu_baseline": {"value": value, "unit": "successors/s", "cores": runs[0]["cores"], "kind": "port",
                             "sample": runs[0]["sample"]},
            "e2e": {"value": value, "unit": "successors/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def bench_sweep(args, local):
    """Batched sweep: 512 instances (256 seeds x {directed, inverse-closed}),
    each wave one persistent cooperative launch."""
    import torch
    from multigpubfs_b200 import workloads
    from multigpubfs_b200.batch import BatchSweep
    torch.cuda.set_device(local)
    graphs = workloads.sweep(512)
    with BatchSweep(graphs, local) as sweep:
        for _ in range(args.warmup):
            sweep.run(host_loop=args.host_loop)
        ref = sweep.layer_tables()
        runs = [sweep.run(host_loop=args.host_loop) for _ in range(args.steps)]
        assert sweep.layer_tables() == ref
    dev = sum(r["device_seconds"] for r in runs) / len(runs)
    succ, states = runs[0]["successors"], runs[0]["states"]
    line = {"metric": "successors/s", "value": succ / dev, "unit": "successors/s", "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": dev * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "u64", "data": "synthetic",
            "config": {"workload": "batched sweep: 512 instances (256 seeds x directed / inverse-closed), n in "
                                   "{7,8,9,10}, 2-3 seeded random generators, exact per-instance Lehmer bitmaps, "
                                   "each wave one persistent cooperative launch",
                       "instances": len(graphs), "states_per_step": states, "successors_per_step": succ},
            "settled_states_per_s": states / dev,
            "wall_ms_per_step": sum(r["seconds"] for r in runs) / len(runs) * 1e3,
            "waves": runs[0]["waves"], "launches_per_step": runs[0]["kernel_launches"],
            "layer_steps": runs[0]["layer_steps"], "gpu_launches": sum(r["kernel_launches"] for r in runs)}
    print(json.dumps(line), flush=True)
    return 0


def bench_planner(args, local):
    """Learned vs plain planner on batched sweeps.  The network is fitted by
    the library's kernels on 4/5 of the layer tables of the 512-instance sweep
    plus 32 S11 / S12 instances on other seeds, and its capacity margin is
    calibrated on the other 1/5.  The plain run
    reserves each instance's orbit bound n!, the learned run its predicted peak
    times the margin (exact rerun on overflow); both must give identical
    tables.  Scenarios: 128 S12 instances with the whole device, and a
    held-out 512-instance sweep (other seeds) under a 1 GiB budget.  The
    learned wall time includes the prediction."""
    import math
    import torch
    from multigpubfs_b200 import workloads
    from multigpubfs_b200.batch import BatchSweep
    from multigpubfs_b200.planner import (PlannerNet, calibrate_margin, predicted_capacities, rollout_device,
                                          training_set)
    torch.cuda.set_device(local)
    t0 = time.perf_counter()
    # Layer tables the BFS generates: the 512-instance sweep (n in 7..10) and
    # 32 S11 / S12 instances on seeds disjoint from the scenarios' instances.
    train = workloads.sweep(512) + [workloads.planner_instance(i, n=n, seed_base=20261204 + 50000 + 100 * n)
                                    for n in (11, 12) for i in range(16)]
    with BatchSweep(train, local) as sw:
        sw.run()
        tables = sw.layer_tables()
    fit_ids = [i for i in range(len(train)) if i % 5]
    cal_ids = [i for i in range(len(train)) if i % 5 == 0]
    X, T = training_set([train[i] for i in fit_ids], [tables[i] for i in fit_ids])
    net = PlannerNet(local, seed=0)
    hist = net.fit(X, T, steps=2000, lr=3e-3)
    margin = calibrate_margin(net, [train[i] for i in cal_ids], [tables[i] for i in cal_ids])
    train_s = time.perf_counter() - t0
    scenarios = [
        ("s12", f"{args.instances} S12 instances, 2-4 seeded random generators plus inverses, whole device",
         [workloads.planner_instance(i) for i in range(args.instances)], None),
        ("sweep_heldout_1gib", "512-instance sweep on held-out seeds, n in {7,8,9,10}, 1 GiB memory budget",
         workloads.sweep(512, seed_base=20261203 + 4096), 1 << 30),
        ("sweep_heldout_256mib", "512-instance sweep on held-out seeds, n in {7,8,9,10}, 256 MiB memory budget",
         workloads.sweep(512, seed_base=20261203 + 4096), 1 << 28),
    ]
    keys = ("seconds", "device_seconds", "waves", "redo_instances", "states", "successors")
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
            out[arm] = sorted(rs, key=lambda r: r["seconds"])[len(rs) // 2]
        same = out["plain"]["layer_tables"] == out["learned"]["layer_tables"]
        same_all &= same
        peaks = [max(t) for t in out["plain"]["layer_tables"]]
        peaks_pred, _, _ = rollout_device(net, graphs)
        logr = sorted(math.log(q / max(1.0, p)) for p, q in zip(peaks_pred, peaks))
        learned_wall = out["learned"]["seconds"] + predict_s
        report[name] = {
            "workload": desc, "instances": len(graphs), "memory_budget_bytes": budget, "identical_tables": same,
            "plain": {k: out["plain"][k] for k in keys},
            "learned": dict({k: out["learned"][k] for k in keys}, predict_seconds=predict_s,
                            wall_with_prediction=learned_wall),
            "speedup_wall": out["plain"]["seconds"] / learned_wall,
            "reserved_frontier_words": {"plain": sum(math.factorial(len(g["start"])) for g in graphs),
                                        "learned": sum(caps)},
            "peak_log_true_over_predicted": {"median_abs": sorted(abs(x) for x in logr)[len(logr) // 2],
                                             "min": logr[0], "max": logr[-1]}}
    main_s = report["s12"]
    line = {"metric": "successors/s", "value": main_s["learned"]["successors"] / main_s["learned"]["wall_with_prediction"],
            "unit": "successors/s", "n_gpus": 1, "steps": max(1, args.steps), "warmup": 1,
            "ms_per_step": main_s["learned"]["wall_with_prediction"] * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u64", "data": "synthetic",
            "config": {"workload": "learned vs plain planner on batched sweeps (value: S12 scenario, learned)"},
            "identical_tables": same_all, "scenarios": report,
            "predictor": {"train_rows": int(len(X)), "loss_first": hist[0], "loss_last": hist[-1],
                          "train_seconds": train_s, "margin": margin}}
    print(json.dumps(line), flush=True)
    return 0 if same_all else 1


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["native", "reference"], default="native")
    ap.add_argument("--workload", choices=sorted(WORKLOADS) + ["sweep512", "planner-s12"], default="s13-lrx")
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
        return bench_sweep(args, local)
    if args.workload == "planner-s12":
        return bench_planner(args, local)

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
    graph = GraphDefinition.permutation(w["gens"], list(range(w["n"])))
    expect = expected_layers(args.workload, w["n"])

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    # ---- value: resident engine, K whole BFS runs ------------------------------------
    eng = NativeGraph(graph, local)
    plan = eng.plan(visited=visited, dedup=dedup, host_loop=args.host_loop)
    for _ in range(args.warmup):
        r = eng.run()
        assert r.layer_sizes == expect, "layer table mismatch in warm-up"
    visible = os.environ.get("CUDA_VISIBLE_DEVICES", "").split(",")
    gpu_index = visible[local] if visible and visible[0] else str(local)
    results = []
    barrier()
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(gpu_index) as clocks:
        start.record()
        wall0 = time.perf_counter()
        for _ in range(args.steps):
            results.append(eng.run())
        stop.record()
        barrier()
        wall = time.perf_counter() - wall0
    device_s = start.elapsed_time(stop) * 1e-3
    for r in results:
        assert r.complete and r.layer_sizes == expect, "layer table mismatch in a timed run"
    device_max = device_s
    if world > 1:
        # Replicas: every rank must hold the same table; the job time is the slowest rank's.
        from multigpubfs_b200 import replicas
        view = replicas.exchange(results[0].layer_sizes, device_s, results[0].successors * args.steps,
                                 device=torch.device("cuda", local))
        device_max = view["device_seconds_max"]
    succ = results[0].successors
    states = results[0].states
    kernel_s = sum(r.kernel_seconds for r in results) / len(results)
    launches = sum(r.kernel_launches for r in results)
    eng.close()

    # ---- e2e: C-ABI handle from host buffers, every step ------------------------------
    e2e_times = []
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
        assert sizes == expect
        d2h = 24 * len(sizes) + 16 * len(sizes) + 8 * w["n"] * (len(cur) + len(prev))
    e2e_t = torch.tensor([sum(e2e_times) / len(e2e_times)], dtype=torch.float64, device="cuda")
    if world > 1:
        dist.all_reduce(e2e_t, op=dist.ReduceOp.MAX)

    if rank == 0:
        peak, peak_kind = measured_peak()
        b_alg = 16 * states + 32 * succ
        achieved = b_alg / kernel_s / 1e9
        traffic = None
        prof = ROOT / "profiles" / f"traffic_{args.workload}.json"
        if prof.exists():
            try:
                traffic = json.loads(prof.read_text()).get(plan["dedup"], {}).get("dram_bytes_per_bfs")
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
                       "planner": plan["planner"], "parallelism": f"replicas{world}",
                       "states_per_bfs": states, "successors_per_bfs": succ,
                       "l2": "working set larger than L2 (bitmap %d MB, frontiers up to several GB)"
                             % (plan["bitmap_bits"] // 8 // (1 << 20))},
            "settled_states_per_s": world * states * args.steps / device_max,
            "wall_ms_per_step": wall / args.steps * 1e3,
            "kernel_ms_per_step": kernel_s * 1e3,
            "e2e": {"value": world * succ / float(e2e_t.item()), "unit": "successors/s",
                    "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic, "peak_kind": peak_kind,
                         "b_alg_bytes": b_alg,
                         "kernel": kernel_names.get(plan["dedup"], "expand_packed (fused layer expansion)")},
            "gpu_launches": launches,
            "clocks": clocks.summary(),
        }
        if world == 1 and not args.no_cpu_baseline:
            line["cpu_baseline"] = cpu_baseline()
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
