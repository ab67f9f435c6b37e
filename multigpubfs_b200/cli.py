"""Command line front end (the in-process analogue of the reference's
``mgbfs graph`` / ``graph-info`` verbs, crates/mgbfs-cli/src/main.rs:54-84).

    python -m multigpubfs_b200.cli plan  <graph.json | family> [--visited ..] [--dedup ..]
    python -m multigpubfs_b200.cli run   <graph.json | family> [--max-layers N] [--repeat R] [--out DIR]

``family`` is one of ``lrx:N`` (L, R, X on S_N), ``coxeter:N`` (adjacent
transpositions on S_N), started from the identity, or ``gl2:P`` (GL(2, P) on
2x2 matrices mod the prime P).  ``run`` prints one JSON
line with the layer table and timings; with ``--out`` it writes the schema-2
report.json / states.json through run_graph instead.
"""
from __future__ import annotations

import argparse
import json
import sys
from pathlib import Path

from .graph_definition import GraphDefinition


def family(spec: str) -> GraphDefinition:
    if spec.endswith(".json") and Path(spec).exists():
        return GraphDefinition.from_dict(json.loads(Path(spec).read_text()))
    kind, _, n = spec.partition(":")
    n = int(n)
    if kind == "lrx":
        left = [(i + 1) % n for i in range(n)]
        right = [(i - 1) % n for i in range(n)]
        x = list(range(n))
        x[0], x[1] = x[1], x[0]
        return GraphDefinition.permutation([left, right, x], list(range(n)), name=f"lrx-{n}",
                                           generator_names=["L", "R", "X"])
    if kind == "coxeter":
        gens = []
        for i in range(n - 1):
            g = list(range(n))
            g[i], g[i + 1] = g[i + 1], g[i]
            gens.append(g)
        return GraphDefinition.permutation(gens, list(range(n)), name=f"coxeter-{n}")
    if kind == "gl2":
        from .workloads import gl2_graph
        return GraphDefinition.from_dict(gl2_graph(n))
    raise SystemExit(f"unknown graph {spec!r}: use a schema-2 JSON file, lrx:N, coxeter:N or gl2:P")


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(prog="python -m multigpubfs_b200.cli")
    ap.add_argument("verb", choices=["plan", "run"])
    ap.add_argument("graph")
    ap.add_argument("--device", type=int, default=0)
    ap.add_argument("--visited", default="auto", choices=["auto", "bitmap", "hash", "hash3"])
    ap.add_argument("--dedup", default="auto", choices=["auto", "atomic", "warp", "sort", "bucket", "grouped"])
    ap.add_argument("--planner", default="plain", choices=["plain", "learned"])
    ap.add_argument("--capacity", type=int, default=None)
    ap.add_argument("--shards", type=int, default=None)
    ap.add_argument("--route-chunk", type=int, default=None,
                    help="routed (bucket) layers: parents per route-and-accept pass, a multiple of 1024 "
                         "(default: the whole layer, or what the free memory holds)")
    ap.add_argument("--max-layers", type=int, default=None)
    ap.add_argument("--max-seconds", type=int, default=None)
    ap.add_argument("--repeat", type=int, default=1)
    ap.add_argument("--out", default=None)
    ap.add_argument("--host-loop", action="store_true",
                    help="one host round trip per layer instead of the whole BFS as one persistent launch "
                         "(each layer is then a separate launch, e.g. for a profiler)")
    a = ap.parse_args(argv)
    graph = family(a.graph)
    if a.out:
        from .launch import run_graph
        report = run_graph(graph, a.out, device=a.device, capacity=a.capacity, max_seconds=a.max_seconds,
                           visited=a.visited, dedup=a.dedup, planner=a.planner, max_layers=a.max_layers)
        print(json.dumps({k: report[k] for k in ("status", "reason", "layer_sizes", "bfs_seconds", "backend")}))
        return 0
    from .engine import NativeGraph
    learned = {"planner": "plain"}
    if a.planner == "learned":
        from .planner import choose_path
        learned = choose_path(graph.to_dict(), device=a.device)
    with NativeGraph(graph, a.device) as engine:
        plan = engine.plan(visited=a.visited, dedup=a.dedup, capacity=a.capacity, shards=a.shards,
                           host_loop=a.host_loop, route_chunk=a.route_chunk, **learned)
        if a.verb == "plan":
            print(json.dumps({"graph": graph.name, "digest": graph.digest(), "plan": plan}))
            return 0
        for i in range(a.repeat):
            r = engine.run(max_layers=a.max_layers, max_seconds=a.max_seconds)
            print(json.dumps({"graph": graph.name, "run": i, "complete": r.complete, "reason": r.reason,
                              "layers": len(r.layer_sizes), "states": r.states, "successors": r.successors,
                              "device_seconds": r.device_seconds, "kernel_seconds": r.kernel_seconds,
                              "kernel_launches": r.kernel_launches, "layer_sizes": r.layer_sizes,
                              "layer_seconds": [round(s, 6) for s in r.layer_seconds], "plan": plan}), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
