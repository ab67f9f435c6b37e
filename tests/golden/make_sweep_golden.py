"""Layer tables of the batched-sweep and planner workloads, made by the C
oracle (oracle/bfs_oracle.c, the CPU restatement of the reference's exact
level BFS, scripts/cpu_small_bfs.py:30-80 and
multigpubfs/graph_definition.py:109-117, itself pinned against the reference's
own outputs by tests/test_oracle.py).

    python tests/golden/make_sweep_golden.py [--s12 8]

Writes sweep_tables.json:
  sweep512            all 512 instances of workloads.sweep(512) (seeds 20261203 + i)
  sweep512_heldout    workloads.sweep(512, seed_base=20261203 + 4096)
  planner_s12         the first --s12 instances of workloads.planner_instance (seeds 20261204 + i)
Each entry keeps, per instance, the sha256 of its generator list (so a change
in the seeded generators is caught before any table is compared) and its
layer table.  Takes about two minutes for the sweeps and about a minute per
S12 instance on 8 cores.
"""
from __future__ import annotations

import argparse
import hashlib
import json
import sys
import time
from pathlib import Path

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
SWEEP_SEED = 20261203
HELDOUT_SEED = SWEEP_SEED + 4096
PLANNER_SEED = 20261204


def generator_digest(graph) -> str:
    text = json.dumps(graph["action"]["generators"], separators=(",", ":"))
    return hashlib.sha256(text.encode()).hexdigest()


def tables(graphs, label):
    from oracle import packed_oracle as P
    out, t0 = [], time.perf_counter()
    for i, g in enumerate(graphs):
        sizes, _, _ = P.packed_bfs(g["action"]["generators"], g["start"], use_bitmap=True)
        out.append(sizes)
        if len(graphs) <= 16:
            print(f"{label} {i}: {sum(sizes):,} states, {len(sizes)} layers, "
                  f"{time.perf_counter() - t0:.0f} s", flush=True)
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--s12", type=int, default=8, help="planner S12 instances to tabulate")
    a = ap.parse_args()
    sys.path.insert(0, str(ROOT))
    from multigpubfs_b200 import workloads
    doc = {"source": "oracle/bfs_oracle.c exact level BFS (Lehmer bitmap), via oracle/packed_oracle.py",
           "recipe": "python tests/golden/make_sweep_golden.py --s12 %d" % a.s12}
    for key, graphs, seed in (("sweep512", workloads.sweep(512), SWEEP_SEED),
                              ("sweep512_heldout", workloads.sweep(512, seed_base=HELDOUT_SEED), HELDOUT_SEED)):
        doc[key] = {"seed_base": seed, "generators_sha256": [generator_digest(g) for g in graphs],
                    "tables": tables(graphs, key)}
        print(key, "done", flush=True)
    s12 = [workloads.planner_instance(i) for i in range(a.s12)]
    doc["planner_s12"] = {"seed_base": PLANNER_SEED, "indices": list(range(a.s12)),
                          "generators_sha256": [generator_digest(g) for g in s12],
                          "tables": tables(s12, "planner_s12")}
    (HERE / "sweep_tables.json").write_text(json.dumps(doc, separators=(",", ":")) + "\n")
    print("wrote", HERE / "sweep_tables.json")


if __name__ == "__main__":
    main()
