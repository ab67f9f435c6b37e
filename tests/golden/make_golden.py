"""Generate the golden vectors in this folder by running the reference's own
Python code (TryDotAtwo/MultiGPUBFS) from a read-only checkout.

    PYTHONDONTWRITEBYTECODE=1 python tests/golden/make_golden.py /path/to/MultiGPUBFS

Outputs (all small JSON files, committed):
  lrx_layers.json        scripts/cpu_small_bfs.py exact_search layer sizes, n = 3..11
  lrx13_layers.json      data/reference/lrx13-layers.json (the reference's shipped S13 table)
  coxeter_bounds.json    multigpubfs/workload_geometry.py coxeter_frontier_bound, n = 2..13
  exact_cases.json       GraphDefinition.exact_layers / successor / inverse_closed / digest
                         on permutation (distinct, repeated-label, directed, wide) and
                         int64 matrix graphs
The reference tree is only read; nothing here is needed at test time.
"""
from __future__ import annotations

import json
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent


def main(root: str) -> None:
    root = Path(root).resolve()
    sys.path.insert(0, str(root))
    sys.path.insert(0, str(root / "scripts"))
    import numpy as np
    from multigpubfs.graph_definition import GraphDefinition
    from multigpubfs.workload_geometry import coxeter_frontier_bound
    import cpu_small_bfs

    # 1. packed LRX CPU search (the reference's fast CPU BFS).
    lrx = {}
    for n in range(3, 12):
        sizes = []
        cpu_small_bfs.exact_search(n, 1, "000000000000000000000000013527dc",
                                   lambda depth, frontier, *rest: sizes.append(len(frontier)))
        lrx[str(n)] = sizes
        print("lrx", n, len(sizes), sum(sizes), flush=True)
    (HERE / "lrx_layers.json").write_text(json.dumps(
        {"source": "scripts/cpu_small_bfs.py:exact_search", "layers": lrx}, indent=0))

    # 2. shipped S13 LRX table.
    table = json.loads((root / "data/reference/lrx13-layers.json").read_text())
    (HERE / "lrx13_layers.json").write_text(json.dumps(
        {"source": "data/reference/lrx13-layers.json", "n": table["n"],
         "generators": table["generators"], "layers": table["layers"]}, indent=0))

    # 3. Coxeter certified bounds.
    cox = {}
    for n in range(2, 14):
        g = []
        for i in range(n - 1):
            p = list(range(n)); p[i], p[i + 1] = p[i + 1], p[i]; g.append(p)
        b = coxeter_frontier_bound(GraphDefinition.permutation(g, list(range(n))))
        cox[str(n)] = {k: b[k] for k in ("maximum_frontier", "maximum_live_states", "order", "depth")}
    (HERE / "coxeter_bounds.json").write_text(json.dumps(
        {"source": "multigpubfs/workload_geometry.py:coxeter_frontier_bound", "bounds": cox}, indent=0))

    # 4. exact_layers cases.
    cases = []

    def add(name, g, probes=None):
        layers = g.exact_layers(1 << 24)
        sizes = [len(x) for x in layers]
        entry = {"name": name, "graph": json.loads(g.to_json()), "digest": g.digest(),
                 "inverse_closed": g.inverse_closed(), "layer_sizes": sizes,
                 "last_layer": layers[-1] if len(layers[-1]) <= 2000 else None,
                 "previous_layer": layers[-2] if len(layers) > 1 and len(layers[-2]) <= 2000 else None}
        kat = []
        states = [g.start] + (probes or [])
        if len(layers) > 1:
            states += layers[1][:2] + layers[-1][:2]
        for s in states:
            for k in range(g.generator_count):
                kat.append({"state": s, "generator": k, "child": g.successor(s, k)})
        entry["successors"] = kat
        cases.append(entry)
        print("case", name, len(sizes), sum(sizes), flush=True)

    def lrx_gens(n):
        return [[(i + 1) % n for i in range(n)], [(i - 1) % n for i in range(n)],
                [1, 0] + list(range(2, n))]

    def cox_gens(n):
        out = []
        for i in range(n - 1):
            p = list(range(n)); p[i], p[i + 1] = p[i + 1], p[i]; out.append(p)
        return out

    def inverse(p):
        q = [0] * len(p)
        for i, x in enumerate(p):
            q[x] = i
        return q

    for n in (3, 4, 5, 6, 7, 8):
        add(f"lrx{n}", GraphDefinition.permutation(lrx_gens(n), list(range(n))))
    for n in (3, 4, 5, 6, 7):
        add(f"coxeter{n}", GraphDefinition.permutation(cox_gens(n), list(range(n))))
    rng = np.random.default_rng(7)
    for i in range(8):
        n = int(rng.choice([5, 6, 7, 8]))
        k = int(rng.choice([2, 3]))
        gens = [[int(x) for x in rng.permutation(n)] for _ in range(k)]
        add(f"random_directed_{i}", GraphDefinition.permutation(gens, list(range(n))))
        closed = gens + [inverse(p) for p in gens if inverse(p) not in gens]
        add(f"random_closed_{i}", GraphDefinition.permutation(closed, list(range(n))))
    add("repeated_labels", GraphDefinition.permutation([[1, 2, 3, 0], [1, 0, 2, 3]], [0, 0, 1, 2]))
    add("repeated_labels_lrx8", GraphDefinition.permutation(lrx_gens(8), [0, 0, 1, 1, 2, 2, 3, 3]))
    add("repeated_labels_negative", GraphDefinition.permutation(cox_gens(6), [-7, -7, 0, 99, 99, 5]))
    add("big_labels", GraphDefinition.permutation(lrx_gens(6), [1000, -5, 7, 1 << 40, 3, 2]))
    add("single_generator_cycle", GraphDefinition.permutation([[1, 2, 0]], [0, 1, 2]))
    add("identity_only", GraphDefinition.permutation([[0, 1, 2, 3]], [0, 1, 2, 3]))
    add("degree_one", GraphDefinition.permutation([[0]], [5]))
    add("cycle300", GraphDefinition.permutation([list(range(1, 300)) + [0]], list(range(300))))
    wide = list(range(20))
    c5 = list(range(20)); c5[0:5] = [1, 2, 3, 4, 0]
    c7 = list(range(20)); c7[5:12] = [6, 7, 8, 9, 10, 11, 5]
    add("wide20_directed", GraphDefinition.permutation([c5, c7], wide))
    add("wide20_closed", GraphDefinition.permutation([c5, c7, inverse(c5), inverse(c7)], wide))
    add("s16_two_generators_small_orbit", GraphDefinition.permutation(
        [[1, 0] + list(range(2, 16)), list(range(14)) + [15, 14]], list(range(16))))
    add("matrix_rect_257", GraphDefinition.matrix(2, 1, [([1, 1, 0, 1], 257)], [256, 2]))
    add("matrix_wrap_mod7", GraphDefinition.matrix(1, 1, [([2], 7)], [(1 << 63) - 1]))
    add("matrix_wrap_nomod", GraphDefinition.matrix(1, 1, [([2], 0)], [(1 << 63) - 1]), probes=[[-2], [1 << 62]])
    add("matrix_mixed_moduli", GraphDefinition.matrix(1, 1, [([2], 5), ([3], 7)], [4]))
    add("matrix_sl2_mod5", GraphDefinition.matrix(2, 2, [([1, 1, 0, 1], 5), ([1, 0, 1, 1], 5)], [1, 0, 0, 1]))
    add("matrix_sl2_mod7_closed", GraphDefinition.matrix(
        2, 2, [([1, 1, 0, 1], 7), ([1, 6, 0, 1], 7), ([1, 0, 1, 1], 7), ([1, 0, 6, 1], 7)], [1, 0, 0, 1]))
    add("matrix_heisenberg_mod3", GraphDefinition.matrix(
        3, 3, [([1, 1, 0, 0, 1, 0, 0, 0, 1], 3), ([1, 0, 0, 0, 1, 1, 0, 0, 1], 3)],
        [1, 0, 0, 0, 1, 0, 0, 0, 1]))
    add("matrix_rect_3x2_mod11", GraphDefinition.matrix(
        3, 2, [([1, 2, 0, 0, 1, 0, 3, 0, 1], 11), ([0, 1, 0, 1, 0, 0, 0, 0, 1], 11)], [1, 0, 0, 1, 2, 5]))
    add("matrix_negative_start_mod9", GraphDefinition.matrix(1, 2, [([2], 9)], [-3, 4]))
    add("matrix_nomod_small", GraphDefinition.matrix(1, 1, [([-1], 0)], [12345]))
    (HERE / "exact_cases.json").write_text(json.dumps(
        {"source": "multigpubfs/graph_definition.py:GraphDefinition", "cases": cases},
        separators=(",", ":")))

    # 5. wrapping known answers (tests/test_graph_definition.py:13-16).
    kat = {
        "wrap_mod7": GraphDefinition.matrix(1, 1, [([2], 7)], [(1 << 63) - 1]).successor([(1 << 63) - 1], 0),
        "wrap_nomod": GraphDefinition.matrix(1, 1, [([2], 0)], [(1 << 63) - 1]).successor([(1 << 63) - 1], 0),
        "overflow_guard_inverse_closed": GraphDefinition.matrix(1, 1, [([(1 << 63) - 1], 3)], [2]).inverse_closed(),
    }
    (HERE / "wrap_kat.json").write_text(json.dumps(kat))


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_golden.py <path of the reference checkout>")
    main(sys.argv[1])
