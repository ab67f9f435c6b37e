"""Generate matrix_groups.json by running the reference's own Python code
(TryDotAtwo/MultiGPUBFS, multigpubfs/graph_definition.py exact_layers and
multigpubfs/workload_geometry.py certified_frontier_bound) from a read-only
checkout:

    PYTHONDONTWRITEBYTECODE=1 python tests/golden/make_matrix_golden.py /path/to/MultiGPUBFS

The cases are SL(2, p) acting on 2x2 matrices from the identity, generated by
[[1,1],[0,1]], [[1,0],[1,1]] and their inverses mod p (orbit p(p^2 - 1)).
They are large enough for concurrent claims of one state in a layer of the
wide-key table.  The reference tree is only read; nothing here is needed at
test time.
"""
from __future__ import annotations

import json
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent


def sl2(GraphDefinition, p):
    gens = [([1, 1, 0, 1], p), ([1, 0, 1, 1], p), ([1, p - 1, 0, 1], p), ([1, 0, p - 1, 1], p)]
    return GraphDefinition.matrix(2, 2, gens, [1, 0, 0, 1])


def main(root: str) -> None:
    root = Path(root).resolve()
    sys.path.insert(0, str(root))
    from multigpubfs.graph_definition import GraphDefinition
    from multigpubfs.workload_geometry import certified_frontier_bound
    out = {"source": "multigpubfs.graph_definition.GraphDefinition.exact_layers", "cases": {}}
    for p in (31, 101):
        g = sl2(GraphDefinition, p)
        layers = [len(x) for x in g.exact_layers(1 << 24)]
        bound = certified_frontier_bound(g)
        out["cases"][f"sl2_mod{p}"] = {"graph": g.to_dict() if hasattr(g, "to_dict") else g.value,
                                       "layers": layers, "certified_bound": bound}
        print(p, sum(layers), len(layers), flush=True)
    (HERE / "matrix_groups.json").write_text(json.dumps(out, indent=1, sort_keys=True) + "\n")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        raise SystemExit("usage: make_matrix_golden.py /path/to/MultiGPUBFS")
    main(sys.argv[1])
