"""Generate lrx14_prefix.json: the first 24 layer sizes of S14 under L, R, X
from the identity, by the reference's own CPU search (scripts/cpu_small_bfs.py
exact_search, TryDotAtwo/MultiGPUBFS) run from a read-only checkout and
cancelled once 24 layers are committed.

    PYTHONDONTWRITEBYTECODE=1 python tests/golden/make_lrx14_prefix.py /path/to/MultiGPUBFS

The reference tree is only read; nothing here is needed at test time.
"""
from __future__ import annotations

import json
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
LAYERS = 24


def main(root: str) -> None:
    root = Path(root).resolve()
    sys.path.insert(0, str(root / "scripts"))
    import cpu_small_bfs

    sizes = []
    out = cpu_small_bfs.exact_search(14, 1, "000000000000000000000000013527dc",
                                     lambda depth, frontier, *rest: sizes.append(len(frontier)),
                                     cancelled=lambda: "prefix done" if len(sizes) >= LAYERS else None)
    assert not out.get("complete", True) and len(sizes) >= LAYERS, out
    (HERE / "lrx14_prefix.json").write_text(json.dumps({
        "source": "scripts/cpu_small_bfs.py exact_search(14, 1, ...) cancelled after the first 24 layers",
        "n": 14, "layers": sizes[:LAYERS], "states": 87178291200}) + "\n")
    print(sizes[:LAYERS])


if __name__ == "__main__":
    main(sys.argv[1])
