"""Named graph families and seeded synthetic sweeps (schema-2 dicts).

* LRX: L = cyclic left shift, R = cyclic right shift, X = swap of positions 0,1
  (multigpubfs/specialized.py:23-25).
* Coxeter: adjacent transpositions s_1..s_{n-1}.
* Sweep instances: n uniform in {7,8,9,10}, 2-3 generators drawn as seeded
  uniform random permutations (numpy default_rng(20261203 + i)); the
  inverse-closed variant adds every generator's inverse.
* Planner instances: S12 with 2-4 seeded random generators plus inverses
  (default_rng(20261204 + i)).
"""
from __future__ import annotations

import numpy as np


def permutation_graph(generators, start, name=""):
    return {"schema": 2, "name": name, "generator_names": [str(i) for i in range(len(generators))],
            "action": {"kind": "permutation", "degree": len(start), "generators": [list(g) for g in generators]},
            "start": list(start), "expected_max_unique_states": None}


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


def with_inverses(gens):
    out = [list(g) for g in gens]
    seen = {tuple(g) for g in out}
    for g in gens:
        inv = [0] * len(g)
        for i, x in enumerate(g):
            inv[x] = i
        if tuple(inv) not in seen:
            seen.add(tuple(inv))
            out.append(inv)
    return out


def sweep_instance(i, inverse_closed, seed_base=20261203):
    rng = np.random.default_rng(seed_base + i)
    n = int(rng.choice([7, 8, 9, 10]))
    k = int(rng.choice([2, 3]))
    gens = [[int(x) for x in rng.permutation(n)] for _ in range(k)]
    if inverse_closed:
        gens = with_inverses(gens)
    return permutation_graph(gens, list(range(n)), name=f"sweep-{i}")


def sweep(count=512, seed_base=20261203):
    """The batched sweep: the directed and the inverse-closed variant of each
    of `count // 2` seeded instances."""
    half = count // 2
    return [sweep_instance(i, closed, seed_base) for i in range(half) for closed in (False, True)]


def planner_instance(i, n=12, seed_base=20261204):
    rng = np.random.default_rng(seed_base + i)
    k = int(rng.choice([2, 3, 4]))
    gens = with_inverses([[int(x) for x in rng.permutation(n)] for _ in range(k)])
    return permutation_graph(gens, list(range(n)), name=f"planner-{i}")
