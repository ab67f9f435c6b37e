"""Named graph families and seeded synthetic sweeps (schema-2 dicts).

* LRX: L = cyclic left shift, R = cyclic right shift, X = swap of positions 0,1
  (multigpubfs/specialized.py:23-25).
* Coxeter: adjacent transpositions s_1..s_{n-1}.
* Sweep instances: n uniform in {7,8,9,10}, 2-3 generators drawn as seeded
  uniform random permutations (numpy default_rng(20261203 + i)); the
  inverse-closed variant adds every generator's inverse.
* Planner instances: S12 with 2-4 seeded random generators plus inverses
  (default_rng(20261204 + i)).
* GL(2, p): 2x2 int64 matrices mod a prime p from the identity under the
  elementary transvections [[1,1],[0,1]], [[1,0],[1,1]], diag(g, 1) for the
  least primitive root g, and their inverses; the orbit is the whole group,
  (p^2 - 1)(p^2 - p) states, against the certified entry-space bound p^4.
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


def primitive_root(p):
    """Least primitive root of the prime p."""
    factors = [q for q in range(2, p) if (p - 1) % q == 0 and all(q % d for d in range(2, int(q ** 0.5) + 1))]
    return next(r for r in range(2, p) if all(pow(r, (p - 1) // q, p) != 1 for q in factors))


def gl2_generators(p):
    """(matrix, modulus) pairs of GL(2, p) (row-major 2x2)."""
    g = primitive_root(p)
    gi = pow(g, p - 2, p)
    mats = [[1, 1, 0, 1], [1, 0, 1, 1], [1, p - 1, 0, 1], [1, 0, p - 1, 1], [g, 0, 0, 1], [gi, 0, 0, 1]]
    return [(m, p) for m in mats]


def gl2_graph(p):
    gens = gl2_generators(p)
    return {"schema": 2, "name": f"gl2-{p}", "generator_names": [str(i) for i in range(len(gens))],
            "action": {"kind": "matrix", "rows": 2, "cols": 2,
                       "generators": [{"matrix": list(m), "modulo": mod} for m, mod in gens]},
            "start": [1, 0, 0, 1], "expected_max_unique_states": None}
