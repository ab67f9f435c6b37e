"""CPU oracle for exact BFS over implicit Cayley / permutation graphs.

TEST INFRASTRUCTURE ONLY.  Only ``tests/``, ``__graft_entry__.smoke()`` and the
``cpu_baseline`` / ``--impl reference`` legs of ``bench.py`` may import this
module, and only as the checker.  The product path (``multigpubfs_b200``) never
imports it and has no CPU fallback.

Each function restates the reference's algorithm in plain Python and cites the
reference file it follows (paths relative to the TryDotAtwo/MultiGPUBFS tree):

* ``successor`` / ``matrix_multiply``   multigpubfs/graph_definition.py:70-83
* ``inverse_closed``                    multigpubfs/graph_definition.py:84-108
* ``exact_layers``                      multigpubfs/graph_definition.py:109-117
* ``multiset_rank`` / ``multiset_unrank`` crates/mgbfs-runtime/src/permutation_bitmap.rs:29-58
* ``coxeter_layers``                    multigpubfs/workload_geometry.py:2-19
* ``lrx_generators``                    multigpubfs/specialized.py:23-25, scripts/cpu_small_bfs.py:21-27

Parity of this oracle is pinned by ``tests/test_oracle.py`` against golden
vectors in ``tests/golden/`` that were produced by running the reference's own
Python code (``tests/golden/make_golden.py``) and against the reference's
shipped ``data/reference/lrx13-layers.json`` table.
"""
from __future__ import annotations

import math

I64_MIN = -(1 << 63)
I64_MAX = (1 << 63) - 1


def wrap_i64(x: int) -> int:
    """Two's-complement wrap to int64 (graph_definition.py:6-7)."""
    return ((x + (1 << 63)) & ((1 << 64) - 1)) - (1 << 63)


def matrix_multiply(mx, state, rows, cols, mod):
    """child = M (rows x rows) . S (rows x cols), int64-wrapped per entry, then
    Python ``%`` (non-negative for mod > 0); mod == 0 keeps the wrapped value
    (graph_definition.py:77-83)."""
    out = []
    for i in range(rows):
        for j in range(cols):
            total = wrap_i64(sum(mx[i * rows + k] * state[k * cols + j] for k in range(rows)))
            out.append(total % mod if mod else total)
    return out


def successor(graph: dict, state, generator: int):
    """Apply one generator (graph_definition.py:70-75). ``graph`` is the schema-2
    dict: permutation generators give child[i] = state[g[i]]."""
    a = graph["action"]
    g = a["generators"][generator]
    if a["kind"] == "permutation":
        return [state[i] for i in g]
    return matrix_multiply(g["matrix"], state, a["rows"], a["cols"], g["modulo"])


def generator_count(graph: dict) -> int:
    return len(graph["action"]["generators"])


def inverse_closed(graph: dict) -> bool:
    """Every generator's inverse is among the generators (graph_definition.py:84-108)."""
    a = graph["action"]
    gs = a["generators"]
    if a["kind"] == "permutation":
        available = {tuple(g) for g in gs}
        for g in gs:
            inv = [0] * len(g)
            for i, x in enumerate(g):
                inv[x] = i
            if tuple(inv) not in available:
                return False
        return True
    n = a["rows"]
    if len({g["modulo"] for g in gs}) != 1:
        return False
    mod = gs[0]["modulo"]
    if mod and mod & (mod - 1):
        for g in gs:
            for i in range(n):
                if sum(abs(v) * (mod - 1) for v in g["matrix"][i * n:(i + 1) * n]) > I64_MAX:
                    return False
    eye = [int(i == j) for i in range(n) for j in range(n)]

    def compose(g, h):
        right = [v % mod for v in h["matrix"]] if mod else h["matrix"]
        return matrix_multiply(g["matrix"], right, n, n, mod)

    for g in gs:
        if not any(compose(g, h) == eye and compose(h, g) == eye for h in gs):
            return False
    for g in gs:
        if g["modulo"] and any(not 0 <= x < g["modulo"] for x in graph["start"]):
            return False
    return True


def exact_layers(graph: dict, maximum_states: int):
    """Set-based level BFS; returns each layer as a sorted list of states
    (graph_definition.py:109-117).  Raises ValueError('ORACLE_CAPACITY')."""
    if type(maximum_states) is not int or maximum_states < 1:
        raise ValueError("ORACLE_CAPACITY")
    start = tuple(graph["start"])
    seen = {start}
    frontier = {start}
    layers = []
    gc = generator_count(graph)
    while frontier:
        layers.append([list(x) for x in sorted(frontier)])
        future = {tuple(successor(graph, list(x), g)) for x in frontier for g in range(gc)} - seen
        if len(seen) + len(future) > maximum_states:
            raise ValueError("ORACLE_CAPACITY")
        seen.update(future)
        frontier = future
    return layers


def layer_sizes(graph: dict, maximum_states: int = 1 << 40):
    return [len(x) for x in exact_layers(graph, maximum_states)]


# ---------------------------------------------------------------------------
# Multiset-permutation rank (lexicographic), permutation_bitmap.rs:29-58.

def multiset_domain(start):
    """Sorted distinct symbols, their counts and the multinomial total."""
    symbols = sorted(set(start))
    counts = [start.count(s) for s in symbols]
    total = math.factorial(len(start))
    for c in counts:
        total //= math.factorial(c)
    return symbols, counts, total


def multiset_rank(start, state) -> int:
    symbols, counts, total = multiset_domain(list(start))
    counts = list(counts)
    ways = total
    rank = 0
    n = len(state)
    for index, symbol in enumerate(state):
        i = symbols.index(symbol)
        if counts[i] == 0:
            raise ValueError("BITMAP_STATE_MULTIPLICITY")
        remaining = n - index
        less = sum(counts[:i])
        rank += ways * less // remaining
        ways = ways * counts[i] // remaining
        counts[i] -= 1
    return rank


def multiset_unrank(start, rank: int):
    symbols, counts, total = multiset_domain(list(start))
    if not 0 <= rank < total:
        raise ValueError("BITMAP_RANK_RANGE")
    counts = list(counts)
    ways = total
    n = len(start)
    state = []
    for index in range(n):
        remaining = n - index
        for i, c in enumerate(counts):
            if c == 0:
                continue
            block = ways * c // remaining
            if rank >= block:
                rank -= block
            else:
                state.append(symbols[i])
                counts[i] -= 1
                ways = block
                break
    return state


# ---------------------------------------------------------------------------
# Product of position components' multiset domains (PositionOrbitDomain,
# crates/mgbfs-runtime/src/permutation_bitmap.rs:61-143).

def position_components(n: int, generators):
    """Classes of positions under i ~ g[i] for every generator, ordered by
    their first position, each ascending (permutation_bitmap.rs:68-82)."""
    parent = list(range(n))

    def root(x):
        while parent[x] != x:
            parent[x] = parent[parent[x]]
            x = parent[x]
        return x
    for g in generators:
        if len(g) != n or sorted(g) != list(range(n)):
            raise ValueError("BITMAP_ORBIT_GENERATOR")
        for i, j in enumerate(g):
            parent[root(i)] = root(j)
    classes = {}
    for i in range(n):
        classes.setdefault(root(i), []).append(i)
    return sorted(classes.values(), key=lambda c: c[0])


def product_domain(start, generators):
    """[(positions, component start values, multiset size)] and the product."""
    comps = []
    size = 1
    for pos in position_components(len(start), generators):
        values = [start[i] for i in pos]
        total = multiset_domain(values)[2]
        comps.append((pos, values, total))
        size *= total
    return comps, size


def product_rank(start, generators, state) -> int:
    """Mixed-radix rank over the components in order, each digit the multiset
    rank of the component's values in position order."""
    comps, size = product_domain(start, generators)
    rank = 0
    for pos, values, total in comps:
        digit = multiset_rank(values, [state[i] for i in pos])
        rank = rank * total + digit
    if rank >= size:
        raise ValueError("BITMAP_RANK_RANGE")
    return rank


def product_unrank(start, generators, rank: int):
    comps, size = product_domain(start, generators)
    if not 0 <= rank < size:
        raise ValueError("BITMAP_RANK_RANGE")
    state = [None] * len(start)
    for pos, values, total in reversed(comps):
        rank, digit = divmod(rank, total)
        for i, v in zip(pos, multiset_unrank(values, digit)):
            state[i] = v
    return state


# ---------------------------------------------------------------------------
# Generator families and certified layer tables.

def lrx_generators(n: int):
    """L = cyclic left shift, R = cyclic right shift, X = swap positions 0,1
    (specialized.py:23-25; cpu_small_bfs.py:21-27): child[i] = state[g[i]]."""
    left = [(i + 1) % n for i in range(n)]
    right = [(i - 1) % n for i in range(n)]
    x = list(range(n))
    x[0], x[1] = x[1], x[0]
    return [left, right, x]


def coxeter_generators(n: int):
    """Adjacent transpositions s_1..s_{n-1}: s_i swaps positions i-1 and i."""
    gens = []
    for i in range(n - 1):
        g = list(range(n))
        g[i], g[i + 1] = g[i + 1], g[i]
        gens.append(g)
    return gens


def coxeter_layers(n: int):
    """Exact layer sizes of S_n under adjacent transpositions: the number of
    permutations with k inversions, by the Mahonian recurrence
    (workload_geometry.py:2-19)."""
    sizes = [1]
    for i in range(1, n + 1):
        out = []
        window = 0
        for j in range(len(sizes) + i - 1):
            if j < len(sizes):
                window += sizes[j]
            if j >= i:
                window -= sizes[j - i]
            out.append(window)
        sizes = out
    return sizes


def permutation_graph(generators, start, name=""):
    """Schema-2 graph dict (graph_definition.py:17-20)."""
    return {
        "schema": 2,
        "name": name,
        "generator_names": [str(i) for i in range(len(generators))],
        "action": {"kind": "permutation", "degree": len(start), "generators": [list(g) for g in generators]},
        "start": list(start),
        "expected_max_unique_states": None,
    }


def matrix_graph(rows, cols, generators, start, name=""):
    return {
        "schema": 2,
        "name": name,
        "generator_names": [str(i) for i in range(len(generators))],
        "action": {"kind": "matrix", "rows": rows, "cols": cols,
                   "generators": [{"matrix": list(m), "modulo": mod} for m, mod in generators]},
        "start": list(start),
        "expected_max_unique_states": None,
    }


def sweep_instance(i: int, inverse_closed_variant: bool, seed_base: int = 20261203):
    """Batched-sweep instance i: n uniform in {7,8,9,10}, k in {2,3} seeded random
    generators (numpy default_rng(seed_base + i)); the inverse-closed variant adds
    each generator's inverse (if distinct and not already present)."""
    import numpy as np
    rng = np.random.default_rng(seed_base + i)
    n = int(rng.choice([7, 8, 9, 10]))
    k = int(rng.choice([2, 3]))
    gens = [[int(x) for x in rng.permutation(n)] for _ in range(k)]
    if inverse_closed_variant:
        gens = add_inverses(gens)
    return permutation_graph(gens, list(range(n)), name=f"sweep-{i}")


def add_inverses(gens):
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
