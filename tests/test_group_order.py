"""Host Schreier-Sims (mgbfs2_group_order) against known group orders and the
CPU oracle's BFS state counts.  No GPU is used: the function is host code."""
import math

import pytest

from multigpubfs_b200 import native, workloads
from oracle import graph_oracle as G
from oracle import packed_oracle as P


def _cycle(n, points):
    g = list(range(n))
    for a, b in zip(points, points[1:] + points[:1]):
        g[a] = b
    return g


@pytest.mark.parametrize("n", range(2, 14))
def test_lrx_and_coxeter_generate_the_symmetric_group(n):
    assert native.group_order(G.lrx_generators(n)) == math.factorial(n)
    assert native.group_order(G.coxeter_generators(n)) == math.factorial(n)


def test_known_groups():
    assert native.group_order([list(range(6))]) == 1                      # identity only
    assert native.group_order([_cycle(9, list(range(9)))]) == 9            # cyclic C9
    assert native.group_order([_cycle(7, [0, 1, 2]), _cycle(7, [2, 3, 4, 5, 6])]) == math.factorial(7) // 2  # A7
    # Two disjoint 3-cycles generate C3 x C3.
    assert native.group_order([_cycle(6, [0, 1, 2]), _cycle(6, [3, 4, 5])]) == 9
    # Rotation and reflection of a square: the dihedral group of order 8.
    assert native.group_order([[1, 2, 3, 0], [0, 3, 2, 1]]) == 8
    # The Mathieu group M11 on 11 points (order 7920), from its standard generators.
    m11 = [[1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 0], [0, 1, 6, 9, 5, 3, 10, 2, 8, 4, 7]]
    assert native.group_order(m11) == 7920


def test_invalid_input():
    with pytest.raises(native.NativeError):
        native.group_order([[0, 0, 1]])
    with pytest.raises(native.NativeError):
        native.group_order([list(range(21))])


def test_matches_oracle_state_counts_on_seeded_sweep():
    # Distinct labels: the BFS settles exactly |G| states, including the
    # instances whose generators generate a proper subgroup of S_n.
    seen_proper = 0
    for i in range(48):
        for closed in (False, True):
            g = workloads.sweep_instance(i, closed)
            gens, start = g["action"]["generators"], g["start"]
            if len(start) > 8:
                continue
            sizes, _, _ = P.packed_bfs(gens, start)
            order = native.group_order(gens)
            assert order == sum(sizes)
            seen_proper += order < math.factorial(len(start)) // 2
    assert seen_proper > 0


def _closure(gens, n):
    """|<gens>| by enumerating the group (small n only)."""
    ident = tuple(range(n))
    seen, frontier = {ident}, [ident]
    while frontier:
        nxt = []
        for a in frontier:
            for g in gens:
                c = tuple(g[a[i]] for i in range(n))
                if c not in seen:
                    seen.add(c)
                    nxt.append(c)
        frontier = nxt
    return len(seen)


def _mobius(p, a, b, c, d):
    """x -> (a x + b) / (c x + d) on the projective line over F_p (p = infinity)."""
    out = []
    for x in range(p + 1):
        num, den = (a, c) if x == p else ((a * x + b) % p, (c * x + d) % p)
        out.append(p if den % p == 0 else num * pow(den, -1, p) % p)
    return out


def test_primitive_groups_that_are_not_alternating():
    # Primitive groups with prime cycles longer than n - 3 only (no Jordan
    # certificate), which must take the Schreier-Sims path.
    cases = [
        ([_mobius(5, 1, 1, 0, 1), _mobius(5, 2, 0, 0, 1), _mobius(5, 0, 1, 1, 0)], 6, 120),  # PGL(2,5)
        ([_mobius(7, 1, 1, 0, 1), _mobius(7, 2, 0, 0, 1), _mobius(7, 0, 6, 1, 0)], 8, 168),  # PSL(2,7)
        ([_mobius(7, 1, 1, 0, 1), _mobius(7, 3, 0, 0, 1), _mobius(7, 0, 1, 1, 0)], 8, 336),  # PGL(2,7)
        ([[(x + 1) % 7 for x in range(7)], [(3 * x) % 7 for x in range(7)]], 7, 42),        # AGL(1,7)
        ([[(x + 1) % 7 for x in range(7)], [(2 * x) % 7 for x in range(7)]], 7, 21),
    ]
    for gens, n, order in cases:
        assert _closure(gens, n) == order
        assert native.group_order(gens) == order


def test_matches_enumeration_on_random_generator_sets():
    # Symmetric, alternating, intransitive (common fixed points, two orbits)
    # and imprimitive (block-preserving) groups.
    import random
    rng = random.Random(20261203)
    for trial in range(240):
        n = rng.randint(2, 7)
        fixed = rng.randint(0, 2) if n > 3 else 0
        m = n - fixed
        gens = []
        for _ in range(rng.randint(1, 3)):
            mode = rng.random()
            q = list(range(m))
            if mode < 0.4:
                rng.shuffle(q)
            elif mode < 0.7 and m >= 4:
                h = m // 2
                a, b = list(range(h)), list(range(h, m))
                rng.shuffle(a)
                rng.shuffle(b)
                q = a + b
            elif m % 2 == 0:
                blocks = list(range(m // 2))
                rng.shuffle(blocks)
                for i, bi in enumerate(blocks):
                    flip = rng.random() < 0.5
                    q[2 * i], q[2 * i + 1] = (2 * bi + flip, 2 * bi + 1 - flip)
            gens.append(q + list(range(m, n)))
        assert native.group_order(gens) == _closure(gens, n), gens


def test_batched_statics_match_the_python_planner():
    from multigpubfs_b200 import planner
    graphs = [workloads.sweep_instance(i, closed) for i in range(40) for closed in (False, True)]
    graphs += [workloads.planner_instance(i) for i in range(4)]
    graphs.append({"action": {"generators": [[1, 0, 2, 3, 4], [1, 2, 3, 4, 0]]}, "start": [7, 7, 3, 3, 9]})
    statics, states = planner.batch_statics(graphs)
    for row, st_count, g in zip(statics, states, graphs):
        st = planner.graph_statics(g["action"]["generators"], g["start"])
        ref = [st.log_orbit, st.n / 16.0, st.gens / 8.0, float(st.inverse_closed), st.mean_log_order,
               st.max_log_order, st.fixed_fraction, st.cycle_fraction]
        assert [float(x) for x in row] == [float(__import__("numpy").float32(x)) for x in ref]
        if len(set(g["start"])) == len(g["start"]):
            assert int(st_count) == native.group_order(g["action"]["generators"])
    assert int(states[-1]) == 30  # 5! / (2! 2! 1!)
