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
