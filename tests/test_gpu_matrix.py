"""Int64 matrix groups on the wide-key path at sizes where one state is often
claimed by several threads in the same layer: SL(2, p) on 2x2 matrices,
against the reference's own exact_layers tables (tests/golden/matrix_groups.json)
on repeated runs, and the group order p(p^2 - 1) beyond the fixtures."""
import pytest

from tests.conftest import golden

pytestmark = pytest.mark.gpu


def _sl2(p):
    from multigpubfs_b200 import GraphDefinition
    gens = [([1, 1, 0, 1], p), ([1, 0, 1, 1], p), ([1, p - 1, 0, 1], p), ([1, 0, p - 1, 1], p)]
    return GraphDefinition.matrix(2, 2, gens, [1, 0, 0, 1])


@pytest.mark.parametrize("case", ["sl2_mod31", "sl2_mod101"])
def test_sl2_tables_match_the_reference_on_every_run(case):
    from multigpubfs_b200 import GraphDefinition
    from multigpubfs_b200.engine import NativeGraph
    fx = golden("matrix_groups.json")["cases"][case]
    g = GraphDefinition.from_dict(fx["graph"])
    with NativeGraph(g) as e:
        e.plan()
        for _ in range(6):
            r = e.run()
            assert r.complete and r.layer_sizes == fx["layers"]


@pytest.mark.parametrize("p", [211, 251])
def test_sl2_orbit_is_the_group_order(p):
    from multigpubfs_b200.engine import NativeGraph
    with NativeGraph(_sl2(p)) as e:
        e.plan()
        for _ in range(3):
            r = e.run()
            assert r.complete and r.states == p * (p * p - 1)
