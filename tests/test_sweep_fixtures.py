"""The batched-sweep and planner fixtures (tests/golden/sweep_tables.json) are
the oracle's tables for exactly the instances the library's workloads
generate: the seeded generators hash to the recorded digests, every table
settles |<generators>| states (Schreier-Sims, host code of libmgbfs2), and the
Python restatement of the reference's exact_layers reproduces the small ones.
No GPU needed."""
import pytest

from multigpubfs_b200 import native, workloads
from oracle import graph_oracle as G
from tests.conftest import generator_digest, sweep_fixture

SETS = {
    "sweep512": lambda: workloads.sweep(512),
    "sweep512_heldout": lambda: workloads.sweep(512, seed_base=20261203 + 4096),
    "planner_s12": lambda: [workloads.planner_instance(i) for i in sweep_fixture("planner_s12")["indices"]],
}


@pytest.mark.parametrize("key", sorted(SETS))
def test_fixture_covers_the_workload(key):
    fixture = sweep_fixture(key)
    graphs = SETS[key]()
    assert len(graphs) == len(fixture["tables"]) == len(fixture["generators_sha256"])
    assert [generator_digest(g) for g in graphs] == fixture["generators_sha256"]
    for g, table in zip(graphs, fixture["tables"]):
        assert table[0] == 1 and all(x > 0 for x in table)
        assert sum(table) == native.group_order(g["action"]["generators"])


def test_small_instances_match_python_oracle():
    fixture = sweep_fixture("sweep512")
    graphs = workloads.sweep(512)
    small = [(g, t) for g, t in zip(graphs, fixture["tables"]) if len(g["start"]) <= 8][:24]
    assert len(small) == 24
    for g, table in small:
        assert G.layer_sizes(g, 10 ** 6) == table
