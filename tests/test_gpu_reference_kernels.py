"""The reference's own GPU BFS (gpu/cayley_bfs.cu, built for sm_100a into
oracle/_ref by `make -C oracle ref-gpu`) run on the same B200: its layer
tables for S_8..S_10 under the adjacent transpositions, in both of its kernel
variants and both candidate layouts, equal the Mahonian layer sizes and this
engine's tables."""
import pytest

from oracle import graph_oracle as G

pytestmark = pytest.mark.gpu


def _ref():
    from oracle import ref_gpu
    if not ref_gpu.available():
        pytest.skip("reference GPU library not built (oracle/_ref)")
    return ref_gpu


@pytest.mark.parametrize("n", [8, 9, 10])
def test_reference_gpu_bfs_matches_this_engine(n):
    ref_gpu = _ref()
    from multigpubfs_b200 import GraphDefinition
    from multigpubfs_b200.engine import NativeGraph
    expect = G.coxeter_layers(n)
    with NativeGraph(GraphDefinition.permutation(G.coxeter_generators(n), list(range(n)))) as e:
        e.plan()
        ours = e.run().layer_sizes
    assert ours == expect
    with ref_gpu.CayleyBfs(n) as ref:
        for variant in (0, 1):
            for layout in (0, 1):
                sizes, kernel_ms, _ = ref.run(variant, layout)
                assert sizes == expect, (variant, layout)
                assert kernel_ms > 0
