"""The drop-in boundary on the host: graph contract, CayleyPy dispatch,
run_graph validation, and the C-ABI library exports.  No GPU needed.

Dispatch tests mirror tests/test_cayleypy_backend.py of the reference with
run_graph mocked; since cayleypy is not installed here, a minimal stand-in
module provides CayleyGraph (only its ``bfs`` attribute is patched).
"""
import json
import re
import sys
import types
from pathlib import Path
from types import SimpleNamespace
from unittest.mock import patch

import pytest

import multigpubfs_b200.cayleypy_backend as api
from multigpubfs_b200 import GraphDefinition, from_cayleypy, run_graph
from multigpubfs_b200.graph_definition import _flatten
from multigpubfs_b200 import native

ROOT = Path(__file__).resolve().parents[1]


# ---------------------------------------------------------------------------
# Graph contract (tests/test_graph_definition.py of the reference).

def test_shape_range_and_schema_validation():
    for gs, start in [([[0, 0]], [0, 1]), ([[0, 1]], [0]), ([[0, 1]], [0, 1 << 63])]:
        with pytest.raises(ValueError):
            GraphDefinition.permutation(gs, start)
    with pytest.raises(ValueError):
        GraphDefinition.matrix(2, 1, [([1], 3)], [1, 2])
    with pytest.raises(ValueError):
        GraphDefinition.matrix(1, 1, [([1], 1)], [1])


def test_identity_name_independent_order_sensitive():
    g = GraphDefinition.permutation([[1, 0, 2], [0, 2, 1]], [0, 1, 2], name="a")
    h = GraphDefinition.permutation([[1, 0, 2], [0, 2, 1]], [0, 1, 2], name="b")
    assert g.digest() == h.digest() and g.inverse_closed()
    assert g.digest() != GraphDefinition.permutation(list(reversed(g.action["generators"])), g.start).digest()
    assert GraphDefinition.from_dict(json.loads(g.to_json())).digest() == g.digest()


def test_digest_matches_reference_golden(exact_cases):
    for case in exact_cases:
        g = GraphDefinition.from_dict(case["graph"])
        assert g.digest() == case["digest"], case["name"]
        assert g.inverse_closed() == case["inverse_closed"], case["name"]


def test_cayleypy_adapter():
    x = SimpleNamespace(generators_type=SimpleNamespace(name="PERMUTATION"), generators_permutations=[[1, 0]],
                        central_state=[0, 0], name="coset", generator_names=["x"])
    g = from_cayleypy(x)
    assert g.start == [0, 0] and g.generator_names == ["x"]
    x = SimpleNamespace(generators_type=SimpleNamespace(name="MATRIX"),
                        generators_matrices=[SimpleNamespace(matrix=[[1, 1], [0, 1]], modulo=257)],
                        central_state=[1, 2], name="rect", generator_names=["t"])
    g = from_cayleypy(x)
    assert g.action == {"kind": "matrix", "rows": 2, "cols": 1, "generators": [{"matrix": [1, 1, 0, 1], "modulo": 257}]}


def test_overflow_inverse_guard():
    assert not GraphDefinition.matrix(1, 1, [([(1 << 63) - 1], 3)], [2]).inverse_closed()
    for modulus in (0, 4):
        assert GraphDefinition.matrix(1, 1, [([(1 << 63) - 1], modulus)], [2]).inverse_closed()
    assert GraphDefinition.matrix(1, 1, [([100], 101)], [2]).inverse_closed()


def test_adapter_rejects_fractional_boolean_and_text_labels():
    for bad in (0.5, True, "1", float("inf"), float("nan")):
        with pytest.raises(ValueError):
            _flatten(bad)
    assert _flatten([1.0, -2, 3]) == [1, -2, 3]
    with pytest.raises(ValueError):
        _flatten(1 << 63)


# ---------------------------------------------------------------------------
# CayleyPy dispatch (tests/test_cayleypy_backend.py of the reference).

class FakeCayleyGraph:
    """Stand-in for cayleypy.CayleyGraph: a definition plus an original bfs."""

    def __init__(self, definition):
        self.definition = definition

    def bfs(self, **kwargs):
        return ("torch", kwargs)


@pytest.fixture()
def cayley(tmp_path, monkeypatch):
    module = types.ModuleType("cayleypy")
    module.CayleyGraph = FakeCayleyGraph
    monkeypatch.setitem(sys.modules, "cayleypy", module)
    original = FakeCayleyGraph.bfs
    definition = SimpleNamespace(generators_type=SimpleNamespace(name="PERMUTATION"),
                                 generators_permutations=[[1, 2, 0], [2, 0, 1], [1, 0, 2]],
                                 central_state=[0, 1, 2], name="lrx-3", generator_names=["L", "R", "X"])
    state = SimpleNamespace(graph=FakeCayleyGraph(definition), root=tmp_path, original=original, calls={})
    yield state
    api.disable_native()
    FakeCayleyGraph.bfs = original


def _native(state):
    def fake(definition, output, **kwargs):
        state.calls["definition"] = definition
        state.calls["options"] = kwargs
        output.mkdir(parents=True)
        (output / "states.json").write_text(json.dumps(dict(current=[[2, 1, 0]], previous_small=[[0, 2, 1]])))
        return dict(status="COMPLETE", layer_sizes=[1, 2, 3])
    return fake


def test_simple_call_and_compact_samples(cayley):
    api.enable_native(api.NativeOptions(output_root=cayley.root))
    with patch.object(api, "run_graph", side_effect=_native(cayley)):
        result = cayley.graph.bfs()
    assert result.bfs_completed and result.layer_sizes == [1, 2, 3]
    assert result.diameter() == 2 and result.num_vertices() == 6
    assert set(result.layer_samples) == {1, 2} and result.layers == {}
    assert cayley.calls["options"]["devices"] is None and cayley.calls["options"]["autotune"] is True
    with pytest.raises(KeyError):
        result.last_layer()


def test_disable_and_reenable(cayley):
    api.enable_native()
    api.enable_native()
    api.disable_native()
    assert FakeCayleyGraph.bfs is cayley.original


def test_one_shot_does_not_patch(cayley):
    with patch.object(api, "run_graph", side_effect=_native(cayley)):
        api.bfs(cayley.graph, output=cayley.root / "one")
    assert FakeCayleyGraph.bfs is cayley.original


def test_torch_preserves_kwargs(cayley):
    api.enable_native()
    assert cayley.graph.bfs(backend="torch", max_diameter=2) == ("torch", dict(max_diameter=2))


def test_unsupported_before_launch(cayley):
    api.enable_native()
    for kwargs in (dict(return_all_edges=True), dict(max_diameter=2), dict(max_layer_size_to_store=None),
                   dict(misspelled=True)):
        with patch.object(api, "run_graph") as run:
            with pytest.raises(NotImplementedError):
                cayley.graph.bfs(**kwargs)
            run.assert_not_called()


def test_single_decoded_start(cayley):
    with patch.object(api, "run_graph", side_effect=_native(cayley)):
        api.bfs(cayley.graph, output=cayley.root / "start", start_states=[[2, 1, 0]])
    assert cayley.calls["definition"].start == [2, 1, 0]


def test_multisource_rejected(cayley):
    with pytest.raises(NotImplementedError):
        api.bfs(cayley.graph, start_states=[[0, 1, 2], [2, 1, 0]])


def test_incomplete_not_diameter(cayley):
    def incomplete(*args, **kwargs):
        report = _native(cayley)(*args, **kwargs)
        report["status"] = "INCOMPLETE"
        return report
    with patch.object(api, "run_graph", side_effect=incomplete):
        result = api.bfs(cayley.graph, output=cayley.root / "partial")
    assert not result.bfs_completed
    with pytest.raises(RuntimeError):
        result.diameter()


def test_runtime_failure_no_cpu_restart(cayley):
    with patch.object(api, "run_graph", side_effect=RuntimeError("GPU failed")):
        with pytest.raises(RuntimeError, match="GPU failed"):
            api.bfs(cayley.graph, backend="auto", output=cayley.root / "failed")


def test_auto_falls_back_only_for_unsupported_options(cayley):
    api.enable_native(default_backend="auto")
    with patch.object(api, "run_graph") as run:
        assert cayley.graph.bfs(return_all_edges=True) == ("torch", dict(return_all_edges=True))
        run.assert_not_called()


def test_full_retained_layer_is_available(cayley):
    def full(*args, **kwargs):
        report = _native(cayley)(*args, **kwargs)
        report["layer_sizes"] = [1, 1, 1]
        return report
    with patch.object(api, "run_graph", side_effect=full):
        result = api.bfs(cayley.graph, output=cayley.root / "full")
    assert result.last_layer().tolist() == [[2, 1, 0]]


def test_explicit_devices_and_budget_forwarded(cayley):
    with patch.object(api, "run_graph", side_effect=_native(cayley)):
        api.bfs(cayley.graph, output=cayley.root / "devices",
                native_options=api.NativeOptions(devices=(1, 0), max_seconds=12, autotune=False))
    assert cayley.calls["options"] == dict(devices=(1, 0), max_seconds=12, autotune=False, memory_backend="legacy",
                                           segment_rows=1 << 32, memory_preset="balanced", segment_strategy="atomic",
                                           bitmap_owner_page=None)


def test_explicit_memory_backend_and_planner_forwarded(cayley):
    for backend in ("segmented24", "permutation_bitmap"):
        with patch.object(api, "run_graph", side_effect=_native(cayley)):
            api.bfs(cayley.graph, output=cayley.root / backend, native_options=api.NativeOptions(memory_backend=backend))
        assert cayley.calls["options"]["memory_backend"] == backend
    with patch.object(api, "run_graph", side_effect=_native(cayley)):
        api.bfs(cayley.graph, output=cayley.root / "learned", native_options=api.NativeOptions(planner="learned"))
    assert cayley.calls["options"]["planner"] == "learned"


def test_collision_with_other_integration(cayley):
    api.enable_native()
    installed = FakeCayleyGraph.bfs
    FakeCayleyGraph.bfs = lambda graph: None
    try:
        with pytest.raises(RuntimeError):
            api.disable_native()
    finally:
        FakeCayleyGraph.bfs = installed


def test_native_options_validation():
    with pytest.raises(ValueError):
        api.NativeOptions(memory_preset="huge")
    with pytest.raises(ValueError):
        api.NativeOptions(segment_rows=0)
    with pytest.raises(ValueError):
        api.NativeOptions(bitmap_owner_page=3, memory_backend="permutation_bitmap")
    with pytest.raises(ValueError):
        api.NativeOptions(bitmap_owner_page=4)
    with pytest.raises(ValueError):
        api.NativeOptions(segment_strategy="fast")
    with pytest.raises(ValueError):
        api.NativeOptions(planner="oracle")


# ---------------------------------------------------------------------------
# run_graph argument validation (launch.py:151-186 of the reference); every
# case is rejected before any device work.

@pytest.mark.parametrize("kwargs,code", [
    (dict(device=0, devices=[0]), "DEVICE_SELECTION_CONFLICT"),
    (dict(device=-1), "INVALID_DEVICE"),
    (dict(devices=[0, 0]), "INVALID_DEVICES"),
    (dict(devices=[0, 1]), "MULTI_DEVICE_NOT_BUILT"),
    (dict(shards=0), "INVALID_SHARDS"),
    (dict(autotune=1), "INVALID_AUTOTUNE"),
    (dict(memory_backend="ram"), "INVALID_MEMORY_BACKEND"),
    (dict(segment_strategy="warp"), "SEGMENT_STRATEGY_REQUIRES_SEGMENTED_BACKEND"),
    (dict(bitmap_owner_page=8), "BITMAP_OWNER_PAGE_REQUIRES_BITMAP"),
    (dict(capacity=0), "INVALID_CAPACITY"),
    (dict(planner="oracle"), "INVALID_PLANNER"),
    (dict(max_seconds=0), "INVALID_MAX_SECONDS"),
])
def test_run_graph_validation(tmp_path, kwargs, code):
    g = GraphDefinition.permutation([[1, 2, 0]], [0, 1, 2])
    with pytest.raises(ValueError, match=code):
        run_graph(g, tmp_path / "out", **kwargs)


def test_bitmap_requires_permutation(tmp_path):
    g = GraphDefinition.matrix(1, 1, [([2], 7)], [3])
    with pytest.raises(ValueError, match="BITMAP_REQUIRES_PERMUTATION_ACTION"):
        run_graph(g, tmp_path / "out", memory_backend="permutation_bitmap")


def test_existing_output_rejected(tmp_path):
    g = GraphDefinition.permutation([[1, 2, 0]], [0, 1, 2])
    (tmp_path / "out").mkdir()
    with pytest.raises(FileExistsError):
        run_graph(g, tmp_path / "out")


# ---------------------------------------------------------------------------
# The C-ABI library: built for sm_100a, loads, exports every declared symbol.

def _declared_symbols():
    text = (ROOT / "include" / "mgbfs2.h").read_text()
    return sorted(set(re.findall(r"\b(mgbfs2_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    import ctypes
    from multigpubfs_b200 import build
    build.build()
    lib = ctypes.CDLL(str(build.LIBRARY))
    declared = _declared_symbols()
    assert len(declared) >= 14
    for name in declared:
        assert hasattr(lib, name), name
    assert set(native.exported_symbols()) == set(declared)


def test_native_binding_loads_without_device():
    lib = native.load()
    assert lib.mgbfs2_status_string(0) == b"OK"
    assert lib.mgbfs2_status_string(2) == b"UNSUPPORTED"


def test_no_cpu_fallback_without_device(tmp_path):
    import torch
    if torch.cuda.is_available():
        pytest.skip("device present")
    g = GraphDefinition.permutation([[1, 2, 0]], [0, 1, 2])
    with pytest.raises(native.NativeUnavailable):
        run_graph(g, tmp_path / "out")


def test_ctypes_mirrors_match_the_header_layout(tmp_path):
    """Every ctypes structure of multigpubfs_b200.native has the size and the
    field offsets of its struct in include/mgbfs2.h, as gcc lays it out (a
    field renamed or moved in one and not the other fails here, on CPU)."""
    import ctypes as C
    import shutil
    import subprocess
    from pathlib import Path

    from multigpubfs_b200 import native
    if not shutil.which("gcc"):
        pytest.skip("gcc not available")
    pairs = {"mgbfs2_graph_desc": native.GraphDesc, "mgbfs2_plan_request": native.PlanRequest,
             "mgbfs2_plan_info": native.PlanInfo, "mgbfs2_run_limits": native.RunLimits,
             "mgbfs2_status": native.RunStatus, "mgbfs2_batch_options": native.BatchOptions,
             "mgbfs2_batch_status": native.BatchStatus}
    root = Path(__file__).resolve().parents[1]
    lines = ["#include <stddef.h>", "#include <stdio.h>", '#include "mgbfs2.h"', "int main(void) {"]
    for cname, py in pairs.items():
        lines.append(f'  printf("{cname} size %zu\\n", sizeof({cname}));')
        for field, _ in py._fields_:
            lines.append(f'  printf("{cname} {field} %zu\\n", offsetof({cname}, {field}));')
    lines += ["  return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c11", "-I", str(root / "include"), str(src), "-o", str(exe)], check=True,
                   capture_output=True, text=True)
    got = {}
    for line in subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.splitlines():
        cname, field, value = line.split()
        got[(cname, field)] = int(value)
    for cname, py in pairs.items():
        assert got[(cname, "size")] == C.sizeof(py), cname
        for field, _ in py._fields_:
            assert got[(cname, field)] == getattr(py, field).offset, (cname, field)
