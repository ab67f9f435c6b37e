"""Test configuration: the `gpu` marker and import paths.

`-m "not gpu"` runs the oracle, host-logic and library-load tests on any CPU
host; `-m gpu` runs the parity tests through the C ABI on a CUDA device.
"""
import json
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
GOLDEN = ROOT / "tests" / "golden"
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (parity tests through libmgbfs2)")


def golden(name):
    return json.loads((GOLDEN / name).read_text())


@pytest.fixture(scope="session")
def exact_cases():
    return golden("exact_cases.json")["cases"]


@pytest.fixture(scope="session")
def lrx_layers():
    return {int(k): v for k, v in golden("lrx_layers.json")["layers"].items()}


@pytest.fixture(scope="session")
def lrx13():
    return golden("lrx13_layers.json")["layers"]


@pytest.fixture(scope="session")
def coxeter_bounds():
    return {int(k): v for k, v in golden("coxeter_bounds.json")["bounds"].items()}


def cuda_available():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def sweep_fixture(key):
    """Oracle layer tables of one batched workload (tests/golden/sweep_tables.json,
    made by tests/golden/make_sweep_golden.py): dict with seed_base,
    generators_sha256 and tables."""
    return golden("sweep_tables.json")[key]


def generator_digest(graph):
    import hashlib
    text = json.dumps(graph["action"]["generators"], separators=(",", ":"))
    return hashlib.sha256(text.encode()).hexdigest()
