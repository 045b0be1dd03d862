"""Test configuration: the ``gpu`` marker, import paths and shared fixtures.

GPU tests (``-m gpu``) call the CUDA engine through the C ABI and compare with the
CPU oracle in ``oracle/``.  CPU tests (``-m "not gpu"``) pin the oracle to the
reference's golden vectors, check the host compiler and the C ABI symbol table.
"""
import json
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
GOLDEN = ROOT / "tests" / "golden"
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

import __graft_entry__  # noqa: E402

rgs = __graft_entry__.package()


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); calls the CUDA engine through the C ABI")


def pytest_collection_modifyitems(config, items):
    import torch

    if torch.cuda.is_available():
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for item in items:
        if "gpu" in item.keywords:
            item.add_marker(skip)


@pytest.fixture(scope="session")
def pkg():
    return rgs


@pytest.fixture(scope="session")
def golden_plans():
    return json.loads((GOLDEN / "plans.json").read_text())


@pytest.fixture(scope="session")
def golden_amplitudes():
    return json.loads((GOLDEN / "amplitudes.json").read_text())


@pytest.fixture(scope="session")
def fixtures():
    return dict(np.load(GOLDEN / "fixtures.npz"))


@pytest.fixture(scope="session")
def rgs70_records():
    return json.loads((GOLDEN / "rgs70_c128.json").read_text())


def graph_from_edges(n, edges):
    g = np.zeros((n, n), dtype=np.uint8)
    for a, b in edges:
        g[a, b] = g[b, a] = 1
    return g


def unitaries_from_json(u):
    return np.array([[[complex(*z) for z in row] for row in m] for m in u])
