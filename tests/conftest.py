"""Shared fixtures.  `-m gpu` tests need a CUDA device and the built
libwos_b200.so; everything else runs on the CPU (oracle, host logic, the C
ABI's exports)."""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))

GOLDEN = ROOT / "tests" / "golden" / "reference_golden.npz"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and libwos_b200.so")


@pytest.fixture(scope="session")
def golden():
    return dict(np.load(GOLDEN))


@pytest.fixture(scope="session")
def oracle():
    from oracle.oracle import Oracle
    return Oracle()


@pytest.fixture(scope="session")
def reference():
    from oracle.oracle import REF_LIB, Reference
    if not REF_LIB.exists():
        pytest.skip("oracle/_ref is not built (the reference sources are not on this machine)")
    return Reference()


@pytest.fixture(scope="session")
def solver():
    from walk_on_spheres_b200 import Solver
    s = Solver(0)
    yield s
    s.close()
