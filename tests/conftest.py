"""Shared fixtures. `-m "not gpu"` runs the oracle, host-ABI and CLI tests on the CPU;
`-m gpu` runs the parity tests of the CUDA paths against the oracle."""
from __future__ import annotations

import json
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
GOLDEN = ROOT / "tests" / "golden"
sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session")
def built():
    """The library and the oracle, built in-tree when missing (both builds are incremental)."""
    from dsmc_suite_b200 import build as B
    from oracle import oracle as O
    B.build()
    O.build()
    return True


@pytest.fixture(scope="session")
def N(built):
    from dsmc_suite_b200 import _native
    return _native


@pytest.fixture(scope="session")
def O(built):
    from oracle import oracle
    return oracle


@pytest.fixture(scope="session")
def golden():
    runs = dict(np.load(GOLDEN / "reference_runs.npz"))
    scal = dict(np.load(GOLDEN / "reference_scalars.npz"))
    meta = json.loads((GOLDEN / "reference_meta.json").read_text())
    return {"runs": runs, "scalars": scal, "meta": meta}


@pytest.fixture(scope="session")
def ctx(built):
    from dsmc_suite_b200 import Context
    c = Context(0)
    yield c
    c.close()


def cold_T(N, ftd=36, ffd=72):
    """Synthetic map with a 60 K night side and fully cold polar rows (freeze paths fire)."""
    T = N.latlon_temperature(ftd, ffd, T_ss=235.0, T_floor=60.0)
    T[:2, :] = 50.0
    T[-2:, :] = 50.0
    return T
