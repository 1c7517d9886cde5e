"""Shared fixtures.  GPU tests are marked ``gpu``; everything else runs on the CPU."""
from __future__ import annotations

import json
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

GOLDEN = ROOT / "tests" / "golden" / "reference_golden.json"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs an sm_100 GPU and the built libwlg.so")


@pytest.fixture(scope="session")
def golden():
    return json.loads(GOLDEN.read_text())


@pytest.fixture(scope="session")
def oracle():
    from oracle.oracle import Oracle
    return Oracle()


@pytest.fixture(scope="session")
def reference():
    from oracle.oracle import Reference, reference_available
    if not reference_available():
        pytest.skip("oracle/_ref/libwlref.so was not built (reference sources absent)")
    return Reference()


def unhex(values) -> np.ndarray:
    return np.array([float.fromhex(v) for v in values], dtype=np.float64)
