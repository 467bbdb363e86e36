"""Shared test setup: import paths, the gpu marker, fixtures."""
from __future__ import annotations

import json
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
PKG = ROOT / "wwocl-boinc_b200"
GOLDEN = ROOT / "tests" / "golden"
for p in (ROOT, PKG):
    if str(p) not in sys.path:
        sys.path.insert(0, str(p))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session")
def oracle():
    from oracle.oracle import Oracle

    return Oracle()


@pytest.fixture(scope="session")
def ref_ranges():
    return json.loads((GOLDEN / "ref_ranges.json").read_text())


@pytest.fixture(scope="session")
def ref_prps():
    return json.loads((GOLDEN / "ref_prps.json").read_text())


@pytest.fixture(scope="session")
def ref_terms():
    return dict(np.load(GOLDEN / "ref_terms.npz"))


@pytest.fixture(scope="session")
def tests_txt():
    return json.loads((GOLDEN / "tests_txt.json").read_text())


@pytest.fixture(scope="session")
def ww():
    import wwcuda

    return wwcuda


def sample_names(terms: dict) -> list[str]:
    return sorted({k[: -len("_p")] for k in terms if k.endswith("_p")})
