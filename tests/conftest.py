"""Shared fixtures.  GPU tests carry @pytest.mark.gpu; everything else runs on CPU."""
import json
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))

GOLDEN = ROOT / "tests" / "golden"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the built native library")


@pytest.fixture(scope="session")
def golden():
    z = np.load(GOLDEN / "reference_golden.npz")
    return {k: z[k] for k in z.files}


@pytest.fixture(scope="session")
def golden_meta():
    return json.loads((GOLDEN / "reference_golden.json").read_text())


@pytest.fixture(scope="session")
def restatement():
    from oracle.oracle import RESTATEMENT, Restatement, build
    if not RESTATEMENT.exists():
        build(reference=False)
    return Restatement()


def rel_linf(a, b):
    """max |a-b| / max |b| per conserved field, the worst field."""
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    axes = tuple(range(1, a.ndim))
    den = np.maximum(np.abs(b).max(axis=axes), 1e-300)
    return float((np.abs(a - b).max(axis=axes) / den).max())
