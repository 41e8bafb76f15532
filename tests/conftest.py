import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
GOLDEN = os.path.join(ROOT, "tests", "golden")
# Root of a checkout of the reference (Ship-Vano/FluidPrjct), when one is at
# hand: tests that read its files directly use it, the others read the
# committed fixtures that tests/golden/make_golden.py made from it.
REFERENCE = os.environ.get("FLUIDPRJCT_REFERENCE", "")


def reference_file(*parts):
    """Path of a file of the reference checkout, or None without one."""
    if not REFERENCE:
        return None
    p = os.path.join(REFERENCE, *parts)
    return p if os.path.exists(p) else None


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); run with -m gpu")


@pytest.fixture(scope="session")
def O():
    """The CPU oracle (test infrastructure)."""
    from oracle import oracle
    oracle.lib()
    return oracle


@pytest.fixture(scope="session")
def golden():
    with open(os.path.join(GOLDEN, "golden.json")) as f:
        return json.load(f)


@pytest.fixture(scope="session")
def golden_particles():
    return np.load(os.path.join(GOLDEN, "particles_m1.npz"))["pos"]


@pytest.fixture(scope="session")
def golden_labels():
    z = np.load(os.path.join(GOLDEN, "labels_fixtures.npz"))
    return {k: z[k] for k in z.files}


def rel_l2(a, b):
    a = np.asarray(a, np.float64).ravel()
    b = np.asarray(b, np.float64).ravel()
    den = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (den if den > 0 else 1.0))
