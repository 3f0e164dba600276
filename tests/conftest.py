import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); parity tests of the CUDA path")
    config.addinivalue_line("markers", "slow: longer statistical tests")


@pytest.fixture(scope="session")
def oracle():
    from oracle.oracle import Oracle
    return Oracle()


@pytest.fixture(scope="session")
def reference():
    """The reference compiled from its own sources (oracle/_ref); skipped when absent."""
    from oracle.oracle import REF_SO, REF_SRC, Reference
    if not os.path.exists(REF_SO) and not os.path.isdir(REF_SRC):
        pytest.skip("reference library not built here and reference sources absent")
    return Reference()


@pytest.fixture(scope="session")
def golden():
    return dict(np.load(os.path.join(GOLDEN, "ref_4x4x4x4.npz")))


@pytest.fixture(scope="session")
def fixtures():
    import json
    with open(os.path.join(GOLDEN, "testcore_fixtures.json")) as f:
        return {k: np.array(v) for k, v in json.load(f).items()}


def rel_err(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))
