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


OBS_SCALARS = ("plaq", "topc", "energy")


def obs_errors(a, b, scalars=OBS_SCALARS, slices=("topct",)):
    """Relative errors of observable vectors, one figure per quantity.

    a, b: one vector or rows of vectors laid out as the named scalars followed
    by equally long per-time-slice arrays ([plaq, topc, energy, topct[Nt]] by
    default).  Each scalar is compared with its own value, each per-slice
    array against the largest |entry| of that array in the same row.
    Returns {name: max over rows}.
    """
    a = np.atleast_2d(np.asarray(a, np.float64))
    b = np.atleast_2d(np.asarray(b, np.float64))
    assert a.shape == b.shape, (a.shape, b.shape)
    ns = len(scalars)
    out = {}
    for i, name in enumerate(scalars):
        out[name] = float(np.max(np.abs(a[:, i] - b[:, i]) / np.abs(b[:, i])))
    rest = b.shape[1] - ns
    if slices and rest:
        nt = rest // len(slices)
        assert nt * len(slices) == rest, (rest, slices)
        for k, name in enumerate(slices):
            sl = slice(ns + k * nt, ns + (k + 1) * nt)
            scale = np.max(np.abs(b[:, sl]), axis=1)
            out[name] = float(np.max(np.max(np.abs(a[:, sl] - b[:, sl]), axis=1) / scale))
    return out


def assert_obs_close(a, b, tol, what="", **kw):
    """Every per-quantity relative error of obs_errors(a, b) at most tol."""
    e = obs_errors(a, b, **kw)
    assert max(e.values()) <= tol, f"{what}: per-observable relative errors {e} above {tol}"
    return e
