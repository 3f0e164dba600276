"""Statistical parity of the GPU Metropolis sampler with the reference's own chain.

The fixture ``golden/ensemble_4x4x4x8_b6.json`` holds the reference's ensemble
plaquette at beta = 6.0 on 4^3 x 8 (eight chains of System::update, 200
thermalisation + 3000 measured sweeps each; made by golden/make_ensemble.py).
The GPU checkerboard sampler (Philox streams, the same RST proposals and accept
rule) must reproduce it within statistical errors: |mean - ref| < 3 sigma, sigma
the two errors combined.
"""
import json
import os

import numpy as np
import pytest

from glac_b200.analysis import binned_mean

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.fixture(scope="module")
def g():
    import glac_b200
    return glac_b200


def _fixture():
    with open(os.path.join(HERE, "golden", "ensemble_4x4x4x8_b6.json")) as f:
        return json.load(f)


def gpu_chains(g, ref, precision, nchains=8):
    N = tuple(ref["lattice"])
    plaqs, accs = [], []
    for i in range(nchains):
        with g.Lattice(N, beta=ref["beta"], precision=precision, n_updates=ref["n_updates"],
                       su3_eps=ref["su3_eps"], seed=500 + i) as L:
            L.hot_start(77 + i)
            L.metropolis(ref["therm_sweeps"])
            p = np.empty(ref["meas_sweeps"])
            a = 0.0
            for k in range(p.size):
                a += L.metropolis(1)
                p[k] = L.measure()[0]
            plaqs.append(p)
            accs.append(a / p.size)
    return plaqs, float(np.mean(accs))


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_ensemble_plaquette_matches_reference(g, precision):
    ref = _fixture()
    plaqs, acc = gpu_chains(g, ref, precision)
    mean, err = binned_mean(plaqs, 20)
    sigma = np.hypot(err, ref["plaquette_error"])
    assert abs(mean - ref["plaquette"]) < 3 * sigma, (mean, err, ref["plaquette"], ref["plaquette_error"])
    # same proposals and accept rule: the acceptance rate agrees too
    assert abs(acc - ref["acceptance"]) < 0.01, (acc, ref["acceptance"])
