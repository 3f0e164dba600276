"""Generates ``ensemble_4x4x4x8_b6.json``: the reference's own Metropolis ensemble
plaquette at beta = 6.0 on a 4^3 x 8 lattice, the statistical-parity target of
the GPU sampler.

Eight independent chains of the reference's System::update (oracle/_ref, built
from the reference sources; GLAC/system.cpp:333-361) start from seeded Haar
fields, get NTHERM thermalisation sweeps, then NMEAS sweeps with the plaquette
(GLAC/observables/plaquette.cpp:26-40) after each.  Each chain is seeded
differently (metropolisSeed, randomMatrixSeed).  The fixture stores the mean
over chains, its error from 20 bins per chain, the Gamma-method tau_int of the
plaquette and the acceptance rate.

Run in a container that holds the reference tree: ``python tests/golden/make_ensemble.py``.
"""
import json
import multiprocessing as mp
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

NS, NT, BETA, EPS, NHITS = 4, 8, 6.0, 0.24, 10
NCHAINS, NTHERM, NMEAS = 8, 200, 3000


def chain(i):
    from oracle.oracle import Oracle, Reference

    ref = Reference().configure(NS, NT, beta=BETA, su3eps=EPS, metropolis_seed=1000.0 + i,
                                matrix_seed=2000.0 + i, nupdates=NHITS)
    start = Oracle().haar_field((NS, NS, NS, NT), 31 + i)
    links, _, _ = ref.metropolis_chain(start, NTHERM)
    _, plaq, acc = ref.metropolis_chain(links, NMEAS)
    return plaq, acc


def main():
    from glac_b200.analysis import binned_mean, gamma_method

    with mp.get_context("spawn").Pool(min(NCHAINS, os.cpu_count() or 1)) as pool:
        res = pool.map(chain, range(NCHAINS))
    plaqs = [r[0] for r in res]
    mean, err = binned_mean(plaqs, 20)
    taus = [gamma_method(p).tau_int for p in plaqs]
    out = dict(
        lattice=[NS, NS, NS, NT], beta=BETA, su3_eps=EPS, n_updates=NHITS, chains=NCHAINS,
        therm_sweeps=NTHERM, meas_sweeps=NMEAS, plaquette=mean, plaquette_error=err,
        tau_int_plaquette=float(np.mean(taus)), acceptance=float(np.mean([r[1] for r in res])),
        chain_means=[float(np.mean(p)) for p in plaqs],
        source="reference System::update (oracle/_ref), seeds metropolisSeed=1000+i, randomMatrixSeed=2000+i, "
               "Haar start from the oracle (seed 31+i)",
    )
    with open(os.path.join(HERE, "ensemble_4x4x4x8_b6.json"), "w") as f:
        json.dump(out, f, indent=1)
    print(json.dumps(out))


if __name__ == "__main__":
    main()
