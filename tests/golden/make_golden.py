"""Generates the committed golden fixtures in this folder.

Run where the reference tree exists: its GLAC folder is $GLAC_REF_SRC, by
default ../reference/GLAC beside the repository (the default of
oracle/Makefile too).  Three kinds of fixture:

* ``testcore_fixtures.json`` -- the known-answer matrices of the reference's
  unit tests (GLAC/tests/unit_tests/testcore.cpp:31-232), read as text from
  the reference's ``setComplex`` calls and scalar assignments.
* ``ref_4x4x4x4.npz`` -- outputs of the reference itself (oracle/_ref,
  compiled from its own sources) on a seeded 4^3 x 4 Haar field: staples and
  flow force (first 64 sites), exponentials, three RK3 flow steps, the
  MasterSamplerTopcXYZ observables before and after, and the first 64 links
  of one recorded Metropolis sweep (proposals, uniforms, decisions).
* ``ref_4x4x4x8_b6_flow.npz`` -- a thermalised 4^3 x 8 field from the
  reference's own Metropolis chain (System::update, beta = 6.0, 300 sweeps from
  a seeded Haar field), the reference's MasterSamplerTopcXYZ observables before
  and after each of 100 RK3 flow steps at eps = 0.01 (plaquette 0.589 -> 0.993,
  |Q| >= 0.21 throughout, so every observable has a scale of its own), and the
  first 64 links per direction of the field after the 100 steps.

  python tests/golden/make_golden.py [testcore|ref4|flow]...   (default: all)
"""
import json
import os
import re
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
REF_SRC = os.environ.get("GLAC_REF_SRC", os.path.join(ROOT, "..", "reference", "GLAC"))
REF = os.path.join(REF_SRC, "tests", "unit_tests", "testcore.cpp")


def parse_testcore(path):
    txt = open(path).read()
    mats = {}
    for name, re_, im_, idx in re.findall(r"(\w+)\.setComplex\(complex\(([-\d.]+),([-\d.]+)\),(\d+)\);", txt):
        mats.setdefault(name, {})[int(idx)] = (float(re_), float(im_))
    out = {}
    for name, entries in mats.items():
        n = 18 if max(entries) > 6 else 8
        v = [0.0] * n
        for idx, (a, b) in entries.items():
            v[idx], v[idx + 1] = a, b
        out[name] = v
    m = re.search(r"m_tracedMatrix\s*=\s*([-\d.]+)", txt)
    out["tracedMatrix"] = float(m.group(1))
    return out


def make_testcore():
    fx = parse_testcore(REF)
    with open(os.path.join(HERE, "testcore_fixtures.json"), "w") as f:
        json.dump(fx, f, indent=1, sort_keys=True)


def make_ref4():
    from oracle.oracle import Oracle, Reference
    o, r = Oracle(), Reference()
    N = (4, 4, 4, 4)
    r.configure(4, 4, beta=6.0, su3eps=0.24, flow_eps=0.01, nupdates=10, nflows=3,
                metropolis_seed=11.0, matrix_seed=12.0)
    links = o.haar_field(N, 20261203)
    Z = r.force(links)
    mats = Z.reshape(-1, 18)[:64] * 0.7
    trace = r.metropolis_trace(links)
    K = 64  # links kept from the per-link arrays
    np.savez_compressed(
        os.path.join(HERE, "ref_4x4x4x4.npz"),
        links=links,
        staples=r.staples(links)[:, :K],
        force=Z[:, :K],
        exp_in=mats,
        exp_morningstar=r.exp(mats, 0),
        exp_luscher=r.exp(mats, 1),
        exp_taylor2=r.exp(mats, 2),
        exp_taylor4=r.exp(mats, 3),
        flow3=r.flow(links, 3),
        observables=r.observables(links),
        observables_flow3=r.observables(r.flow(links, 3)),
        plaquette=np.array([r.plaquette(links)]),
        mc_U_before=trace["U_before"][:K], mc_staples=trace["staples"][:K], mc_X=trace["X"][:K],
        mc_r=trace["r"][:K], mc_accept=trace["accept"][:K], mc_order=trace["order"][:K],
    )


def make_flow(nsteps=100, K=64):
    from oracle.oracle import Oracle, Reference
    o, r = Oracle(), Reference()
    N = (4, 4, 4, 8)
    r.configure(4, 8, beta=6.0, su3eps=0.24, flow_eps=0.01, nupdates=10, nflows=nsteps,
                metropolis_seed=31.0, matrix_seed=37.0)
    start, plaq, acc = r.metropolis_chain(o.haar_field(N, 101), 300)
    cur = start
    rows = [r.observables(cur)]
    for _ in range(nsteps):
        cur = r.flow(cur, 1)
        rows.append(r.observables(cur))
    np.savez_compressed(
        os.path.join(HERE, "ref_4x4x4x8_b6_flow.npz"),
        links=start, flow_eps=np.array([0.01]), observables=np.array(rows), links_end=cur[:, :K],
        chain_plaquette=plaq, chain_acceptance=np.array([acc]),
    )


def main(which):
    makers = {"testcore": make_testcore, "ref4": make_ref4, "flow": make_flow}
    for name in which or list(makers):
        makers[name]()


if __name__ == "__main__":
    main(sys.argv[1:])
