"""Generates the committed golden fixtures in this folder.

Run in a container that holds the reference tree (its path is the REF_SRC
default of oracle/Makefile).  Two kinds of fixture:

* ``testcore_fixtures.json`` -- the known-answer matrices of the reference's
  unit tests (GLAC/tests/unit_tests/testcore.cpp:31-232), read as text from
  the reference's ``setComplex`` calls and scalar assignments.
* ``ref_4x4x4x4.npz`` -- outputs of the reference itself (oracle/_ref,
  compiled from its own sources) on a seeded 4^3 x 4 Haar field: staples and
  flow force (first 64 sites), exponentials, three RK3 flow steps, the
  MasterSamplerTopcXYZ observables before and after, and the first 64 links
  of one recorded Metropolis sweep (proposals, uniforms, decisions).
"""
import json
import os
import re
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
REF = "/root/reference/GLAC/tests/unit_tests/testcore.cpp"


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


def main():
    fx = parse_testcore(REF)
    with open(os.path.join(HERE, "testcore_fixtures.json"), "w") as f:
        json.dump(fx, f, indent=1, sort_keys=True)

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


if __name__ == "__main__":
    main()
