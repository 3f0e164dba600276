"""The benchmark size 32^3 x 64 (2,097,152 sites).

Parity with the reference itself (oracle/_ref, the GLAC sources compiled
here): on the benchmark's own start field (seeded Haar field + 600 FP32
Metropolis sweeps at beta = 6.2), one RK3 step of Flow::flowField
(GLAC/flow/flow.cpp:43-73) and MasterSamplerTopcXYZ::calculate
(GLAC/observables/mastersamplertopcxyz.cpp:236-384) before and after it, in
FP64 (<= 1e-12) and FP32 (<= 1e-5), observables quantity by quantity.  The
reference takes a few minutes of CPU for this; the two reference runs go to
two spawned processes.

Properties that hold at any size: gauge invariance (the reference's own
check, latticeoperations.cpp:750-813), covariance under a one-site shift in
time (which swaps the parities of every site), the sign change of Q and q(t)
under a reflection x -> -x, FP32 against FP64 over a flow,
sweeps that compose, per-site densities that sum to the global observables,
and unitarity after the flow."""
import multiprocessing as mp
import os
import tempfile

import numpy as np
import pytest

from conftest import ROOT, assert_obs_close, obs_errors, rel_err
from test_oracle import flip_charge, gauge_transform, reflect_x

pytestmark = pytest.mark.gpu

N = (32, 32, 32, 64)
TOL = {"fp64": 1e-12, "fp32": 1e-5}
Q_TOL = {"fp64": 1e-9, "fp32": 1e-3}


@pytest.fixture(scope="module")
def g():
    import glac_b200
    return glac_b200


@pytest.fixture(scope="module")
def start(g):
    """A Haar start after 5 FP64 sweeps at beta = 6.2 (host layout, FP64)."""
    with g.Lattice(N, beta=6.2, precision="fp64", seed=7) as L:
        L.hot_start(7)
        L.metropolis(5)
        return L.get_links()


@pytest.fixture(scope="module")
def bench_start(g):
    """bench.py's start field: Haar(20261203), 5 sweeps, reunitarised, 595
    sweeps, reunitarised; FP32 at beta = 6.2, 10 hits, SU3Eps = 0.24."""
    with g.Lattice(N, beta=6.2, precision="fp32", n_updates=10, su3_eps=0.24, flow_eps=0.01, seed=20261203,
                   stream_id=0, reunit_interval=0) as L:
        L.hot_start(20261203)
        L.metropolis(5)
        L.reunitarize()
        L.metropolis(595)
        L.reunitarize()
        return L.get_links()


def _reference_leg(args):
    """Spawned worker: the reference's observables of the field in `path`, or
    (job "flow") its observables after one RK3 step, with the flowed field
    written to `out`."""
    path, job, out = args
    import sys
    sys.path.insert(0, ROOT)
    from oracle.oracle import Reference
    links = np.load(path)
    r = Reference().configure(N[0], N[3], beta=6.2, flow_eps=0.01, nflows=1)
    if job == "obs":
        return r.observables(links)
    flowed = r.flow(links, 1)
    np.save(out, flowed)
    return r.observables(flowed)


@pytest.fixture(scope="module")
def reference_step(bench_start, reference):
    """(observables before, observables after, field after) of one reference RK3 step."""
    with tempfile.TemporaryDirectory() as d:
        src, dst = os.path.join(d, "start.npy"), os.path.join(d, "flowed.npy")
        np.save(src, bench_start)
        with mp.get_context("spawn").Pool(2) as pool:
            obs0, obs1 = pool.map(_reference_leg, [(src, "obs", None), (src, "flow", dst)])
        return obs0, obs1, np.load(dst)


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_one_flow_step_vs_reference_full_size(g, bench_start, reference_step, prec):
    obs0, obs1, flowed = reference_step
    with g.Lattice(N, beta=6.2, precision=prec, flow_eps=0.01) as L:
        L.set_links(bench_start)
        obs = L.flow(1)
        links = L.get_links()
    e0 = assert_obs_close(obs[0], obs0, TOL[prec], f"{prec} t = 0")
    e1 = assert_obs_close(obs[1], obs1, TOL[prec], f"{prec} after one step")
    assert rel_err(links, flowed) < TOL[prec]
    print(prec, "32^3x64 relative errors: t = 0", e0, "after one step", e1,
          "links", rel_err(links, flowed))


def measured(g, links, prec):
    with g.Lattice(N, beta=6.2, precision=prec) as L:
        L.set_links(links)
        return L.measure()


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_gauge_invariance_full_size(g, oracle, start, prec):
    W = oracle.haar_field(N, 99)[0].copy()
    a = measured(g, start, prec)
    b = measured(g, gauge_transform(start, W, N), prec)
    assert rel_err(b[[0, 2]], a[[0, 2]]) < TOL[prec]
    assert np.max(np.abs(b[1:2] - a[1:2])) < Q_TOL[prec]
    assert np.max(np.abs(b[3:] - a[3:])) < Q_TOL[prec]  # q(t) per slice


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_time_shift_covariance_full_size(g, start, prec):
    # U'(x, t) = U(x, t - 1): every site changes parity; globals stay, q(t) rolls by one slice
    shifted = np.roll(start.reshape(4, N[3], N[2] * N[1] * N[0], 18), 1, axis=1).reshape(start.shape)
    a = measured(g, start, prec)
    b = measured(g, shifted, prec)
    assert rel_err(b[[0, 2]], a[[0, 2]]) < TOL[prec]
    assert abs(b[1] - a[1]) < Q_TOL[prec]
    assert np.max(np.abs(b[3:] - np.roll(a[3:], 1))) < Q_TOL[prec]


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_reflection_flips_the_charge_full_size(g, start, prec):
    # x -> -x reverses the orientation: the plaquette and E stay, Q and q(t)
    # change sign, at t = 0 and over 10 flow steps (the flow commutes with it)
    obs = {}
    for name, f in (("a", start), ("r", reflect_x(start, N))):
        with g.Lattice(N, beta=6.2, precision=prec, flow_eps=0.01) as L:
            L.set_links(f)
            obs[name] = L.flow(10)
    r, fa = obs["r"], flip_charge(obs["a"])
    e = obs_errors(r[:, [0, 2]], fa[:, [0, 2]], scalars=("plaq", "energy"), slices=())
    assert max(e.values()) < 10 * TOL[prec], e
    assert np.max(np.abs(r[:, 1] - fa[:, 1])) < Q_TOL[prec]
    assert np.max(np.abs(r[:, 3:] - fa[:, 3:])) < Q_TOL[prec]
    print(prec, "reflection: plaq/E", e, "Q at t = 0 and after 10 steps", obs["a"][[0, -1], 1],
          "max |dQ|", np.max(np.abs(r[:, 1] - fa[:, 1])))


def test_fp32_flow_tracks_fp64_full_size(g, start):
    obs = {}
    for prec in ("fp64", "fp32"):
        with g.Lattice(N, beta=6.2, precision=prec, flow_eps=0.01) as L:
            L.set_links(start)
            obs[prec] = L.flow(20)
            if prec == "fp32":
                assert L.unitarity_violation() < 1e-5
    a, b = obs["fp64"], obs["fp32"]
    assert a.shape == (21, 3 + N[3])
    e = obs_errors(b, a)
    print("FP32 vs FP64 over 20 flow steps:", e)
    assert e["plaq"] < TOL["fp32"] and e["energy"] < TOL["fp32"]
    assert np.max(np.abs(b[:, 1] - a[:, 1])) < Q_TOL["fp32"]
    assert np.all(np.diff(a[:, 0]) > 0)  # the flow smooths: plaquette rises every step


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_sweeps_compose_full_size(g, start, prec):
    with g.Lattice(N, beta=6.2, precision=prec, seed=5) as A, g.Lattice(N, beta=6.2, precision=prec, seed=5) as B:
        A.set_links(start)
        B.set_links(start)
        acc_a = A.metropolis(2)
        acc_b = B.metropolis(1) + B.metropolis(1)
        assert A.sweep == B.sweep == 2
        assert np.array_equal(A.get_links(), B.get_links())
        assert abs(acc_a - acc_b / 2) < 1e-12
        assert 0.02 < acc_a < 0.8


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_densities_sum_to_globals_full_size(g, start, prec):
    with g.Lattice(N, beta=6.2, precision=prec) as L:
        L.set_links(start)
        obs, q, e = L.measure_density()
        assert rel_err(obs, L.measure()) < 1e-14
    assert q.shape == e.shape == (int(np.prod(N)),)
    assert abs(q.sum() - obs[1]) < 1e-9
    assert abs(e.sum() / q.size - obs[2]) < 1e-10 * abs(obs[2])
    # q(t) per slice from the density, lexicographic order with t slowest
    qt = q.reshape(N[3], -1).sum(axis=1)
    assert np.max(np.abs(qt - obs[3:])) < 1e-9
