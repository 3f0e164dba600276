"""The batched ensemble (glac_ensemble_*) against single-lattice contexts.

Lattice i of an ensemble draws from Philox stream stream_id + i, exactly as a
single context with that stream id, and runs the same kernel bodies; so its
start field, its sweeps and its flow observables agree with that context's.
The CUDA-graph schedule equals the eager one, and replays draw fresh numbers.
"""
import numpy as np
import pytest

from conftest import assert_obs_close

pytestmark = pytest.mark.gpu

DIMS = [(4, 4, 4, 8), (6, 4, 4, 4), (8, 8, 8, 16), (4, 6, 8, 10)]
BETAS = [6.0, 5.7, 6.2, 6.45]
SEED = 0x51D


@pytest.fixture(scope="module")
def g():
    import glac_b200
    return glac_b200


@pytest.fixture(scope="module")
def ens():
    from glac_b200 import ensemble
    return ensemble


def rel(a, b):
    return np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300)


@pytest.mark.parametrize("prec,tol", [("fp64", 1e-12), ("fp32", 1e-5)])
def test_ensemble_matches_single_contexts(g, ens, prec, tol):
    with ens.Ensemble(DIMS, BETAS, precision=prec, seed=SEED, stream_id=7, flow_eps=0.02) as E:
        E.hot_start(99)
        acc = E.metropolis(3)
        obs = E.flow(4)
        links = [E.get_links(i) for i in range(len(DIMS))]
    for i, (d, b) in enumerate(zip(DIMS, BETAS)):
        with g.Lattice(d, beta=b, precision=prec, seed=SEED, stream_id=7 + i, flow_eps=0.02) as L:
            L.hot_start(99)
            a = L.metropolis(3)
            want_links = L.get_links()
            want_obs = L.flow(4)
        assert rel(links[i], want_links) < tol, i
        assert abs(acc[i] - a) < 1e-12 if prec == "fp64" else abs(acc[i] - a) < 0.01, i
        # the single context measures inside its flow stage 0, the ensemble in a
        # pass of its own: the same quantities to rounding, quantity by quantity
        assert_obs_close(obs[i], want_obs, tol * 10, f"lattice {i}")


def test_graph_equals_eager_and_replays_draw_fresh_numbers(g, ens):
    kw = dict(precision="fp32", seed=SEED, flow_eps=0.02)
    with ens.Ensemble(DIMS, BETAS, **kw) as A, ens.Ensemble(DIMS, BETAS, **kw) as B:
        A.hot_start(5)
        B.hot_start(5)
        acc_a, obs_a, sec = A.run(2, 3)  # captured
        acc_b = B.metropolis(2)
        obs_b = B.flow(3)
        assert sec > 0
        assert np.array_equal(acc_a, acc_b)
        for i in range(len(DIMS)):
            assert np.array_equal(obs_a[i], obs_b[i])
            assert np.array_equal(A.get_links(i), B.get_links(i))
        n0 = A.launch_count
        acc_a2, obs_a2, _ = A.run(2, 3)  # replayed: sweep counter advanced on the device
        assert A.launch_count > n0
        acc_b2 = B.metropolis(2)
        obs_b2 = B.flow(3)
        assert np.array_equal(acc_a2, acc_b2)
        for i in range(len(DIMS)):
            assert np.array_equal(obs_a2[i], obs_b2[i])
        assert not np.array_equal(obs_a2[0], obs_a[0])


def test_autotune_leaves_chains_alone(g, ens):
    with ens.Ensemble(DIMS, BETAS, precision="fp32", seed=SEED) as E, \
            ens.Ensemble(DIMS, BETAS, precision="fp32", seed=SEED) as F:
        E.hot_start(8)
        F.hot_start(8)
        E.metropolis(1)
        F.metropolis(1)
        rep = E.autotune(1)
        assert rep["flow"][0] > 0 and rep["metropolis"][0] > 0 and rep["observables"][0] > 0
        for i in range(len(DIMS)):
            assert np.array_equal(E.get_links(i), F.get_links(i))
        # every observable variant measures the same flowed fields
        chosen = E.tuning
        base = None
        for v in range(3):
            E.tuning = [0, 0, v]
            obs = E.flow(2)
            if base is None:
                base = obs
            else:
                for i in range(len(DIMS)):
                    assert rel(obs[i], base[i]) < 1e-5
        E.tuning = chosen
        # every variant computes the same chain
        a, b = E.metropolis(2), F.metropolis(2)
        assert np.allclose(a, b, atol=0.01)
        for i in range(len(DIMS)):
            assert rel(E.get_links(i), F.get_links(i)) < 1e-4


def test_ensemble_errors(g, ens):
    with pytest.raises(g.GlacError):
        ens.Ensemble([(4, 4, 4, 5)], [6.0])
    with pytest.raises(g.GlacError):
        ens.Ensemble([(4, 4, 4, 4)], [6.0], precision=9)
    with ens.Ensemble([(4, 4, 4, 4)], [6.0]) as E:
        with pytest.raises(g.GlacError):
            E.metropolis(1)  # no field yet
        E.hot_start(1)
        with pytest.raises(g.GlacError):
            E.get_links(3)
        with pytest.raises(g.GlacError):
            E.tuning = [0, 0, 5]


@pytest.mark.parametrize("prec,tol", [("fp64", 1e-12), ("fp32", 1e-5)])
def test_ensemble_measurement_inside_stage0_matches_standalone(g, ens, prec, tol):
    # every flow measurement but the last comes from the next step's stage 0;
    # with fused_measure = 0 each is a pass of its own: the same to rounding
    kw = dict(precision=prec, seed=SEED, flow_eps=0.02)
    with ens.Ensemble(DIMS, BETAS, **kw) as A, ens.Ensemble(DIMS, BETAS, **kw) as B:
        B.set_option("fused_measure", 0)
        for E in (A, B):
            E.hot_start(8)
            E.metropolis(20)
        oa, ob = A.flow(4), B.flow(4)
        for i in range(len(DIMS)):
            assert_obs_close(oa[i], ob[i], 4 * tol, f"lattice {i}")


def test_persistent_launch_equals_graph(g, ens):
    # the whole schedule in one cooperative launch with grid barriers between
    # the phases gives what the CUDA graph of per-phase launches gives
    kw = dict(precision="fp32", seed=SEED, flow_eps=0.02)
    with ens.Ensemble(DIMS, BETAS, **kw) as A, ens.Ensemble(DIMS, BETAS, **kw) as B:
        A.hot_start(6)
        B.hot_start(6)
        acc_a, obs_a, _ = A.run(3, 4)
        acc_b, obs_b, sec = B.run_persistent(3, 4)
        assert sec > 0
        assert np.max(np.abs(acc_a - acc_b)) < 1e-3
        for i in range(len(DIMS)):
            assert_obs_close(obs_b[i], obs_a[i], 1e-5, f"lattice {i}")
            assert rel(B.get_links(i), A.get_links(i)) < 1e-5
        # both continue the same random stream
        acc_a, obs_a, _ = A.run(2, 1)
        acc_b, obs_b, _ = B.run_persistent(2, 1)
        assert np.max(np.abs(acc_a - acc_b)) < 1e-3


def test_persistent_barrier_wait_runs_out_and_recovers(g, ens):
    # one block held back (test mode): the others' bounded barrier waits run out,
    # the call reports a timeout, and the ensemble works again afterwards
    kw = dict(precision="fp32", seed=SEED, flow_eps=0.02)
    with ens.Ensemble(DIMS, BETAS, **kw) as A, ens.Ensemble(DIMS, BETAS, **kw) as B:
        A.hot_start(6)
        A.set_option("persistent_wait_ms", 100)
        A.set_option("persistent_test_stall", 1)
        with pytest.raises(g.GlacError) as e:
            A.run_persistent(1, 1)
        assert e.value.status == g.GLAC_ERR_TIMEOUT
        A.set_option("persistent_test_stall", 0)
        A.set_option("persistent_wait_ms", 5000)
        A.hot_start(6)
        B.hot_start(6)
        _, obs_a, _ = A.run_persistent(2, 2)
        _, obs_b, _ = B.run(2, 2)
        for i in range(len(DIMS)):
            assert_obs_close(obs_a[i], obs_b[i], 1e-5, f"lattice {i}")
