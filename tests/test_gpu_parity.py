"""Parity of the CUDA path (through the C ABI) against the oracle and the
reference.  Tolerances: FP64 <= 1e-12 relative, FP32 <= 1e-5 relative (the
bars of the hot-path specification); accept decisions bit-identical.

Observable vectors are compared one quantity at a time (conftest.obs_errors):
the plaquette, Q and the energy each against its own value, q(t) against the
largest |q(t)| of its row.  Matrices (links, staples, forces, exponentials),
whose entries are all of order one, are compared by the largest entry error
against the largest entry (conftest.rel_err)."""
import os

import numpy as np
import pytest

from conftest import GOLDEN, assert_obs_close, rel_err
from test_oracle import gauge_transform, to_c

pytestmark = pytest.mark.gpu

TOL = {"fp64": 1e-12, "fp32": 1e-5}
N4 = (4, 4, 4, 4)


@pytest.fixture(scope="module")
def g():
    import glac_b200
    return glac_b200


def lattice(g, N, precision, **kw):
    return g.Lattice(N, precision=precision, **kw)


def test_known_answers_on_device(g, fixtures):
    # dS(U=0, U'=U1, A=UTrace) = -(beta/3) ReTr(U1 UTrace) = -(beta/3)(-21)
    z = np.zeros(18)
    for prec in ("fp64", "fp32"):
        ds = g.delta_s_batch(z, fixtures["U1"], fixtures["UTrace"], 3.0, prec)
        assert ds[0] == 21.0


def test_delta_s_cold_lattice(g):
    # actiontests.cpp:67-114 through the device staple and dS
    for prec in ("fp64", "fp32"):
        with lattice(g, (4, 4, 4, 8), prec) as L:
            L.cold_start()
            A = L.staples().reshape(-1, 18)
            U = L.get_links().reshape(-1, 18)
            Up = np.zeros_like(U)
            Up[:, [0, 8, 16]] = 2.0
            ds = g.delta_s_batch(U, Up, A, 6.0, prec)
            assert np.max(np.abs(ds + 36.0)) <= 1e-15 if prec == "fp64" else 1e-5


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_staples_and_force_vs_reference(g, golden, oracle, prec):
    with lattice(g, N4, prec) as L:
        L.set_links(golden["links"])
        K = golden["staples"].shape[1]
        assert rel_err(L.staples()[:, :K], golden["staples"]) < TOL[prec]
        assert rel_err(L.force()[:, :K], golden["force"]) < TOL[prec]
        assert rel_err(L.staples(), oracle.staples(N4, golden["links"])) < TOL[prec]


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
@pytest.mark.parametrize("kind", ["morningstar", "luscher", "taylor2", "taylor4"])
def test_exponentials_vs_reference(g, golden, prec, kind):
    out = g.exp_batch(golden["exp_in"], prec, kind)
    assert rel_err(out, golden["exp_" + kind]) < TOL[prec]


def expm_reference(Z):
    """exp by scaling and squaring of a degree-24 Taylor polynomial in long double."""
    Zl = np.asarray(Z, dtype=np.clongdouble)
    nrm = np.max(np.abs(Zl).sum(axis=2), axis=1)
    k = np.maximum(0, np.ceil(np.log2(np.maximum(nrm.astype(np.float64), 1e-300) / 0.25))).astype(int)
    out = np.empty(Zl.shape, dtype=np.complex128)
    for i in range(Zl.shape[0]):
        A = Zl[i] / (2.0 ** k[i])
        S = np.eye(3, dtype=np.clongdouble)
        P = np.eye(3, dtype=np.clongdouble)
        for j in range(1, 25):
            P = P @ A / j
            S = S + P
        for _ in range(k[i]):
            S = S @ S
        out[i] = S.astype(np.complex128)
    m = np.empty((Z.shape[0], 18))
    m[:, 0::2], m[:, 1::2] = out.real.reshape(-1, 9), out.imag.reshape(-1, 9)
    return m


def test_morningstar_extreme_inputs(g, oracle):
    rng = np.random.default_rng(1)
    for scale in (1e-6, 1e-3, 1.0, 3.0):
        H = rng.standard_normal((256, 3, 3)) + 1j * rng.standard_normal((256, 3, 3))
        Z = (H - np.conj(np.transpose(H, (0, 2, 1)))) * 0.5
        Z -= np.eye(3) * (np.trace(Z, axis1=1, axis2=2)[:, None, None] / 3)
        Z *= scale
        m = np.empty((256, 18))
        m[:, 0::2], m[:, 1::2] = Z.real.reshape(256, 9), Z.imag.reshape(256, 9)
        want = expm_reference(Z)
        for prec in ("fp64", "fp32"):
            assert rel_err(g.exp_batch(m, prec), want) < (1e-13 if prec == "fp64" else 2e-6), (scale, prec)
    # Z = 0: identity (the reference divides 0/0 there, su3exp.cpp:30-31)
    e = g.exp_batch(np.zeros((1, 18)))
    assert np.array_equal(e[0][[0, 8, 16]], [1.0, 1.0, 1.0])


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_flow_and_observables_vs_reference(g, golden, prec):
    with lattice(g, N4, prec, flow_eps=0.01) as L:
        L.set_links(golden["links"])
        obs = L.flow(3)
        assert_obs_close(obs[0], golden["observables"], TOL[prec], "t = 0")
        assert_obs_close(obs[3], golden["observables_flow3"], TOL[prec], "after 3 steps")
        assert rel_err(L.get_links(), golden["flow3"]) < TOL[prec]


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_thermalized_field_flow_vs_reference(g, prec):
    # A field from the reference's own Metropolis chain (plaquette 0.589),
    # flowed 100 RK3 steps at eps = 0.01 to plaquette 0.993: every one of the
    # 101 measurements against the reference's, quantity by quantity, and the
    # links at the end (tests/golden/make_golden.py, fixture "flow").
    fx = np.load(os.path.join(GOLDEN, "ref_4x4x4x8_b6_flow.npz"))
    want = fx["observables"]
    nsteps = want.shape[0] - 1
    with lattice(g, (4, 4, 4, 8), prec, flow_eps=float(fx["flow_eps"][0])) as L:
        L.set_links(fx["links"])
        obs = L.flow(nsteps)
        K = fx["links_end"].shape[1]
        assert rel_err(L.get_links()[:, :K], fx["links_end"]) < TOL[prec]
    assert want[0, 0] < 0.6 and want[-1, 0] > 0.99 and np.min(np.abs(want[:, 1])) > 0.2
    e = assert_obs_close(obs, want, TOL[prec], f"{prec}, 101 measurements")
    print(prec, "largest relative errors over the flow:", e)


def test_fp32_lanes_across_the_t_cut(g, oracle):
    # FP32 carries t and t + Nt/2 in the two lanes of one thread; a field that
    # differs strongly between the halves checks the lane swap at the cut
    N = (4, 4, 4, 8)
    links = oracle.haar_field(N, 314)
    V = int(np.prod(N))
    half = V // 2
    rng = np.random.default_rng(7)
    H = rng.standard_normal((4 * half, 3, 3)) + 1j * rng.standard_normal((4 * half, 3, 3))
    Z = 0.05 * (H - np.conj(np.transpose(H, (0, 2, 1))))
    Z -= np.eye(3) * (np.trace(Z, axis1=1, axis2=2)[:, None, None] / 3)
    m = np.empty((4 * half, 18))
    m[:, 0::2], m[:, 1::2] = Z.real.reshape(-1, 9), Z.imag.reshape(-1, 9)
    links[:, half:] = oracle.exp(m, 0).reshape(4, half, 18)  # upper half in t: near unity
    want_obs = oracle.observables(N, links)
    want_flow = oracle.flow(N, links, 0.02, 2)
    with lattice(g, N, "fp32", flow_eps=0.02) as L:
        L.set_links(links)
        assert_obs_close(L.measure(), want_obs, 1e-5, "fp32 lanes")
        assert rel_err(L.staples(), oracle.staples(N, links)) < 1e-5
        L.flow(2, measure=False)
        assert rel_err(L.get_links(), want_flow) < 1e-5


def test_autotune_restores_state_and_keeps_results(g, oracle):
    N = (8, 8, 8, 8)
    start = oracle.haar_field(N, 21)
    for prec in ("fp64", "fp32"):
        with lattice(g, N, prec, seed=9) as A, lattice(g, N, prec, seed=9) as B:
            A.set_links(start)
            B.set_links(start)
            rep = A.autotune(2)
            assert np.array_equal(A.get_links(), start if prec == "fp64" else B.get_links())
            for fam in ("flow", "metropolis", "observables"):
                assert rep[fam][0] > 0
            # every variant computes the same thing; the chain continues identically
            acc_a, acc_b = A.metropolis(2), B.metropolis(2)
            assert acc_a == acc_b
            assert np.array_equal(A.get_links(), B.get_links())
            for v in range(4):
                try:
                    A.tuning = [v, v, v]
                except g.GlacError:
                    continue
                A.set_links(start)
                B.set_links(start)
                assert_obs_close(A.flow(2), B.flow(2), TOL[prec], f"variant {v}")


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_flow_variants_agree(g, oracle, prec):
    # (z, t) pairs of two 128-site chunks and Nz, Nt multiples of 4, so the
    # tiled chunk order really permutes the blocks; every flow variant (register
    # caps, site-block shapes) must give the same field and observables
    N = (32, 16, 8, 8)
    start = oracle.haar_field(N, 31)
    ref = None
    for v in range(4):
        with lattice(g, N, prec) as L:
            try:
                L.tuning = [v, 0, 0]
            except g.GlacError:
                continue
            L.set_links(start)
            obs = L.flow(3)
            links = L.get_links()
        if ref is None:
            ref = (obs, links)
            assert rel_err(links, oracle.flow(N, start, 0.01, 3)) < TOL[prec]
        else:
            assert rel_err(links, ref[1]) < TOL[prec]
            assert_obs_close(obs, ref[0], TOL[prec], f"variant {v}")


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
@pytest.mark.parametrize("N", [(6, 4, 6, 8), (8, 8, 8, 16)])
def test_measurement_inside_flow_stage0(g, oracle, prec, N):
    # glac_flow measures the field before each step inside that step's stage 0
    # (the clover from the staple pieces, combined per site afterwards); with
    # fused_measure = 0 every field is measured by the stand-alone pass.  On the
    # oracle's own flowed fields (set before each one-step flow, so both
    # measure exactly the same field): fused, stand-alone and oracle agree to
    # the bar, and both modes flow the field the same.
    with lattice(g, N, "fp64", beta=6.0, seed=77) as C:
        C.set_links(oracle.haar_field(N, 77))
        C.metropolis(10)
        cur = C.get_links()
    modes = (1, 2, 3, 4) if prec == "fp32" else (1, 2)  # kernel forms of the fused stage 0
    with lattice(g, N, prec, flow_eps=0.02) as B:
        B.set_option("fused_measure", 0)
        for k in range(4):
            B.set_links(cur)
            ob = B.flow(1)
            want = oracle.observables(N, cur)
            assert_obs_close(ob[0], want, TOL[prec], f"stand-alone, field {k}")
            nxt = oracle.flow(N, cur, 0.02, 1)
            assert rel_err(B.get_links(), nxt) < TOL[prec]
            for mode in modes:
                with lattice(g, N, prec, flow_eps=0.02) as A:
                    A.set_option("fused_measure", mode)
                    A.set_links(cur)
                    oa = A.flow(1)
                    assert_obs_close(oa[0], want, TOL[prec], f"fused {mode}, field {k}")
                    assert_obs_close(oa, ob, TOL[prec], f"fused {mode} vs stand-alone, field {k}")
                    assert rel_err(A.get_links(), nxt) < TOL[prec]
            cur = nxt


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_flow_vs_live_reference_larger(g, oracle, reference, prec):
    # Step by step at eps = 0.02 from a field 20 FP64 sweeps away from a Haar
    # start (plaquette ~0.5; the plaquette of the Haar field itself is ~0, where a
    # relative error says nothing): after step k the field and the observables
    # within k times the one-step bar, since each step adds its own rounding
    # differences (FP64 on B200: ~3e-13 per step in the links).
    N = (8, 8, 8, 8)
    reference.configure(8, 8, flow_eps=0.02, nflows=4)
    with lattice(g, N, "fp64", beta=6.0, seed=4242) as C:
        C.set_links(oracle.haar_field(N, 4242))
        C.metropolis(20)
        links = C.get_links()
    with lattice(g, N, prec, flow_eps=0.02) as L:
        L.set_links(links)
        cur = links
        assert_obs_close(L.measure(), reference.observables(cur), TOL[prec], "t = 0")
        for k in range(1, 5):
            cur = reference.flow(cur, 1)
            obs = L.flow(1)
            err = rel_err(L.get_links(), cur)
            assert err < k * TOL[prec], (k, err)
            assert_obs_close(obs[1], reference.observables(cur), k * TOL[prec], f"after {k} steps")


@pytest.mark.parametrize("kind", ["luscher", "taylor2", "taylor4"])
def test_flow_alternate_exponentials(g, oracle, golden, kind):
    k = {"luscher": 1, "taylor2": 2, "taylor4": 3}[kind]
    want = oracle.flow(N4, golden["links"], 0.01, 2, k)
    with lattice(g, N4, "fp64", flow_eps=0.01, exp_func=kind) as L:
        L.set_links(golden["links"])
        L.flow(2, measure=False)
        assert rel_err(L.get_links(), want) < 1e-12


def test_accept_decisions_bit_identical(g, golden):
    U, acc = g.accept_fed(golden["mc_U_before"], golden["mc_staples"], golden["mc_X"], golden["mc_r"], 6.0, "fp64")
    assert np.array_equal(acc, golden["mc_accept"])


def test_accept_decisions_full_reference_sweep(g, oracle, reference):
    reference.configure(4, 8, beta=6.0, su3eps=0.24, nupdates=10, metropolis_seed=17.0, matrix_seed=19.0)
    tr = reference.metropolis_trace(oracle.haar_field((4, 4, 4, 8), 3))
    U, acc = g.accept_fed(tr["U_before"], tr["staples"], tr["X"], tr["r"], 6.0, "fp64")
    assert np.array_equal(acc, tr["accept"])
    last = {}
    for k, (mu, s) in enumerate(tr["order"]):
        last[(mu, s)] = k
    final = np.array([U[last[(mu, s)]] for mu in range(4) for s in range(512)]).reshape(4, 512, 18)
    assert rel_err(final, tr["links"]) < 1e-13


@pytest.mark.parametrize("flips", [True, False])
def test_checkerboard_sweep_matches_oracle(g, oracle, flips):
    N = (4, 4, 4, 8)
    start = oracle.haar_field(N, 7)
    with lattice(g, N, "fp64", beta=6.0, su3_eps=0.24, n_updates=10, seed=0x1234_5678_9ABC, stream_id=3) as L:
        L.set_links(start)
        L.set_option("su2_sign_flips", int(flips))
        ref = start
        total = 0
        for sweep in range(3):
            ref, a = oracle.metropolis_sweep(N, ref, 6.0, 0.24, 10, 0x1234_5678_9ABC, 3, sweep, flips)
            total += a
        acc = L.metropolis(3)
        assert abs(acc * 4 * 10 * L.V * 3 - total) < 0.5
        assert rel_err(L.get_links(), ref) < 1e-12


def test_hot_start_matches_oracle(g, oracle):
    N = (4, 4, 4, 8)
    for prec in ("fp64", "fp32"):
        with lattice(g, N, prec) as L:
            L.hot_start(99)
            got = L.get_links()
            assert rel_err(got, oracle.haar_field(N, 99)) < (1e-13 if prec == "fp64" else 1e-6)
            assert L.unitarity_violation() < (1e-13 if prec == "fp64" else 1e-6)


def test_set_get_roundtrip(g, oracle):
    N = (4, 6, 4, 8)
    links = oracle.haar_field(N, 5)
    with lattice(g, N, "fp64") as L:
        L.set_links(links)
        assert np.array_equal(L.get_links(), links)
    with lattice(g, N, "fp32") as L:
        L.set_links(links)
        assert rel_err(L.get_links(), links) < 1e-7


def test_cold_lattice_flow_stays_identity(g):
    # the reference yields NaN here (0/0 in su3exp.cpp:30-31); the device path returns 1
    with lattice(g, (4, 4, 4, 4), "fp64") as L:
        L.cold_start()
        obs = L.flow(2)
        assert np.all(np.isfinite(obs))
        assert obs[-1][0] == 1.0


def test_state_and_argument_errors(g):
    with lattice(g, (4, 4, 4, 4), "fp64") as L:
        with pytest.raises(g.GlacError) as e:
            L.flow(1)
        assert e.value.status == g.GLAC_ERR_STATE
        L.cold_start()
        with pytest.raises(g.GlacError) as e:
            L.metropolis(-1)
        assert e.value.status == g.GLAC_ERR_ARG


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_gauge_invariance_on_device(g, oracle, prec):
    N = (8, 8, 8, 16)
    links = oracle.haar_field(N, 10)
    W = oracle.haar_field(N, 11)[0]
    gt = gauge_transform(links, W, N)
    with lattice(g, N, prec) as L:
        L.set_links(links)
        a = L.measure()
        L.set_links(gt)
        b = L.measure()
    assert_obs_close(b[:3], a[:3], 1e-12 if prec == "fp64" else 1e-5, "gauge transformed", slices=())


def test_uneven_extents_and_obs_plan(g, oracle):
    # Nx != Ny != Nz and half-slices that are not whole warps (6*4*6/2 = 72 sites)
    N = (6, 4, 6, 4)
    links = oracle.haar_field(N, 12)
    with lattice(g, N, "fp64") as L:
        L.set_links(links)
        assert_obs_close(L.measure(), oracle.observables(N, links), 1e-12, "uneven extents")
        assert rel_err(L.staples(), oracle.staples(N, links)) < 1e-12


@pytest.mark.parametrize("prec,tol", [("fp64", 1e-12), ("fp32", 1e-5)])
def test_charge_density_matches_reference(g, oracle, reference, prec, tol):
    # LatticeActionChargeDensity's per-site fields (the energyTopcFieldDensity sampler)
    N = (4, 4, 4, 8)
    reference.configure(4, 8, flow_eps=0.02, nflows=4)
    links = oracle.flow(N, oracle.haar_field(N, 17), 0.02, 3)
    q_ref, e_ref, obs_ref = reference.density(links)
    with lattice(g, N, prec) as L:
        L.set_links(links)
        obs, q, e = L.measure_density()
        assert_obs_close(obs, L.measure(), 1e-12, "density pass vs measurement")
    assert np.max(np.abs(q - q_ref)) < tol * np.max(np.abs(q_ref))
    assert np.max(np.abs(e - e_ref)) < tol * np.max(np.abs(e_ref))
    assert abs(q.sum() - obs[1]) < 1e-10 and abs(e.sum() / L.V - obs[2]) < 1e-9 * abs(obs[2])
    assert_obs_close(obs[:3], obs_ref, tol, "density sampler", slices=())


def test_sweep_counter_continues_the_stream(g, oracle):
    N = (4, 4, 4, 8)
    start = oracle.haar_field(N, 3)
    with lattice(g, N, "fp64", seed=11) as A, lattice(g, N, "fp64", seed=11) as B:
        A.set_links(start)
        A.metropolis(3)
        mid = A.get_links()
        A.metropolis(2)
        B.set_links(mid)
        B.sweep = 3  # as restored from a checkpoint sidecar
        B.metropolis(2)
        assert A.sweep == B.sweep == 5
        assert np.array_equal(A.get_links(), B.get_links())


@pytest.mark.parametrize("prec,tol", [("fp64", 1e-12), ("fp32", 1e-5)])
def test_weinberg_matches_reference(g, oracle, reference, prec, tol):
    N = (4, 4, 4, 8)
    reference.configure(4, 8, flow_eps=0.02, nflows=4)
    for seed in (19, 23):
        links = oracle.flow(N, oracle.haar_field(N, seed), 0.02, 3)
        want = reference.supersampler(links)
        with lattice(g, N, prec) as L:
            L.set_links(links)
            got = L.measure_weinberg()
            base = L.measure()
        assert_obs_close(got, want, tol, "weinberg", scalars=("plaq", "topc", "energy", "weinberg"),
                         slices=("topct", "weinbergt"))
        assert_obs_close(np.r_[got[:3], got[4:12]], base, 1e-12, "weinberg vs plain sampler")


def test_observables_at_the_largest_time_extent(g, oracle):
    # Nt = 1024 fills the per-slice arrays of the reduction; larger Nt is rejected at creation
    N = (4, 4, 4, 1024)
    links = oracle.haar_field(N, 41)
    with lattice(g, N, "fp64") as L:
        L.set_links(links)
        got = L.measure()
        assert got.size == 3 + 1024
        assert_obs_close(got, oracle.observables(N, links), 1e-12, "Nt = 1024")
        _, q, _ = L.measure_density()
        assert abs(q.sum() - got[1]) < 1e-9
    with pytest.raises(g.GlacError):
        lattice(g, (4, 4, 4, 1026), "fp64")
