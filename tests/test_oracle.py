"""The oracle (C restatement) pinned against the reference's own known answers,
the committed reference outputs, and -- where it is built -- the reference itself."""
import numpy as np
import pytest

from conftest import rel_err

N4 = (4, 4, 4, 4)


def test_known_answer_matrix_algebra(oracle, fixtures):
    # GLAC/tests/unit_tests/su3operations.cpp:38-70 with testcore.cpp fixtures
    assert np.array_equal(oracle.su3_mul(fixtures["U1"], fixtures["U2"]), fixtures["UMul"])
    assert np.array_equal(oracle.su3_dagger(fixtures["U1"]), fixtures["UCT"])
    # traceRealMultiplication(U1, UTrace) = -21 (testsuite.cpp:1080)
    assert oracle.retr_mul(fixtures["U1"], fixtures["UTrace"]) == fixtures["tracedMatrix"]


def test_known_answer_hermitian_projection(fixtures):
    # makeHermitian multiplies by -i (su3.h:354-365); U1AntiHermitian -> U1Hermitian
    ah = fixtures["U1AntiHermitian"]
    h = np.empty(18)
    h[0::2], h[1::2] = ah[1::2], -ah[0::2]
    assert np.array_equal(h, fixtures["U1Hermitian"])


def test_known_answer_rst(oracle, fixtures):
    # randommatrixtests.cpp:10-46: RST product and its inverse (= dagger)
    X = oracle.rst_multiply(fixtures["s_r"], fixtures["s_s"], fixtures["s_t"], False)
    assert np.array_equal(X, fixtures["U_RST"])
    Xi = oracle.rst_multiply(fixtures["s_r"], fixtures["s_s"], fixtures["s_t"], True)
    assert np.array_equal(Xi, oracle.su3_dagger(fixtures["U_RST"]))


def test_philox_known_answers(oracle):
    # Random123 known-answer vectors for philox4x32-10
    assert [hex(x) for x in oracle.philox([0, 0, 0, 0], [0, 0])] == \
        ["0x6627e8d5", "0xe169c58d", "0xbc57ac4c", "0x9b00dbd8"]
    assert [hex(x) for x in oracle.philox([0xFFFFFFFF] * 4, [0xFFFFFFFF] * 2)] == \
        ["0x408f276d", "0x41c83b0e", "0xa20bc7c6", "0x6d5451fd"]
    assert [hex(x) for x in oracle.philox([0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344],
                                          [0xA4093822, 0x299F31D0])] == \
        ["0xd16cfe09", "0x94fdcceb", "0x5001e420", "0x24126ea1"]


def test_delta_s_cold_lattice(oracle):
    # actiontests.cpp:67-114: cold lattice, U' = 2*1 -> dS = -36 for every link
    N = (4, 4, 4, 8)
    V = int(np.prod(N))
    links = np.zeros((4, V, 18))
    links[:, :, [0, 8, 16]] = 1.0
    A = oracle.staples(N, links)
    Up = np.zeros(18)
    Up[[0, 8, 16]] = 2.0
    for mu in range(4):
        for s in (0, 17, V - 1):
            assert abs(oracle.delta_s(links[mu, s], Up, A[mu, s], 6.0) + 36.0) <= 1e-15


def test_oracle_vs_golden_reference_outputs(oracle, golden):
    L = golden["links"]
    K = golden["staples"].shape[1]
    assert rel_err(oracle.staples(N4, L)[:, :K], golden["staples"]) < 1e-13
    assert rel_err(oracle.force(N4, L)[:, :K], golden["force"]) < 1e-13
    for k, name in enumerate(["exp_morningstar", "exp_luscher", "exp_taylor2", "exp_taylor4"]):
        assert rel_err(oracle.exp(golden["exp_in"], k), golden[name]) < 1e-13, name
    assert rel_err(oracle.flow(N4, L, 0.01, 3), golden["flow3"]) < 1e-13
    assert rel_err(oracle.observables(N4, L), golden["observables"]) < 1e-12
    assert rel_err(oracle.observables(N4, golden["flow3"]), golden["observables_flow3"]) < 1e-12
    assert abs(oracle.plaquette(N4, L) - golden["plaquette"][0]) < 1e-14


def test_oracle_accept_decisions_match_recorded_sweep(oracle, golden):
    U, acc = oracle.accept_fed(golden["mc_U_before"], golden["mc_staples"], golden["mc_X"], golden["mc_r"], 6.0)
    assert np.array_equal(acc, golden["mc_accept"])


def test_oracle_vs_live_reference(oracle, reference):
    reference.configure(4, 8, beta=6.0, su3eps=0.24, flow_eps=0.01, nupdates=10, nflows=2)
    N = (4, 4, 4, 8)
    L = oracle.haar_field(N, 777)
    assert rel_err(oracle.staples(N, L), reference.staples(L)) < 1e-13
    assert rel_err(oracle.force(N, L), reference.force(L)) < 1e-13
    assert rel_err(oracle.flow(N, L, 0.01, 2), reference.flow(L, 2)) < 1e-13
    assert rel_err(oracle.observables(N, L), reference.observables(L)) < 1e-12
    # the plain MasterSampler (mastersampler.cpp:161-287) agrees with the topct variant
    assert rel_err(reference.observables_nt(L), reference.observables(L)[:3]) < 1e-13


def test_reference_trace_replays_system_update(oracle, reference):
    reference.configure(4, 4, beta=6.0, su3eps=0.24, nupdates=10, metropolis_seed=3.0, matrix_seed=5.0)
    L = oracle.haar_field(N4, 99)
    tr = reference.metropolis_trace(L)
    after, _ = reference.metropolis(L, 1)
    assert np.max(np.abs(tr["links"] - after)) < 1e-14
    U, acc = oracle.accept_fed(tr["U_before"], tr["staples"], tr["X"], tr["r"], 6.0)
    assert np.array_equal(acc, tr["accept"])


def test_oracle_gauge_invariance(oracle):
    # latticeoperations.cpp:750-813: plaquette unchanged under U_mu(n) -> W(n) U_mu(n) W(n+mu)^+
    N = (4, 4, 4, 4)
    V = int(np.prod(N))
    L = oracle.haar_field(N, 5)
    W = oracle.haar_field(N, 6)[0]
    Lg = gauge_transform(L, W, N)
    o1, o2 = oracle.observables(N, L), oracle.observables(N, Lg)
    assert rel_err(o2, o1) < 1e-12


def to_c(m):
    m = np.asarray(m).reshape(m.shape[:-1] + (3, 3, 2))
    return m[..., 0] + 1j * m[..., 1]


def from_c(c):
    out = np.empty(c.shape[:-2] + (18,))
    out[..., 0::2] = c.real.reshape(c.shape[:-2] + (9,))
    out[..., 1::2] = c.imag.reshape(c.shape[:-2] + (9,))
    return out


def gauge_transform(L, W, N):
    V = int(np.prod(N))
    Lc, Wc = to_c(L), to_c(W)
    idx = np.arange(V).reshape(N[::-1])  # [t, z, y, x]
    out = np.empty_like(Lc)
    for mu in range(4):
        ax = 3 - mu
        nxt = np.roll(idx, -1, axis=ax).reshape(-1)
        out[mu] = Wc @ Lc[mu] @ np.conj(np.transpose(Wc[nxt], (0, 2, 1)))
    return from_c(out)


def reflect_x(L, N):
    """The field reflected in x (x -> -x mod Nx): U'_mu(n) = U_mu(R n) for mu != 0
    and U'_0(n) = U_0(R n - e_0)^+, the link from R n to R n - e_0 walked
    backwards.  A reflection reverses the orientation: the plaquette and E stay,
    Q and every q(t) change sign."""
    Nx = N[0]
    Lc = to_c(L).reshape((4,) + tuple(N[::-1]) + (3, 3))  # [mu, t, z, y, x, 3, 3]
    out = Lc[:, :, :, :, (-np.arange(Nx)) % Nx].copy()
    back = Lc[0][:, :, :, (-np.arange(Nx) - 1) % Nx]
    out[0] = np.conj(np.swapaxes(back, -1, -2))
    return from_c(out.reshape(4, -1, 3, 3))


def flip_charge(obs):
    """[plaq, topc, energy, topct[Nt]] with the charge and its slices negated."""
    o = np.array(obs, np.float64, copy=True)
    o[..., 1] *= -1
    o[..., 3:] *= -1
    return o


def test_oracle_reflection_flips_the_charge(oracle):
    # the parity symmetry Q -> -Q, and the flow commutes with the reflection
    N = (4, 4, 4, 8)
    L = oracle.haar_field(N, 31)
    R = reflect_x(L, N)
    assert rel_err(reflect_x(R, N), L) == 0.0
    o, r = oracle.observables(N, L), oracle.observables(N, R)
    assert abs(o[1]) > 1e-3
    assert np.max(np.abs(r - flip_charge(o))) < 1e-12 * np.max(np.abs(o))
    F = oracle.flow(N, L, 0.01, 3)
    assert rel_err(oracle.flow(N, R, 0.01, 3), reflect_x(F, N)) < 1e-13


def test_haar_field_is_special_unitary(oracle):
    L = oracle.haar_field((4, 4, 4, 4), 1234)
    M = to_c(L.reshape(-1, 18))
    eye = np.eye(3)
    assert np.max(np.abs(M @ np.conj(np.transpose(M, (0, 2, 1))) - eye)) < 1e-13
    assert np.max(np.abs(np.linalg.det(M) - 1.0)) < 1e-13
    # Haar: <|Tr U|^2> = 1 over SU(3)
    assert abs(np.mean(np.abs(np.trace(M, axis1=1, axis2=2)) ** 2) - 1.0) < 0.1


def test_reunitarize_projects_and_is_idempotent(oracle):
    L = oracle.haar_field((4, 4, 4, 4), 42).reshape(-1, 18)
    noisy = L + 1e-6 * np.random.default_rng(0).standard_normal(L.shape)
    R = oracle.reunitarize(noisy)
    M = to_c(R)
    assert np.max(np.abs(M @ np.conj(np.transpose(M, (0, 2, 1))) - np.eye(3))) < 1e-14
    assert np.max(np.abs(np.linalg.det(M) - 1.0)) < 1e-14
    assert np.max(np.abs(oracle.reunitarize(R) - R)) < 1e-15
    assert np.max(np.abs(R - L)) < 1e-5
