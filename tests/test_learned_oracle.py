"""The NumPy restatement of the learned proposal spread (oracle/mlp.py), on CPU:
gauge invariance of the features, their values on a cold lattice, the analytic
gradient against finite differences, and the BF16 emulation against FP64."""
import numpy as np
import pytest

from oracle import mlp


def _random_su3(rng, n):
    Z = rng.standard_normal((n, 3, 3)) + 1j * rng.standard_normal((n, 3, 3))
    Q, R = np.linalg.qr(Z)
    d = np.diagonal(R, axis1=1, axis2=2)
    Q = Q * (d / np.abs(d))[:, None, :]
    det = np.linalg.det(Q)
    return Q / (det ** (1.0 / 3.0))[:, None, None]


def _to18(M):
    M = M.reshape(-1, 3, 3)
    out = np.empty((M.shape[0], 18))
    out[:, 0::2], out[:, 1::2] = M.real.reshape(-1, 9), M.imag.reshape(-1, 9)
    return out


def test_features_cold_lattice():
    # cold lattice: A = 6 * 1 -> s = 6, k = 2 beta, det A = 216
    f = mlp.features(_to18(6.0 * np.eye(3)), 6.0)[0]
    assert np.allclose(f, [np.log(12.0), 0, 0, 1, 0, 1, 1 / 12.0, 0], atol=1e-14)


def test_features_gauge_invariant_and_link_independent(oracle):
    N = (4, 4, 4, 4)
    V = 256
    links = oracle.haar_field(N, 5)
    A = oracle.staples(N, links).reshape(4, V, 18)
    f0 = mlp.features(A.reshape(-1, 18), 6.0)
    # gauge transformation U_mu(n) -> O(n) U_mu(n) O(n+mu)^+
    rng = np.random.default_rng(2)
    O = _random_su3(rng, V)
    U = mlp.as_complex(links.reshape(-1, 18)).reshape(4, V, 3, 3)
    Ut = np.empty_like(U)
    for mu in range(4):
        for s in range(V):
            c = np.unravel_index(s, (N[3], N[2], N[1], N[0]))[::-1]
            c2 = list(c)
            c2[mu] = (c2[mu] + 1) % N[mu]
            s2 = c2[0] + N[0] * (c2[1] + N[1] * (c2[2] + N[2] * c2[3]))
            Ut[mu, s] = O[s] @ U[mu, s] @ np.conj(O[s2]).T
    At = oracle.staples(N, _to18(Ut).reshape(4, V, 18)).reshape(-1, 18)
    f1 = mlp.features(At, 6.0)
    assert np.max(np.abs(f1 - f0)) < 1e-10
    # the staple of U_mu(n) does not involve U_mu(n): changing the link leaves its features
    links2 = links.copy().reshape(4, V, 18)
    links2[1, 17] = _to18(_random_su3(rng, 1))[0]
    A2 = oracle.staples(N, links2).reshape(4, V, 18)
    assert np.array_equal(A2[1, 17], A[1, 17])


def _problem(seed, n=200, K=12):
    rng = np.random.default_rng(seed)
    P = np.zeros(mlp.NPARAMS)
    P[mlp.W1:mlp.B1] = rng.standard_normal(256) * 0.5
    P[mlp.B1:mlp.W2] = rng.standard_normal(32) * 0.1
    P[mlp.W2:mlp.B2] = rng.standard_normal(1024) * 0.25
    P[mlp.B2:mlp.W3] = rng.standard_normal(32) * 0.1
    P[mlp.W3:mlp.B3] = rng.standard_normal(32) * 0.3
    P[mlp.B3] = -0.5
    X = rng.standard_normal((n, 8))
    grid = np.geomspace(0.03, 0.9, K)
    J = np.abs(rng.standard_normal((n, K))) * np.sin(np.pi * grid / 1.0)[None, :]
    return P, X, J, grid


def test_gradient_matches_finite_differences():
    P, X, J, grid = _problem(3)
    loss, g = mlp.loss_grad(P, X, J, grid, emulate=False)
    rng = np.random.default_rng(4)
    h = 1e-6
    idx = np.concatenate([rng.choice(np.arange(mlp.B1), 6, replace=False), np.arange(mlp.B1, mlp.B1 + 3),
                          rng.choice(np.arange(mlp.W2, mlp.B2), 6, replace=False), np.arange(mlp.B2, mlp.B2 + 3),
                          np.arange(mlp.W3, mlp.W3 + 4), [mlp.B3]])
    for k in idx:
        Pp, Pm = P.copy(), P.copy()
        Pp[k] += h
        Pm[k] -= h
        fd = (mlp.loss_grad(Pp, X, J, grid, emulate=False)[0] - mlp.loss_grad(Pm, X, J, grid, emulate=False)[0]) / (2 * h)
        assert abs(fd - g[k]) < 1e-6 + 1e-4 * abs(g[k]), (k, fd, g[k])


def test_bf16_emulation_close_to_fp64():
    P, X, J, grid = _problem(5)
    l0, g0 = mlp.loss_grad(P, X, J, grid, emulate=False)
    l1, g1 = mlp.loss_grad(P, X, J, grid, emulate=True)
    assert abs(l1 - l0) < 0.02 * abs(l0)
    assert np.linalg.norm(g1 - g0) < 0.15 * np.linalg.norm(g0)  # BF16 weights carry ~3 digits
    assert mlp.bf16(np.float32(1.0 + 2 ** -9)) == 1.0          # ties to even
    assert mlp.bf16(np.float32(1.0 + 3 * 2 ** -9)) == 1.0 + 2 ** -7


def test_adam_step_direction():
    P = np.array([1.0, -1.0])
    m, v = np.zeros(2), np.zeros(2)
    mlp.adam(P, m, v, np.array([0.5, -2.0]), 1, 0.1)
    assert np.allclose(P, [0.9, -0.9])  # first step moves each parameter by lr against its gradient's sign
