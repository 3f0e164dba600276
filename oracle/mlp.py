"""NumPy restatement of the learned proposal spread: staple features, the
network's forward pass, the expected-squared-jump loss, its gradient and Adam.

TEST INFRASTRUCTURE ONLY: the checker of the GPU kernels in
glac_b200/csrc/learned.cuh and learned.cu.  Never on the product path.

The component has no counterpart in the reference (whose proposals all use the
run-config's SU3Eps, GLAC/math/matrices/su3matrixgenerator.cpp:16-35); its
parity is "unpinned" by the reference and rests on this restatement plus the
physics checks in the tests (ensemble plaquette, symmetric proposal).

With ``emulate=True`` the BF16 roundings of the tensor-core kernels are applied
at the same points (inputs, weights, first-layer bias, activations, and the
deltas that enter the backward products); sums are FP64.  With
``emulate=False`` everything is FP64, for finite-difference checks.
"""
from __future__ import annotations

import numpy as np

W1, B1, W2, B2, W3, B3, NPARAMS = 0, 256, 288, 1312, 1344, 1376, 1377
LEAK = 0.0625


def bf16(x):
    """Round to bfloat16 (nearest, ties to even) and return as float64."""
    x = np.ascontiguousarray(x, np.float32)
    b = x.view(np.uint32).astype(np.uint64)
    b = (b + 0x7FFF + ((b >> 16) & 1)) & 0xFFFF0000
    return b.astype(np.uint32).view(np.float32).astype(np.float64)


def unpack(P):
    P = np.asarray(P, np.float64)
    return (P[W1:B1].reshape(8, 32), P[B1:W2], P[W2:B2].reshape(32, 32), P[B2:W3], P[W3:B3], P[B3])


def as_complex(m18):
    m = np.asarray(m18, np.float64).reshape(-1, 18)
    return (m[:, 0::2] + 1j * m[:, 1::2]).reshape(-1, 3, 3)


def features(staples18, beta):
    """The eight gauge-invariant features of each staple A (rows of 18 reals)."""
    A = as_complex(staples18)
    W = A @ np.conj(np.transpose(A, (0, 2, 1)))
    t1 = np.real(np.trace(W, axis1=1, axis2=2))
    t2 = np.sum(np.abs(W) ** 2, axis=(1, 2))
    t3 = np.real(np.trace(W @ W @ W, axis1=1, axis2=2))
    det = np.linalg.det(A)
    s2 = np.maximum(t1 / 3.0, 1e-30)
    s = np.sqrt(s2)
    k = beta * s / 3.0
    f = np.empty((A.shape[0], 8))
    f[:, 0] = np.log(k)
    f[:, 1] = t2 / (3 * s2 * s2) - 1
    f[:, 2] = t3 / (3 * s2 ** 3) - 1
    f[:, 3] = det.real / (s2 * s)
    f[:, 4] = det.imag / (s2 * s)
    f[:, 5] = np.abs(det) / (s2 * s)
    f[:, 6] = 1.0 / k
    f[:, 7] = beta / 6.0 - 1.0
    return f


def _act(x):
    return np.where(x > 0, x, LEAK * x)


def _slope(x):
    return np.where(x > 0, 1.0, LEAK)


def forward(P, X, emulate=True):
    """z for each feature row; also the intermediate values the backward pass needs."""
    w1, b1, w2, b2, w3, b3 = unpack(P)
    r = bf16 if emulate else (lambda v: np.asarray(v, np.float64))
    Xb = r(X)
    pre1 = Xb @ r(w1) + r(b1)
    h1 = r(_act(pre1))
    pre2 = h1 @ r(w2) + b2
    h2 = r(_act(pre2))
    z = h2 @ r(w3) + b3
    return z, dict(Xb=Xb, pre1=pre1, h1=h1, pre2=pre2, h2=h2, w2=r(w2), w3=r(w3))


def spread(P, X, eps_min, eps_max, emulate=True):
    z, _ = forward(P, X, emulate)
    return eps_min + (eps_max - eps_min) / (1.0 + np.exp(-z))


def interp(J, grid, eps):
    """J_i(eps_i) linear between grid points, and its slope."""
    K = grid.size
    k = np.clip(np.searchsorted(grid, eps, side="right") - 1, 0, K - 2)
    rows = np.arange(J.shape[0])
    slope = (J[rows, k + 1] - J[rows, k]) / (grid[k + 1] - grid[k])
    return J[rows, k] + slope * (eps - grid[k]), slope


def loss_grad(P, X, J, grid, emulate=True):
    """L = -(1/n) sum_i J_i(eps(f_i)) and dL/dP (flat, NPARAMS)."""
    grid = np.asarray(grid, np.float64)
    J = np.asarray(J, np.float64)
    n = X.shape[0]
    e0, e1 = grid[0], grid[-1]
    span = e1 - e0
    z, c = forward(P, X, emulate)
    sg = 1.0 / (1.0 + np.exp(-z))
    eps = e0 + span * sg
    Jv, slope = interp(J, grid, eps)
    loss = -Jv.mean()
    d3 = -(1.0 / n) * slope * span * sg * (1.0 - sg)
    r = bf16 if emulate else (lambda v: v)
    g = np.zeros(NPARAMS)
    g[W3:B3] = c["h2"].T @ d3
    g[B3] = d3.sum()
    d2 = d3[:, None] * c["w3"][None, :] * _slope(c["pre2"])
    g[B2:W3] = d2.sum(axis=0)
    d2b = r(d2)
    g[W2:B2] = (c["h1"].T @ d2b).ravel()
    d1 = (d2b @ c["w2"].T) * _slope(c["pre1"])
    g[B1:W2] = d1.sum(axis=0)
    g[W1:B1] = (c["Xb"].T @ r(d1)).ravel()
    return loss, g


def adam(P, m, v, grad, step, lr):
    """One Adam step (Kingma & Ba, arXiv:1412.6980, Algorithm 1), in place."""
    m[:] = 0.9 * m + 0.1 * grad
    v[:] = 0.999 * v + 0.001 * grad * grad
    c1, c2 = 1 - 0.9 ** step, 1 - 0.999 ** step
    P[:] = P - lr * (m / c1) / (np.sqrt(v / c2) + 1e-8)
    return P
