"""GPU tests of the learned proposal spread, through the C ABI.

* features and expected-squared-jump data of the kernels against the oracle
  (oracle/mlp.py, oracle_esj_link);
* the tensor-core forward pass and gradient against the oracle's BF16-emulating
  restatement; training on the GPU reaches a known optimum;
* exactness: a chain whose spread varies link by link with the staple still
  reproduces the reference's ensemble plaquette;
* what the network gains over the fixed spread on held-out data.
"""
import json
import os

import numpy as np
import pytest

from oracle import mlp

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.fixture(scope="module")
def g():
    import glac_b200
    return glac_b200


@pytest.fixture(scope="module")
def torch():
    import torch
    return torch


@pytest.fixture(scope="module")
def learned():
    from glac_b200 import learned
    return learned


def f32(a):
    return np.asarray(a, np.float32).astype(np.float64)


def random_params(seed, w3=0.3, b3=-0.5):
    rng = np.random.default_rng(seed)
    P = np.zeros(mlp.NPARAMS)
    P[mlp.W1:mlp.B1] = rng.standard_normal(256) * 0.5
    P[mlp.B1:mlp.W2] = rng.standard_normal(32) * 0.1
    P[mlp.W2:mlp.B2] = rng.standard_normal(1024) * 0.25
    P[mlp.B2:mlp.W3] = rng.standard_normal(32) * 0.1
    P[mlp.W3:mlp.B3] = rng.standard_normal(32) * w3
    P[mlp.B3] = b3
    return P.astype(np.float32)


def esj_rows(g, torch, L, grid, trials, stride, snapshot):
    rows = L.esj_rows(stride)
    feat = torch.empty((rows, 8), dtype=torch.float32, device="cuda")
    esj = torch.empty((rows, max(len(grid), 1)), dtype=torch.float32, device="cuda")
    ids = torch.empty(rows, dtype=torch.int32, device="cuda")
    n = L.esj_data_ptr(grid, trials, stride, snapshot, feat.data_ptr(), esj.data_ptr(), ids.data_ptr(), rows)
    assert n == rows
    return feat.cpu().numpy(), esj.cpu().numpy(), ids.cpu().numpy().view(np.uint32)


@pytest.mark.parametrize("prec,tol", [("fp64", 1e-6), ("fp32", 3e-4)])
def test_features_match_oracle(g, torch, oracle, prec, tol):
    N, V = (4, 4, 4, 8), 512
    links = oracle.haar_field(N, 11)
    with g.Lattice(N, beta=6.0, precision=prec) as L:
        L.set_links(links)
        feat, _, ids = esj_rows(g, torch, L, [], 1, 1, 0)
    assert np.array_equal(np.sort(ids), np.arange(4 * V))
    want = mlp.features(oracle.staples(N, links).reshape(-1, 18)[ids], 6.0)
    assert np.max(np.abs(feat - want) / (1 + np.abs(want))) < tol


@pytest.mark.parametrize("prec,flips", [("fp64", True), ("fp64", False), ("fp32", False)])
def test_esj_matches_oracle(g, torch, oracle, prec, flips):
    N, V, beta, seed, stream = (4, 4, 4, 8), 512, 6.0, 77, 3
    links = oracle.haar_field(N, 12)
    for sw in range(6):  # off the Haar start, so that a fair share of moves is accepted
        links, _ = oracle.metropolis_sweep(N, links, beta, 0.24, 10, 5, 0, sw)
    grid = f32(np.geomspace(0.03, 0.9, 8))
    with g.Lattice(N, beta=beta, precision=prec, seed=seed, stream_id=stream) as L:
        L.set_links(links)
        L.set_option("su2_sign_flips", int(flips))
        feat, esj, ids = esj_rows(g, torch, L, grid, 3, 4, 5)
    A = oracle.staples(N, links).reshape(-1, 18)
    U = links.reshape(-1, 18)
    want = np.array([oracle.esj_link(U[i], A[i], beta, 10, grid, 3, seed, i, 5, stream, flips) for i in ids])
    d = np.abs(esj - want)
    assert want.mean() > 0.01  # moves get accepted: the comparison is not trivial
    if prec == "fp64":  # the rows are stored as float32
        assert np.all(d <= 1.2e-7 * np.abs(want) + 1e-12)
    else:  # FP32: the same draws; an accept decision at the threshold may flip
        assert np.mean(d < 1e-4) > 0.97
        assert abs(esj.mean() - want.mean()) < 0.01 * want.mean()


@pytest.mark.parametrize("mode,n", [(0, 3000), (1, 3000), (1, 200_000)])
def test_forward_matches_oracle(g, torch, learned, mode, n):
    # mode 0: the sampler's warp routine; mode 1: tcgen05 tensor-core tiles of
    # 128 rows (3000 rows: a partial last tile; 200k rows: several tiles per CTA)
    rng = np.random.default_rng(1)
    X = rng.standard_normal((n, 8)).astype(np.float32)
    P = random_params(2)
    with learned.ProposalNet() as net:
        net.params = P
        net.set_forward_mode(mode)
        got = net.forward(torch.from_numpy(X).cuda(), 0.03, 0.9).cpu().numpy()
    want = mlp.spread(P, X, f32(0.03)[()], f32(0.9)[()], emulate=True)
    d = np.abs(got - want)
    assert np.median(d) < 1e-5 and d.max() < 5e-3
    assert got.std() > 0.05  # the spread really varies with the features


def test_tensor_core_and_warp_inference_agree(g, torch, learned):
    rng = np.random.default_rng(8)
    X = torch.from_numpy(rng.standard_normal((50_000, 8)).astype(np.float32)).cuda()
    with learned.ProposalNet() as net:
        net.params = random_params(9)
        net.set_forward_mode(0)
        a = net.forward(X, 0.03, 0.9).cpu().numpy()
        net.set_forward_mode(1)
        b = net.forward(X, 0.03, 0.9).cpu().numpy()
    # the same rounding points; the two tensor-core paths sum the FP32 products in different orders
    d = np.abs(a - b)
    assert np.median(d) < 1e-6 and d.max() < 5e-3


def test_tensor_core_wait_timeout_is_reported_and_recovers(g, torch, learned):
    # The tcgen05 kernel bounds every completion wait by the GPU's global timer.
    # With no MMA issued (test mode) its first wait runs out with nothing in
    # flight: the call returns GLAC_ERR_TIMEOUT, the device stays usable, and the
    # next normal pass on the same trainer gives the right spreads.
    rng = np.random.default_rng(4)
    X = rng.standard_normal((1000, 8)).astype(np.float32)
    P = random_params(5)
    want = mlp.spread(P, X, f32(0.03)[()], f32(0.9)[()], emulate=True)
    Xd = torch.from_numpy(X).cuda()
    with learned.ProposalNet() as net:
        net.params = P
        net.set_forward_mode(1)
        net.set_tc_wait(2_000_000, issue_mma=False)  # 2 ms
        with pytest.raises(g.GlacError) as e:
            net.forward(Xd, 0.03, 0.9)
        assert e.value.status == g.GLAC_ERR_TIMEOUT
        net.set_tc_wait(1_000_000_000, issue_mma=True)
        got = net.forward(Xd, 0.03, 0.9).cpu().numpy()
    d = np.abs(got - want)
    assert np.median(d) < 1e-5 and d.max() < 5e-3
    torch.cuda.synchronize()


def test_gradient_matches_oracle(g, torch, learned):
    rng = np.random.default_rng(3)
    n, K = 5000, 16
    X = rng.standard_normal((n, 8)).astype(np.float32)
    grid = f32(np.geomspace(0.03, 0.9, K))
    J = (np.abs(rng.standard_normal((n, K))) * np.sin(np.pi * grid)[None, :]).astype(np.float32)
    P = random_params(4)
    with learned.ProposalNet() as net:
        net.params = P
        loss, grad = net.loss_grad(torch.from_numpy(X).cuda(), torch.from_numpy(J).cuda(), grid)
        # deterministic: the same call gives the same bits
        loss2, grad2 = net.loss_grad(torch.from_numpy(X).cuda(), torch.from_numpy(J).cuda(), grid)
    assert loss == loss2 and np.array_equal(grad, grad2)
    lo, go = mlp.loss_grad(P.astype(np.float64), X, J, grid, emulate=True)
    assert abs(loss - lo) < 1e-4 * abs(lo)
    for a, b in ((mlp.W1, mlp.B1), (mlp.B1, mlp.W2), (mlp.W2, mlp.B2), (mlp.B2, mlp.W3), (mlp.W3, mlp.NPARAMS)):
        assert np.linalg.norm(grad[a:b] - go[a:b]) < 0.02 * np.linalg.norm(go[a:b]) + 1e-7, (a, b)


def test_training_finds_known_optimum(g, torch, learned):
    # J_i(eps) peaks at eps*(x_i) = 0.1 + 0.5 sigmoid(2 x_i0): the trained spread must follow it
    rng = np.random.default_rng(5)
    n, grid = 65536, f32(np.geomspace(0.03, 0.9, 24))
    X = rng.standard_normal((n, 8)).astype(np.float32)
    target = 0.1 + 0.5 / (1 + np.exp(-2 * X[:, 0]))
    J = np.exp(-((grid[None, :] - target[:, None]) / 0.15) ** 2).astype(np.float32)
    with learned.ProposalNet() as net:
        net.init(9, grid[0], grid[-1], 0.24)
        Xd, Jd = torch.from_numpy(X).cuda(), torch.from_numpy(J).cuda()
        losses = net.train(Xd, Jd, grid, 1500, 4096, 3e-3)
        eps = net.forward(Xd, grid[0], grid[-1]).cpu().numpy()
    assert losses[-100:].mean() < 0.8 * losses[:10].mean()
    assert np.mean(np.abs(eps - target)) < 0.03


def test_learned_chain_keeps_reference_plaquette(g):
    # A spread that varies over [0.1, 0.6] link by link with the staple, with
    # every SU(2) factor near +1, must leave the equilibrium unchanged.  Each
    # chain is thermalised like the reference's (Haar start, 200 plain sweeps),
    # then continues with the learned proposal for the measured sweeps.
    with open(os.path.join(HERE, "golden", "ensemble_4x4x4x8_b6.json")) as f:
        ref = json.load(f)
    from glac_b200.analysis import binned_mean
    P = random_params(6, w3=0.6, b3=0.0)
    plaqs, spreads = [], []
    for i in range(8):
        with g.Lattice(tuple(ref["lattice"]), beta=ref["beta"], precision="fp32", seed=900 + i) as L:
            L.hot_start(300 + i)
            L.metropolis(ref["therm_sweeps"])
            L.set_option("su2_sign_flips", 0)
            L.set_proposal_net(P, 0.1, 0.6)
            p = np.empty(ref["meas_sweeps"])
            for k in range(p.size):
                L.metropolis(1)
                p[k] = L.measure()[0]
            plaqs.append(p)
    mean, err = binned_mean(plaqs, 20)
    sigma = np.hypot(err, ref["plaquette_error"])
    assert abs(mean - ref["plaquette"]) < 3 * sigma, (mean, err, ref["plaquette"])


def test_trained_spread_against_the_method_without_it(g, torch, learned):
    # What the network gains, on held-out rows (mean squared jump per link
    # update): over the method without it -- the plain sampler, the reference's
    # proposal at SU3Eps = 0.24 -- a factor of ~3.3 (3.34 at 32^3 x 64, beta = 6.2);
    # over the same family at 0.24 ~1.1; against the best fixed spread of the
    # family, found by a grid search, it ties (0.9999): the network finds that
    # spread itself and learns almost no per-link variation, so a tie is what
    # this asserts there.
    grid = learned.DEFAULT_GRID
    with g.Lattice((8, 8, 8, 16), beta=6.0, precision="fp32", seed=3) as L:
        L.hot_start(3)
        L.metropolis(300)
        feat, esj, plain = learned.collect_esj(L, 200, 10, 2, grid, trials=4)
    net, rep = learned.train_proposal(feat, esj, grid, steps=800, batch=4096, lr=3e-3, seed=1, esj_plain=plain)
    net.close()
    print("learned spread on held-out rows:", {k: rep[k] for k in ("gain_vs_plain", "gain_vs_024",
                                                                   "gain_vs_best_fixed", "eps_learned_mean",
                                                                   "eps_learned_std", "best_fixed_eps")})
    assert rep["gain_vs_plain"] > 2.5, rep
    assert rep["gain_vs_024"] > 1.05, rep
    assert abs(rep["gain_vs_best_fixed"] - 1.0) < 0.01, rep
    # and its spread lies within one grid step (a factor 1.255) of the best grid point
    assert abs(np.log(rep["eps_learned_mean"] / rep["best_fixed_eps"])) < np.log(grid[1] / grid[0]), rep
