"""Learned Metropolis proposal spread: data, training and the tau_int comparison.

No counterpart in the reference, whose proposals all use the run-config's
SU3Eps (GLAC/math/matrices/su3matrixgenerator.cpp:16-35).  A network maps eight
gauge-invariant features of a link's staple to the spread of that link's
proposals; the staple is unchanged by the link's own update, so the proposal
stays symmetric and the accept step of GLAC/system.cpp:333-361 keeps the chain
exact.  The plain fixed-spread sampler is both its fallback (no network set)
and the yardstick it is measured against (plaquette, <Q^2>, tau_int).

Pipeline (all on the GPU through the C ABI; device buffers are torch tensors):
  collect_esj   plain-sampler sweeps; every `every` sweeps, expected-squared-jump
                rows (features, J(eps_k) on a spread grid) of a strided link sample
                for the learned family (SU(2) factors near +1, glac_set_option
                "su2_sign_flips" 0), and the reference proposal's J(0.24) beside it
  train_proposal  Adam on L = -mean J(eps(f)), BF16 tensor-core forward/backward
  tau_study     plain FP64 / plain FP32 / no-flip best fixed spread (ablation) /
                learned FP32 chains from one start:
                tau_int of the plaquette and of Q(t) (Gamma method), effective
                Q samples per second

``python -m glac_b200.learned study [--dims 24,24,24,48] [--beta 6.0] ...``
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import time

import numpy as np

from . import MLP_NPARAMS, GlacError, Lattice, lib
from .analysis import gamma_method

DEFAULT_GRID = np.geomspace(0.03, 0.9, 16)


def _torch():
    import torch

    if not torch.cuda.is_available():
        raise RuntimeError("the learned proposal needs a CUDA device")
    return torch


class ProposalNet:
    """Trainer of the spread network (glac_mlp_* in include/glac_b200.h)."""

    def __init__(self, device: int = 0):
        self._h = C.c_void_p()
        st = lib().glac_mlp_create(int(device), C.byref(self._h))
        if st != 0:
            raise GlacError(st, "glac_mlp_create failed")
        self.device = device

    def _ck(self, st):
        if st != 0:
            raise GlacError(st, lib().glac_mlp_last_error(self._h).decode())

    def close(self):
        if self._h.value:
            lib().glac_mlp_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def init(self, seed: int, eps_min: float, eps_max: float, eps0: float = 0.24):
        self._ck(lib().glac_mlp_init(self._h, int(seed), float(eps_min), float(eps_max), float(eps0)))

    @property
    def params(self) -> np.ndarray:
        p = np.empty(MLP_NPARAMS, np.float32)
        self._ck(lib().glac_mlp_get_params(self._h, p.ctypes.data))
        return p

    @params.setter
    def params(self, p):
        p = np.ascontiguousarray(p, np.float32)
        if p.size != MLP_NPARAMS:
            raise ValueError(f"need {MLP_NPARAMS} parameters")
        self._ck(lib().glac_mlp_set_params(self._h, p.ctypes.data))

    def set_forward_mode(self, mode: int):
        """0: the sampler's warp-level routine (default); 1: tcgen05 tensor-core tiles."""
        self._ck(lib().glac_mlp_set_forward_mode(self._h, int(mode)))

    def set_tc_wait(self, wait_ns: int, issue_mma: bool = True):
        """Test hook of mode 1: the completion-wait limit of the tcgen05 kernel in
        ns, and (issue_mma=False) a pass that issues no MMA so that its wait runs out."""
        self._ck(lib().glac_mlp_test_tc_wait(self._h, int(wait_ns), int(bool(issue_mma))))

    def forward(self, features, eps_min: float, eps_max: float):
        torch = _torch()
        f = features.contiguous()
        out = torch.empty(f.shape[0], dtype=torch.float32, device=f.device)
        torch.cuda.synchronize()
        self._ck(lib().glac_mlp_forward(self._h, f.data_ptr(), f.shape[0], float(eps_min), float(eps_max),
                                        out.data_ptr()))
        return out

    def loss_grad(self, features, esj, grid):
        torch = _torch()
        g = np.ascontiguousarray(grid, np.float64)
        grad = np.empty(MLP_NPARAMS, np.float32)
        loss = C.c_double(0.0)
        f, j = features.contiguous(), esj.contiguous()
        torch.cuda.synchronize()
        self._ck(lib().glac_mlp_loss_grad(self._h, f.data_ptr(), j.data_ptr(), f.shape[0], g.size, g,
                                          C.byref(loss), grad.ctypes.data))
        return loss.value, grad

    def train(self, features, esj, grid, steps: int, batch: int, lr: float):
        torch = _torch()
        g = np.ascontiguousarray(grid, np.float64)
        losses = np.empty(max(int(steps), 1))
        f, j = features.contiguous(), esj.contiguous()
        torch.cuda.synchronize()
        self._ck(lib().glac_mlp_train(self._h, f.data_ptr(), j.data_ptr(), f.shape[0], g.size, g, int(steps),
                                      int(batch), float(lr), losses.ctypes.data))
        return losses[: int(steps)]


def collect_esj(L: Lattice, sweeps: int, every: int, stride: int, grid=DEFAULT_GRID, trials: int = 4,
                snapshot0: int = 0, flips: bool = False, baseline_eps: float = 0.24):
    """Plain-sampler sweeps (the reference's proposal) with an ESJ snapshot every `every` sweeps.

    Returns (features, esj, esj_plain) on the device: esj[row, k] for the
    proposal family being trained (SU(2) sign flips on or off) at grid[k], and
    esj_plain[row] for the reference's own proposal at baseline_eps on the same
    links and configurations.
    """
    torch = _torch()
    rows = L.esj_rows(stride)
    nsnap = sweeps // every
    feat = torch.empty((nsnap * rows, 8), dtype=torch.float32, device="cuda")
    esj = torch.empty((nsnap * rows, len(grid)), dtype=torch.float32, device="cuda")
    plain = torch.empty((nsnap * rows, 1), dtype=torch.float32, device="cuda")
    scratch = torch.empty((rows, 8), dtype=torch.float32, device="cuda")
    for i in range(nsnap):
        L.set_option("su2_sign_flips", 1)
        L.metropolis(every)
        n = L.esj_data_ptr([baseline_eps], trials, stride, snapshot0 + i, scratch.data_ptr(),
                           plain[i * rows].data_ptr(), None, rows)
        L.set_option("su2_sign_flips", int(flips))
        n2 = L.esj_data_ptr(grid, trials, stride, snapshot0 + i, feat[i * rows].data_ptr(),
                            esj[i * rows].data_ptr(), None, rows)
        assert n == rows and n2 == rows
    L.set_option("su2_sign_flips", 1)
    return feat, esj, plain


def esj_at(esj, grid, eps):
    """Mean over rows of J_i(eps_i) (linear between grid points); eps a scalar or per-row tensor."""
    torch = _torch()
    g = torch.as_tensor(np.asarray(grid, np.float32), device=esj.device)
    e = torch.as_tensor(eps, dtype=torch.float32, device=esj.device).expand(esj.shape[0]).contiguous()
    k = torch.clamp(torch.searchsorted(g, e, right=True) - 1, 0, g.numel() - 2)
    rows = torch.arange(esj.shape[0], device=esj.device)
    j0, j1 = esj[rows, k], esj[rows, k + 1]
    return float((j0 + (j1 - j0) * (e - g[k]) / (g[k + 1] - g[k])).mean())


def train_proposal(feat, esj, grid=DEFAULT_GRID, steps=3000, batch=8192, lr=2e-3, seed=7, holdout=0.1,
                   esj_plain=None, net: ProposalNet | None = None):
    """Shuffle, hold out a fraction, train; returns (net, report).

    The report gives the held-out mean squared jump per link update of the
    trained spread, of the family's fixed spreads (0.24 and the best grid
    point), and, when esj_plain is given, of the reference's own proposal.
    """
    torch = _torch()
    gen = torch.Generator(device="cuda")
    gen.manual_seed(seed)
    idx = torch.randperm(feat.shape[0], device="cuda", generator=gen)
    feat, esj = feat[idx].contiguous(), esj[idx].contiguous()
    nh = int(feat.shape[0] * holdout)
    f_tr, j_tr, f_ho, j_ho = feat[nh:], esj[nh:], feat[:nh], esj[:nh]
    scale = float(j_tr.mean())
    net = net or ProposalNet()
    net.init(seed, float(grid[0]), float(grid[-1]), 0.24)
    t0 = time.time()
    losses = net.train(f_tr, j_tr / scale, grid, steps, min(batch, f_tr.shape[0]), lr)
    t_train = time.time() - t0
    eps_ho = net.forward(f_ho, float(grid[0]), float(grid[-1]))
    fixed = [esj_at(j_ho, grid, float(e)) for e in grid]
    rep = dict(
        rows_train=int(f_tr.shape[0]), rows_holdout=nh, steps=int(steps), batch=int(batch), lr=lr,
        train_seconds=t_train, loss_first=float(losses[0]) * scale, loss_last=float(losses[-1]) * scale,
        esj_learned=esj_at(j_ho, grid, eps_ho), esj_fixed_024=esj_at(j_ho, grid, 0.24),
        esj_best_fixed=max(fixed), best_fixed_eps=float(grid[int(np.argmax(fixed))]),
        eps_learned_mean=float(eps_ho.mean()), eps_learned_std=float(eps_ho.std()),
    )
    rep["gain_vs_024"] = rep["esj_learned"] / rep["esj_fixed_024"]
    rep["gain_vs_best_fixed"] = rep["esj_learned"] / rep["esj_best_fixed"]
    if esj_plain is not None:
        rep["esj_plain_reference_proposal"] = float(esj_plain[idx][:nh].mean())
        rep["gain_vs_plain"] = rep["esj_learned"] / rep["esj_plain_reference_proposal"]
    return net, rep


def run_chain(start, dims, beta, precision, sweeps, meas_every, flow_eps, flow_steps, seed, params=None,
              grid=DEFAULT_GRID, su3_eps=0.24, flips=True, label="", reunit_interval=10):
    """One chain from `start`: plaquette after every sweep, Q(t = flow_eps * flow_steps) every meas_every."""
    plaq = np.empty(sweeps)
    Q = []
    acc = 0.0
    reunit = reunit_interval if precision == "fp32" else 0
    with Lattice(dims, beta=beta, precision=precision, su3_eps=su3_eps, seed=seed, reunit_interval=reunit) as L, \
            Lattice(dims, beta=beta, precision=precision, flow_eps=flow_eps, seed=seed) as F:
        L.set_links(start)
        L.set_option("su2_sign_flips", int(flips))
        if params is not None:
            L.set_proposal_net(params, float(grid[0]), float(grid[-1]))
        L.autotune(2)  # launch variants per chain (field and RNG state restored)
        F.set_links(start)
        F.autotune(2)
        L.sync()
        t0 = time.perf_counter()
        for i in range(sweeps):
            acc += L.metropolis(1)
            plaq[i] = L.measure()[0]
            if (i + 1) % meas_every == 0:
                F.copy_from(L)
                F.flow(flow_steps, measure=False)
                Q.append(F.measure()[1])
        F.sync()
        wall = time.perf_counter() - t0
        unitarity = L.unitarity_violation()
    Q = np.asarray(Q)
    gp, gq = gamma_method(plaq), gamma_method(Q)
    return dict(
        label=label, precision=precision, learned=params is not None, su3_eps=None if params is not None else su3_eps,
        su2_sign_flips=bool(flips), sweeps=sweeps, wall_s=wall, acceptance=acc / sweeps,
        reunit_interval=reunit, unitarity_violation_end=unitarity,
        plaquette=gp.mean, plaquette_err=gp.error, tau_int_plaquette=gp.tau_int, tau_int_plaquette_err=gp.tau_error,
        n_Q=int(Q.size), Q2=float(np.mean(Q * Q)), Q2_err=float(gamma_method(Q * Q).error),
        tau_int_Q=gq.tau_int * meas_every, tau_int_Q_err=gq.tau_error * meas_every,
        eff_Q_per_s=Q.size / (2.0 * gq.tau_int) / wall,
        eff_plaq_per_s=sweeps / (2.0 * gp.tau_int) / wall,
    )


def tau_study(dims=(24, 24, 24, 48), beta=6.0, therm=500, train_sweeps=2000, every=20, stride=64, trials=4,
              sweeps=5000, meas_every=10, flow_eps=0.02, flow_t=1.0, seed=20261203, steps=3000, replicas=1):
    dims = tuple(dims)
    out = dict(dims=list(dims), beta=beta, therm=therm, train_sweeps=train_sweeps, esj_every=every,
               esj_stride=stride, esj_trials=trials, sweeps=sweeps, meas_every=meas_every, flow_eps=flow_eps,
               flow_t=flow_t, grid=[float(x) for x in DEFAULT_GRID])
    t0 = time.time()
    with Lattice(dims, beta=beta, precision="fp32", seed=seed, reunit_interval=10) as L:
        L.hot_start(seed)
        L.metropolis(therm)
        feat, esj, plain = collect_esj(L, train_sweeps, every, stride, DEFAULT_GRID, trials)
        L.reunitarize()
        start = L.get_links()
    out["collect_seconds"] = time.time() - t0
    net, rep = train_proposal(feat, esj, DEFAULT_GRID, steps=steps, seed=seed, esj_plain=plain)
    params = net.params
    net.close()
    del feat, esj, plain
    out["training"] = rep
    fs = int(round(flow_t / flow_eps))
    kinds = [
        dict(precision="fp64", label="plain fp64"),
        dict(precision="fp32", label="plain fp32"),
        dict(precision="fp32", su3_eps=rep["best_fixed_eps"], flips=False, label="fp32 no-flip fixed best eps (ablation)"),
        dict(precision="fp32", params=params, flips=False, label="fp32 learned"),
    ]
    out["replicas"] = replicas
    out["chains"] = []
    for ki, kw in enumerate(kinds):
        runs = [run_chain(start, dims, beta, kw["precision"], sweeps, meas_every, flow_eps, fs,
                          seed + 1 + 100 * ki + r, **{k: v for k, v in kw.items() if k != "precision"})
                for r in range(replicas)]
        c = dict(runs[0])
        for key in ("wall_s", "acceptance", "plaquette", "tau_int_plaquette", "tau_int_Q", "Q2", "eff_Q_per_s",
                    "eff_plaq_per_s"):
            v = np.array([x[key] for x in runs])
            c[key] = float(v.mean())
            c[key + "_replica_err"] = float(v.std(ddof=1) / np.sqrt(len(v))) if len(v) > 1 else None
        c["replica_tau_int_Q"] = [x["tau_int_Q"] for x in runs]
        out["chains"].append(c)
    base = out["chains"][0]
    for c in out["chains"]:
        c["eff_Q_ratio_vs_plain_fp64"] = c["eff_Q_per_s"] / base["eff_Q_per_s"]
        c["eff_plaq_ratio_vs_plain_fp64"] = c["eff_plaq_per_s"] / base["eff_plaq_per_s"]
    out["params"] = [float(x) for x in params]
    return out


def _main():
    ap = argparse.ArgumentParser(prog="python -m glac_b200.learned")
    sub = ap.add_subparsers(dest="cmd", required=True)
    p = sub.add_parser("study", help="train the spread network and compare tau_int with the plain sampler")
    p.add_argument("--dims", default="24,24,24,48")
    p.add_argument("--beta", type=float, default=6.0)
    p.add_argument("--therm", type=int, default=500)
    p.add_argument("--train-sweeps", type=int, default=2000)
    p.add_argument("--every", type=int, default=20)
    p.add_argument("--stride", type=int, default=64)
    p.add_argument("--sweeps", type=int, default=5000)
    p.add_argument("--meas-every", type=int, default=10)
    p.add_argument("--steps", type=int, default=3000)
    p.add_argument("--replicas", type=int, default=1, help="independent chains per sampler")
    p.add_argument("--out", default="")
    a = ap.parse_args()
    r = tau_study(tuple(int(x) for x in a.dims.split(",")), a.beta, a.therm, a.train_sweeps, a.every, a.stride,
                  sweeps=a.sweeps, meas_every=a.meas_every, steps=a.steps, replicas=a.replicas)
    s = json.dumps(r)
    if a.out:
        with open(a.out, "w") as f:
            f.write(s)
    summary = {k: v for k, v in r.items() if k not in ("params", "grid")}
    print(json.dumps(summary))


if __name__ == "__main__":
    _main()
