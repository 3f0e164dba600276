"""Physics studies run on the GPU path.

``python -m glac_b200.studies large [--dims 48,48,48,96] [--beta 6.45]``
    Rates of the large run: plain FP64, plain FP32 and learned FP32 Metropolis
    (link-updates/s), FP32 and FP64 flow with per-step observables (site-steps/s),
    the HBM GB/s of the flow stage, and one full flow to t = 4 (400 RK3 steps).

``python -m glac_b200.studies precision [--dims 32,32,32,64] [--steps 1000]``
    Flow-only precision test: a start field from plain FP64 Metropolis sweeps
    (seeded Haar start), flowed with Luescher RK3 (Morningstar-Peardon
    exponential, FP64 global sums) once with FP64 links and once with FP32
    links.  Reports, per flow step, the plaquette, E(t), t^2 E(t) and Q(t) of
    both runs and the FP32 deviation from FP64.  E is the clover energy density
    in physical normalisation, E = -E_ref / 64, with E_ref the reference's
    energy observable (GLAC/observables/mastersampler.cpp:13-15, 175-287).
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np

from . import Lattice


def energy_physical(e_ref):
    """Clover E(t) from the reference's energy output ((1/V) sum ReTr C C, C = 8 i F a^2)."""
    return -np.asarray(e_ref) / 64.0


def precision_study(dims=(32, 32, 32, 64), beta=6.2, sweeps=600, steps=1000, eps=0.01, seed=20261203,
                    start=None):
    """Returns a dict of per-step arrays (fp64, fp32, deviations) and a summary."""
    t0 = time.time()
    with Lattice(dims, beta=beta, precision="fp64", flow_eps=eps, seed=seed) as L64:
        if start is None:
            L64.hot_start(seed)
            L64.metropolis(sweeps)
            start = L64.get_links()
        else:
            L64.set_links(start)
        t_start = time.time() - t0
        obs64 = L64.flow(steps)
    with Lattice(dims, beta=beta, precision="fp32", flow_eps=eps, seed=seed) as L32:
        L32.set_links(start)
        obs32 = L32.flow(steps)
    t = eps * np.arange(steps + 1)
    out = {"t": t}
    for tag, o in (("fp64", obs64), ("fp32", obs32)):
        E = energy_physical(o[:, 2])
        out[tag] = {"plaq": o[:, 0], "E": E, "t2E": t * t * E, "Q": o[:, 1]}
    summary = {}
    for k in ("plaq", "E", "t2E", "Q"):
        a, b = out["fp64"][k], out["fp32"][k]
        d = np.abs(b - a)
        rel = d / np.maximum(np.abs(a), 1e-300)
        summary[k] = {
            "max_abs_dev": float(d.max()),
            "max_rel_dev": float(rel[1:].max() if k == "t2E" else rel.max()),
            "final_fp64": float(a[-1]),
            "final_fp32": float(b[-1]),
        }
    summary["dims"] = list(dims)
    summary["beta"] = beta
    summary["sweeps"] = sweeps
    summary["steps"] = steps
    summary["seconds"] = time.time() - t0
    summary["start_seconds"] = t_start
    out["summary"] = summary
    return out


STAGE_BYTES_FP32 = (704, 832, 704)  # per site: 4 links read + 4 written + force traffic per RK3 stage


def large_run(dims=(48, 48, 48, 96), beta=6.45, therm=200, seed=20261203, flow_steps=400):
    import torch

    from . import learned as lp

    V = int(np.prod(dims))
    out = {"dims": list(dims), "beta": beta, "sites": V, "therm_sweeps": therm}

    def timed(L, fn):
        st = torch.cuda.ExternalStream(L.stream)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        fn()
        e1.record(st)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / 1e3

    with Lattice(dims, beta=beta, precision="fp32", seed=seed, reunit_interval=10) as L:
        L.hot_start(seed)
        L.metropolis(5)
        out["autotune_fp32"] = L.autotune(2)
        L.metropolis(therm)
        out["link_updates_per_s_fp32_plain"] = 4 * V * 20 / timed(L, lambda: L.metropolis(20))
        feat, esj, plain = lp.collect_esj(L, 50, 10, 256, lp.DEFAULT_GRID, trials=4)
        net, rep = lp.train_proposal(feat, esj, lp.DEFAULT_GRID, steps=1000, batch=8192, lr=2e-3, seed=1,
                                     esj_plain=plain)
        params = net.params
        net.close()
        del feat, esj, plain
        out["training"] = rep
        L.set_option("su2_sign_flips", 0)
        L.set_proposal_net(params, float(lp.DEFAULT_GRID[0]), float(lp.DEFAULT_GRID[-1]))
        L.metropolis(2)
        out["link_updates_per_s_fp32_learned"] = 4 * V * 20 / timed(L, lambda: L.metropolis(20))
        L.set_proposal_net(None)
        L.set_option("su2_sign_flips", 1)
        L.reunitarize()
        start = L.get_links()
        with Lattice(dims, beta=beta, precision="fp32", seed=seed) as F:
            F.set_links(start)
            F.autotune(2)
            F.set_links(start)
            obs = np.empty((flow_steps + 1, 3 + dims[3]))
            t = timed(F, lambda: F.flow(flow_steps, out=obs))
            out["flow_fp32_seconds_to_t4"] = t
            out["flow_site_steps_per_s_fp32"] = V * flow_steps / t
            st = np.array(F.flow_stage_times(10))
            out["flow_stage_ms_fp32"] = [float(x) * 1e3 for x in st]
            out["flow_stage0_algorithmic_GBps_fp32"] = STAGE_BYTES_FP32[0] * V / float(st[0]) / 1e9
            out["t2E_at_t4"] = float(16.0 * (-obs[-1, 2] / 64.0))
            out["Q_at_t4"] = float(obs[-1, 1])
    with Lattice(dims, beta=beta, precision="fp64", seed=seed) as L64:
        L64.set_links(start)
        L64.metropolis(2)
        out["link_updates_per_s_fp64_plain"] = 4 * V * 10 / timed(L64, lambda: L64.metropolis(10))
        L64.set_links(start)
        out["flow_site_steps_per_s_fp64"] = V * 20 / timed(L64, lambda: L64.flow(20))
    out["learned_fp32_vs_plain_fp64_link_updates"] = (out["link_updates_per_s_fp32_learned"]
                                                      / out["link_updates_per_s_fp64_plain"])
    return out


def _main():
    ap = argparse.ArgumentParser(prog="python -m glac_b200.studies")
    sub = ap.add_subparsers(dest="study", required=True)
    p = sub.add_parser("precision", help="FP32 vs FP64 flow observables")
    p.add_argument("--dims", default="32,32,32,64")
    p.add_argument("--beta", type=float, default=6.2)
    p.add_argument("--sweeps", type=int, default=600)
    p.add_argument("--steps", type=int, default=1000)
    p.add_argument("--seed", type=int, default=20261203)
    p.add_argument("--npz", default="", help="write the per-step arrays here")
    q = sub.add_parser("large", help="rates of the 48^3x96 learned-proposal run")
    q.add_argument("--dims", default="48,48,48,96")
    q.add_argument("--beta", type=float, default=6.45)
    q.add_argument("--therm", type=int, default=200)
    a = ap.parse_args()
    if a.study == "large":
        print(json.dumps(large_run(tuple(int(x) for x in a.dims.split(",")), a.beta, a.therm)))
        return
    if a.study == "precision":
        dims = tuple(int(x) for x in a.dims.split(","))
        r = precision_study(dims, a.beta, a.sweeps, a.steps, seed=a.seed)
        if a.npz:
            flat = {"t": r["t"]}
            for tag in ("fp64", "fp32"):
                for k, v in r[tag].items():
                    flat[f"{tag}_{k}"] = v
            np.savez_compressed(a.npz, **flat)
        print(json.dumps(r["summary"]))


if __name__ == "__main__":
    _main()
