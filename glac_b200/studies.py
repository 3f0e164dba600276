"""Physics studies run on the GPU path.

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
    a = ap.parse_args()
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
