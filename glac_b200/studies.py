"""Physics studies run on the GPU path.

``python -m glac_b200.studies large [--dims 48,48,48,96] [--beta 6.45]``
    Rates of the large run: plain FP64, plain FP32 and learned FP32 Metropolis
    (link-updates/s), FP32 and FP64 flow with per-step observables (site-steps/s),
    the HBM GB/s of the flow stage, and one full flow to t = 4 (400 RK3 steps).

``python -m glac_b200.studies target [--replicas 0,1,2,3] [--samplers ...] [--out f.json]``
``python -m glac_b200.studies target-combine f1.json f2.json ...``
    The effective-topological-charge study at 32^3 x 64, beta = 6.2: from
    independently thermalised starts (one per replica), chains of the plain
    FP64 sampler (the reference's proposal, SU3Eps = 0.24), the plain FP32
    sampler, the FP32 sampler with the no-flip proposal family at its best fixed
    spread (the ablation) and the FP32 learned-spread sampler; Q and E at flow
    time t and the plaquette every `meas_every` sweeps; effective Q samples per
    second = N_meas / (2 tau_int,Q) / wall seconds (sweeps and measurements),
    tau_int by the replica Gamma method, errors by a delete-one-replica
    jackknife.  Replicas can be run in separate processes and combined.

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


# ---------------------------------------------------------------------------
# effective topological-charge samples per second at the target configuration
# ---------------------------------------------------------------------------
TARGET = dict(dims=(32, 32, 32, 64), beta=6.2, therm=3000, sweeps=30000, meas_every=100, flow_eps=0.04,
              flow_t=2.0, train_therm=1000, train_sweeps=400, train_every=20, seed=20261203,
              # chain length per sampler: the plain kernel decorrelates Q slowest
              # (tau_int,Q ~ 1000 sweeps at 32^3 x 64, beta = 6.2), the FP64 chains
              # give its FP64 wall time and a consistency check of the FP32 twin
              sweeps_by={"plain_fp64": 10000, "plain_fp32": 60000, "ablation_fp32": 30000,
                         "learned_fp32": 30000})
SAMPLERS = ("plain_fp64", "plain_fp32", "ablation_fp32", "learned_fp32")


def target_training(cfg=TARGET):
    """Train the spread network on ESJ data of the plain FP32 sampler at the
    target coupling; returns (params, training report)."""
    from . import learned as lp
    dims, beta, seed = tuple(cfg["dims"]), cfg["beta"], cfg["seed"]
    with Lattice(dims, beta=beta, precision="fp32", seed=seed, stream_id=999, reunit_interval=10) as L:
        L.hot_start(seed + 999)
        L.set_option("su2_sign_flips", 0)
        L.metropolis(cfg["train_therm"])
        L.set_option("su2_sign_flips", 1)
        feat, esj, plain = lp.collect_esj(L, cfg["train_sweeps"], cfg["train_every"], 64, lp.DEFAULT_GRID, trials=4)
    net, rep = lp.train_proposal(feat, esj, lp.DEFAULT_GRID, steps=3000, seed=seed, esj_plain=plain)
    params = net.params
    net.close()
    return params, rep


def target_start(cfg, replica, params=None, best_eps=0.36):
    """Replica `replica`'s start: its own Haar field thermalised by cfg["therm"]
    sweeps of the no-flip FP32 sampler at best_eps (reunitarised every 10)."""
    dims, beta, seed = tuple(cfg["dims"]), cfg["beta"], cfg["seed"]
    with Lattice(dims, beta=beta, precision="fp32", su3_eps=best_eps, seed=seed, stream_id=1000 + replica,
                 reunit_interval=10) as L:
        L.hot_start(seed + 7919 * (replica + 1))
        L.set_option("su2_sign_flips", 0)
        L.metropolis(cfg["therm"])
        L.reunitarize()
        return L.get_links()


def q_chain(start, cfg, sampler, replica, params=None, best_eps=0.36):
    """One chain of `sampler` from `start`; every meas_every sweeps the plaquette
    of the chain and Q, E of a flowed copy at t = flow_t.  Wall seconds cover the
    sweeps and the measurements (device synchronised at both ends)."""
    from .learned import DEFAULT_GRID
    dims, beta, seed = tuple(cfg["dims"]), cfg["beta"], cfg["seed"]
    prec = "fp64" if sampler.endswith("fp64") else "fp32"
    flips = sampler.startswith("plain")
    eps = best_eps if sampler.startswith("ablation") else 0.24
    stream = 10 * replica + SAMPLERS.index(sampler)
    fs = int(round(cfg["flow_t"] / cfg["flow_eps"]))
    sweeps = int(cfg.get("sweeps_by", {}).get(sampler, cfg["sweeps"]))
    nmeas = sweeps // cfg["meas_every"]
    plaq, Q, E = np.empty(nmeas), np.empty(nmeas), np.empty(nmeas)
    acc = 0.0
    with Lattice(dims, beta=beta, precision=prec, su3_eps=eps, seed=seed, stream_id=stream,
                 reunit_interval=10 if prec == "fp32" else 0) as L, \
            Lattice(dims, beta=beta, precision=prec, flow_eps=cfg["flow_eps"], seed=seed) as F:
        L.set_links(start)
        L.set_option("su2_sign_flips", int(flips))
        if sampler.startswith("learned"):
            L.set_proposal_net(params, float(DEFAULT_GRID[0]), float(DEFAULT_GRID[-1]))
        L.autotune(2)  # launch variants (field and random stream restored)
        F.set_links(start)
        F.autotune(2)
        L.sync()
        F.sync()
        t0 = time.perf_counter()
        for i in range(nmeas):
            acc += L.metropolis(cfg["meas_every"])
            plaq[i] = L.measure()[0]
            F.copy_from(L)
            F.flow(fs, measure=False)
            o = F.measure()
            Q[i], E[i] = o[1], o[2]
        F.sync()
        wall = time.perf_counter() - t0
    return dict(sampler=sampler, replica=replica, precision=prec, su3_eps=None if sampler.startswith("learned") else eps,
                su2_sign_flips=flips, sweeps=nmeas * cfg["meas_every"], meas_every=cfg["meas_every"], wall_s=wall,
                acceptance=acc / nmeas, plaq=plaq.tolist(), Q=Q.tolist(), E=E.tolist())


def target_run(replicas, samplers=SAMPLERS, cfg=TARGET, params=None, out_path=""):
    """Chains of the given samplers for the given replicas (training first when
    params is None); a JSON-able dict that target_combine merges, also written
    to out_path after every replica."""
    out = dict(config={k: (list(v) if isinstance(v, tuple) else v) for k, v in cfg.items()}, chains=[])
    if params is None:
        params, rep = target_training(cfg)
        out["training"] = rep
    else:
        rep = None
    params = np.asarray(params, np.float32)
    best = float(rep["best_fixed_eps"]) if rep else float(cfg.get("best_eps", 0.36))
    out["params"] = [float(x) for x in params]
    out["best_eps"] = best
    for r in replicas:
        t0 = time.time()
        start = target_start(cfg, r, params, best)
        therm_s = time.time() - t0
        for smp in samplers:
            c = q_chain(start, cfg, smp, r, params, best)
            c["therm_seconds"] = therm_s
            out["chains"].append(c)
        if out_path:
            with open(out_path, "w") as f:
                json.dump(out, f)
    return out


def target_combine(runs):
    """Per sampler: tau_int of Q and of the plaquette (replica Gamma method),
    effective Q samples per second, means; ratios to plain FP64 with
    delete-one-replica jackknife errors.  tau_int,Q of the plain FP64 sampler
    is also given from its FP32 twin (the same Markov kernel up to rounding),
    pooled with it when both ran."""
    from .analysis import gamma_method_replicas, jackknife
    chains = [c for r in runs for c in r["chains"]]
    by = {}
    for c in chains:
        by.setdefault(c["sampler"], {})[c["replica"]] = c
    res = {}

    def stats(cs):
        tq = gamma_method_replicas([c["Q"] for c in cs])
        tp = gamma_method_replicas([c["plaq"] for c in cs])
        q2 = gamma_method_replicas([np.square(c["Q"]) for c in cs])
        te = gamma_method_replicas([c["E"] for c in cs])
        nmeas = sum(len(c["Q"]) for c in cs)
        wall = sum(c["wall_s"] for c in cs)
        return dict(tau_Q=tq.tau_int * cs[0]["meas_every"], tau_Q_err=tq.tau_error * cs[0]["meas_every"],
                    tau_plaq=tp.tau_int * cs[0]["meas_every"], plaq=tp.mean, plaq_err=tp.error,
                    Q2=q2.mean, Q2_err=q2.error, E=te.mean, E_err=te.error, n_meas=nmeas, wall_s=wall,
                    sweep_seconds=wall / sum(c["sweeps"] for c in cs),
                    eff_Q_per_s=nmeas / (2.0 * tq.tau_int) / wall, replicas=sorted(c["replica"] for c in cs),
                    acceptance=float(np.mean([c["acceptance"] for c in cs])))

    for smp, reps in by.items():
        res[smp] = stats(list(reps.values()))
    common = sorted(set.intersection(*[set(v) for v in by.values()])) if by else []
    base = "plain_fp64" if "plain_fp64" in res else None
    if base:
        for smp in res:
            res[smp]["eff_Q_ratio_vs_plain_fp64"] = res[smp]["eff_Q_per_s"] / res[base]["eff_Q_per_s"]
            if len(common) >= 2:
                loo = []
                for k in common:
                    keep = [r for r in common if r != k]
                    a = stats([by[smp][r] for r in keep])
                    b = stats([by[base][r] for r in keep])
                    loo.append(a["eff_Q_per_s"] / b["eff_Q_per_s"])
                res[smp]["eff_Q_ratio_err"] = jackknife(loo)
    if "plain_fp32" in res and "plain_fp64" in res:
        # The FP64 path with tau_int,Q of its FP32 twin (the same Markov kernel:
        # the same proposals from the same streams and the same accept rule, only
        # the rounding differs), which runs long chains at a third of the cost:
        # effective samples per second = 1 / (2 tau_int,Q [sweeps] x seconds per
        # sweep, measurements included).  Ratios with a delete-one-replica
        # jackknife over the replicas all three samplers share.
        # (The FP64 seconds per sweep come from all its chains: a timing, not a
        # statistical estimate; the jackknife runs over the replicas that the
        # sampler and the FP32 twin share.)
        f64 = res["plain_fp64"]

        def eff_twin(keep, smp):
            a = stats([by[smp][r] for r in keep])
            tw = stats([by["plain_fp32"][r] for r in keep])
            return (tw["tau_Q"] * f64["sweep_seconds"]) / (a["tau_Q"] * a["sweep_seconds"])

        f64["eff_Q_per_s_twin_tau"] = 1.0 / (2.0 * res["plain_fp32"]["tau_Q"] * f64["sweep_seconds"])
        for smp in res:
            res[smp]["eff_Q_ratio_vs_plain_fp64_twin_tau"] = (1.0 / (2.0 * res[smp]["tau_Q"] * res[smp]["sweep_seconds"])
                                                            / f64["eff_Q_per_s_twin_tau"])
            shared = sorted(set(by[smp]) & set(by["plain_fp32"]))
            if len(shared) >= 2 and smp != "plain_fp64":
                loo = [eff_twin([r for r in shared if r != k], smp) for k in shared]
                res[smp]["eff_Q_ratio_twin_tau_err"] = jackknife(loo)
    # Q diffusion: D(lag) = <(Q_{i+lag} - Q_i)^2> over all chains of a sampler.
    # For lags well below tau_int,Q it grows as 2 <Q^2> lag / tau, so D per
    # sweep is proportional to the rate at which Q decorrelates, and
    # D(lag) / (lag x seconds per sweep) compares effective Q samples per second
    # between samplers without an estimate of tau_int itself, with far smaller
    # statistical errors when the chains are only tens of tau_int long.
    meas_every = chains[0]["meas_every"]
    for lag_sweeps in (200, 500, 1000):
        k = lag_sweeps // meas_every
        key = f"Q_diffusion_{lag_sweeps}"
        for smp, reps in by.items():
            per = {r: float(np.mean((np.asarray(c["Q"])[k:] - np.asarray(c["Q"])[:-k]) ** 2)) for r, c in reps.items()}
            n = {r: len(c["Q"]) - k for r, c in reps.items()}
            D = sum(per[r] * n[r] for r in per) / sum(n.values())
            res[smp][key] = D
            if len(per) >= 2:
                loo = [sum(per[r] * n[r] for r in per if r != q) / sum(n[r] for r in per if r != q) for q in per]
                res[smp][key + "_err"] = jackknife(loo)
        if "plain_fp64" in res:
            base = res["plain_fp64"][key] / res["plain_fp64"]["sweep_seconds"]
            rel_base = res["plain_fp64"].get(key + "_err", 0.0) / res["plain_fp64"][key]
            for smp in res:
                ratio = res[smp][key] / res[smp]["sweep_seconds"] / base
                res[smp][f"eff_Q_ratio_vs_plain_fp64_diffusion_{lag_sweeps}"] = ratio
                if smp != "plain_fp64" and key + "_err" in res[smp]:
                    rel = res[smp][key + "_err"] / res[smp][key]
                    res[smp][f"eff_Q_ratio_vs_plain_fp64_diffusion_{lag_sweeps}_err"] = ratio * float(
                        np.hypot(rel, rel_base))
    return dict(config=runs[0]["config"], best_eps=runs[0].get("best_eps"), samplers=res,
                training=next((r["training"] for r in runs if r.get("training")), None))


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
    t = sub.add_parser("target", help="effective Q samples/s at 32^3x64, beta=6.2, per sampler")
    t.add_argument("--replicas", default="0,1,2,3")
    t.add_argument("--samplers", default=",".join(SAMPLERS))
    t.add_argument("--sweeps", type=int, default=0, help="one chain length for all samplers (default: per sampler)")
    t.add_argument("--meas-every", type=int, default=TARGET["meas_every"])
    t.add_argument("--therm", type=int, default=TARGET["therm"])
    t.add_argument("--dims", default="32,32,32,64")
    t.add_argument("--params", default="", help="JSON of an earlier run whose trained network to reuse")
    t.add_argument("--out", default="")
    c = sub.add_parser("target-combine", help="merge target runs and print the summary")
    c.add_argument("files", nargs="+")
    a = ap.parse_args()
    if a.study == "target":
        cfg = dict(TARGET, meas_every=a.meas_every, therm=a.therm, dims=tuple(int(x) for x in a.dims.split(",")))
        if a.sweeps:  # one length for every sampler
            cfg["sweeps"], cfg["sweeps_by"] = a.sweeps, {}
        params = None
        if a.params:
            with open(a.params) as f:
                prev = json.load(f)
            params = prev["params"]
            cfg["best_eps"] = prev["best_eps"]
        r = target_run([int(x) for x in a.replicas.split(",")], a.samplers.split(","), cfg, params, a.out)
        print(json.dumps(target_combine([r])["samplers"]))
        return
    if a.study == "target-combine":
        runs = []
        for fn in a.files:
            with open(fn) as f:
                runs.append(json.load(f))
        print(json.dumps(target_combine(runs), indent=1))
        return
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
