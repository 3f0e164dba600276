"""Benchmark of the GLAC hot path on B200.

Workload (one GPU): gradient flow of a 32^3 x 64 lattice (2,097,152 sites) at
beta = 6.2, links in FP32 with FP64 reductions, Luscher RK3 at eps = 0.01,
Morningstar-Peardon exponential; the start field is a seeded Haar field after
600 checkerboard Metropolis sweeps (10 hits, SU3Eps = 0.24).  One "step" is one
RK3 flow step followed by the plaquette / energy / topological-charge
measurement, as GLAC's System::flowConfiguration does per flow step.

Metric: flow site-steps/s (sites x steps / s), higher is better.  Also
reported: the same without per-step observables, FP64, Metropolis
link-updates/s, the roofline of the flow-stage kernel, the reference's CPU
path timed on this host, and an end-to-end number through the C ABI with host
buffers.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

Under torchrun (N > 1) every rank flows its own independent lattice (replicas,
no collective on the data path); value = all ranks' site-steps / max time.
"""
from __future__ import annotations

import argparse
import json
import multiprocessing as mp
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

DIMS = (32, 32, 32, 64)
BETA = 6.2
FLOW_EPS = 0.01
SU3_EPS = 0.24
NHITS = 10
THERM_SWEEPS = 600
METRIC = "flow site-steps/s at 32^3x64 (RK3 step + plaq/E/Q measurement per step)"
UNIT = "site-steps/s"
WORKLOAD = "GLAC gradient flow 32^3x64, beta=6.2, eps=0.01, FP32 links + FP64 sums, per-step observables"
# algorithmic bytes per site for the three RK3 stages in FP32 (18 reals/link, 8 reals/force):
# reads 4 links + writes 4 links per stage, force written (stage 0), read+written (1), read (2)
STAGE_BYTES_FP32 = (8 * 72 + 4 * 32, 8 * 72 + 8 * 32, 8 * 72 + 4 * 32)
STAGE_BYTES_FP64 = tuple(2 * b for b in STAGE_BYTES_FP32)
# stage 0 with the measurement's clover parts: + 12 slots x 32 B + 4 plaquette floats per site written
STAGE0_MEAS_BYTES_FP32 = STAGE_BYTES_FP32[0] + 12 * 32 + 4 * 4
# dram__bytes_read.sum + dram__bytes_write.sum of one ncu capture of that launch at
# 32^3x64 (k_flow_stage0_meas_r128, profiles/flow_stage0_meas_fp32_32x32x32x64.md)
NCU_TRAFFIC_STAGE0_MEAS_FP32 = 707025920 + 1665065000
# FP32 FLOP per site of that launch: (2 x FFMA + FADD + FMUL) thread instructions
# counted by ncu (sm__sass_thread_inst_executed_op_{ffma,fadd,fmul}_pred_on) on the
# 32^3x64 launch = (2 x 13,178,503,168 + 1,472,200,704 + 1,627,389,952) / 2,097,152
FLOPS_PER_SITE_STAGE0_MEAS_FP32 = 14046
# the same count for the plain stage-0 launch (no measurement):
# (2 x 12,071,206,912 + 494,927,872 + 1,098,907,648) / 2,097,152
FLOPS_PER_SITE_STAGE0_FP32 = 12272
SM_COUNT, FP32_LANES_PER_SM = 148, 128
# The metric's third leg, effective Q samples/s of the learned FP32 sampler
# against the plain FP64 GPU path at 32^3x64, beta = 6.2: a study of
# 4 replicas x tens of thousands of sweeps per sampler (about 40 GPU-minutes),
# recorded in profiles/eff_q_study_32x32x32x64_b6.2.md and reproduced by
# `python -m glac_b200.studies target`; bench.py reports it, it does not
# re-measure it.
EFF_Q_STUDY = {"measured_in_this_run": False, "source": "profiles/eff_q_study_32x32x32x64_b6.2.md",
               "ratio_learned_fp32_vs_plain_fp64": 8.06, "err": 0.63,
               "ratio_ablation_fp32_vs_plain_fp64": 8.97, "ablation_err": 0.89,
               "estimator": "Q diffusion over 500 sweeps per second of sweeps + measurements, replica jackknife",
               "replicas": 12, "plaquette_learned_minus_fp64_sigma": 0.6}
# The study's ratio factorises as (Q diffusion per sweep, learned / plain FP64:
# D(500) 19.2 / 5.82) x (seconds per sweep with measurements, plain FP64 /
# learned: 9.616 / 3.933 ms).  The second factor is re-measured in every bench
# run on the bench's own lattice (same lattice, coupling and measurement
# schedule); the first needs chains of 10^4-10^5 sweeps and is quoted.
EFF_Q_DIFFUSION_PER_SWEEP_RATIO = (19.2 / 5.82, 0.63 / 8.06 * 19.2 / 5.82)
EFF_Q_SWEEPS_TIMED = 300
# Metropolis: algorithmic bytes per link update in FP32 (9 link transfers x 72 B)
METRO_BYTES_FP32 = 9 * 72
# FP32 FLOP per link update (10 hits) from one ncu capture of k_metropolis_r96<float>
# at 32^3x64: 2580 FFMA + 225 FADD + 607 FMUL per link update
FLOPS_PER_LINK_UPDATE_METRO_FP32 = 2 * 2580 + 225 + 607


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


# ---------------------------------------------------------------------------
# clocks sampled during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    """SM clock and clock-event reasons of one GPU, sampled in a thread while the
    GPU works: by NVML queries every 2 ms (read-only: current and maximum SM
    clock, current clock-event reasons), or by `nvidia-smi -lms 100` where NVML
    is unavailable.  stop(window) summarises the samples taken inside the
    perf_counter window (t0, t1) when there are at least three, else all."""
    NAMES = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap", "hw_power_brake_slowdown")
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int, period_s: float = 0.002):
        self.dev = device_index
        self.period = period_s
        self.samples = []  # (perf_counter, sm MHz, set of reasons)
        self.smax = None
        self.proc = None
        self.nvml = None
        self.stop_flag = threading.Event()

    def _nvml_handle(self):
        import pynvml
        pynvml.nvmlInit()
        n = pynvml.nvmlDeviceGetCount()
        uuid = None
        try:
            import torch
            uuid = str(torch.cuda.get_device_properties(self.dev).uuid)
        except Exception:
            uuid = None
        for i in range(n):
            h = pynvml.nvmlDeviceGetHandleByIndex(i)
            u = pynvml.nvmlDeviceGetUUID(h)
            u = u.decode() if isinstance(u, bytes) else u
            if uuid and u.replace("GPU-", "") == uuid.replace("GPU-", ""):
                return pynvml, h
        return pynvml, pynvml.nvmlDeviceGetHandleByIndex(self.dev if self.dev < n else 0)

    def start(self):
        try:
            nv, h = self._nvml_handle()
            bits = {"hw_slowdown": nv.nvmlClocksEventReasonHwSlowdown,
                    "hw_thermal_slowdown": nv.nvmlClocksEventReasonHwThermalSlowdown,
                    "sw_thermal_slowdown": nv.nvmlClocksEventReasonSwThermalSlowdown,
                    "sw_power_cap": nv.nvmlClocksEventReasonSwPowerCap,
                    "hw_power_brake_slowdown": nv.nvmlClocksEventReasonHwPowerBrakeSlowdown}
            self.smax = float(nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM))
            self.nvml = (nv, h, bits)
            self.t = threading.Thread(target=self._poll, daemon=True)
            self.t.start()
            return
        except Exception:
            self.nvml = None
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.dev), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except FileNotFoundError:
            self.proc = None

    def _poll(self):
        nv, h, bits = self.nvml
        while not self.stop_flag.is_set():
            try:
                sm = float(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM))
                r = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
            except Exception:
                break
            self.samples.append((time.perf_counter(), sm, {k for k, b in bits.items() if r & b}))
            time.sleep(self.period)

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.strip().split(",")]
            if len(parts) < 9:
                continue
            try:
                sm = float(parts[1])
                self.smax = float(parts[2])
            except ValueError:
                continue
            rs = {nm for nm, v in zip(self.NAMES[:4], parts[5:9]) if v.lower().startswith("active")}
            self.samples.append((time.perf_counter(), sm, rs))

    def stop(self, window=None):
        if self.nvml:
            self.stop_flag.set()
            self.t.join(timeout=5)
            how = "NVML every 2 ms"
        elif self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            how = "nvidia-smi every 100 ms"
        else:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["clock sampling unavailable"]}
        sel = self.samples
        if window is not None:
            inside = [x for x in self.samples if window[0] <= x[0] <= window[1]]
            if len(inside) >= 3:
                sel = inside
        sm = [x[1] for x in sel]
        reasons = set().union(*[x[2] for x in sel]) if sel else set()
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": self.smax,
                "sm_mhz_min": min(sm) if sm else None, "reasons": sorted(reasons), "samples": len(sm),
                "sampled_by": how,
                "window": ("all samples" if window is None else
                           "timed region" if sel is not self.samples else "all samples (under 3 in the timed region)")}


# ---------------------------------------------------------------------------
# CPU baseline and reference arm: the reference's own flow + measurement
# (oracle/_ref, the GLAC sources compiled with the reference's -O3 -march=native
# where the host CPU allows, else the oracle C port), one process per core on
# independent 32^3 x 64 lattices -- the reference parallelises only through MPI
# domain decomposition, which this single-node build does not have.
# ---------------------------------------------------------------------------
# peak resident memory of one reference process flowing and measuring a lattice,
# per site (measured: 9.53 GB peak at 32^3 x 64 = 4545 B per site, rounded up)
REF_BYTES_PER_SITE = 5000


def host_memory_available():
    """Bytes this process may still use: MemAvailable, capped by a cgroup limit."""
    avail = None
    try:
        with open("/proc/meminfo") as f:
            for line in f:
                if line.startswith("MemAvailable:"):
                    avail = int(line.split()[1]) * 1024
    except OSError:
        pass
    for lim, use in (("/sys/fs/cgroup/memory.max", "/sys/fs/cgroup/memory.current"),
                     ("/sys/fs/cgroup/memory/memory.limit_in_bytes", "/sys/fs/cgroup/memory/memory.usage_in_bytes")):
        try:
            with open(lim) as f:
                raw = f.read().strip()
            if raw == "max":
                continue
            with open(use) as f:
                room = int(raw) - int(f.read().strip())
            avail = room if avail is None else min(avail, room)
        except (OSError, ValueError):
            continue
    return avail


def cpu_model():
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown CPU"


def _cpu_worker(args, barrier, results):
    """One process: warm up on an 8^3 x 16 lattice, build its own Haar field at
    dims, wait for the others, then time nsteps x (RK3 step + measurement)."""
    idx, kind, dims, nsteps, seed, warm = args
    sys.path.insert(0, ROOT)
    from oracle.oracle import Oracle, Reference
    o = Oracle()
    r = Reference() if kind == "reference" else None
    if warm and r is not None:
        r.configure(8, 16, beta=BETA, flow_eps=FLOW_EPS, nflows=warm)
        r.time_flow_measure(o.haar_field((8, 8, 8, 16), seed), warm)
    links = o.haar_field(dims, seed)
    if r is not None:
        r.configure(dims[0], dims[3], beta=BETA, flow_eps=FLOW_EPS, nflows=nsteps)
    barrier.wait(timeout=900)
    if r is not None:
        dt = r.time_flow_measure(links, nsteps)
    else:
        t0 = time.perf_counter()
        cur = links
        for _ in range(nsteps):
            cur = o.flow(dims, cur, FLOW_EPS, 1)
            o.observables(dims, cur)
        dt = time.perf_counter() - t0
    results.put((idx, dt))


def cpu_kind():
    from oracle.oracle import REF_SO
    return "reference" if os.path.exists(REF_SO) else "port"


def cpu_flow_rate(nsteps_per_proc: int = 1, dims=DIMS, procs=None, warm=0):
    """Aggregate site-steps/s of the reference's flow + per-step observables on
    this host: `procs` processes (default: one per core, as many as host memory
    holds) each flow and measure their own lattice for nsteps_per_proc steps,
    started together; value = all lattice-steps / the slowest process's time."""
    kind = cpu_kind()
    V = int(np.prod(dims))
    cores = os.cpu_count() or 1
    avail = host_memory_available()
    by_mem = max(1, int(0.8 * avail // (REF_BYTES_PER_SITE * V))) if avail else cores
    procs = procs or max(1, min(cores, by_mem))
    build = "oracle C port (reference library absent)"
    if kind == "reference":
        from oracle.oracle import ref_library
        build = f"GLAC sources compiled as oracle/_ref ({ref_library()[1]})"
    ctx = mp.get_context("spawn")
    barrier, results = ctx.Barrier(procs), ctx.Queue()
    workers = [ctx.Process(target=_cpu_worker, args=((i, kind, dims, nsteps_per_proc, 1000 + i, warm), barrier,
                                                     results)) for i in range(procs)]
    t0 = time.perf_counter()
    for w in workers:
        w.start()
    res = [results.get(timeout=3600) for _ in workers]
    for w in workers:
        w.join()
    wall = time.perf_counter() - t0
    if any(w.exitcode != 0 for w in workers):
        raise RuntimeError("a CPU baseline process failed")
    slowest = max(dt for _, dt in res)
    value = procs * nsteps_per_proc * V / slowest
    sample = (f"{procs} processes x {nsteps_per_proc} step(s) (RK3 flow + MasterSamplerTopcXYZ, eps={FLOW_EPS}) "
              f"on independent {dims[0]}^3x{dims[3]} Haar fields, started together; {build}; "
              f"{cores} cores ({cpu_model()}), process count limited by "
              f"{'host memory' if procs < cores else 'cores'} at {REF_BYTES_PER_SITE * V / 1e9:.1f} GB each")
    return {"value": value, "unit": UNIT, "cores": procs, "kind": kind, "sample": sample,
            "wall_s": round(wall, 2), "timed_s": round(slowest, 2), "per_core": value / procs,
            "lattice_steps": procs * nsteps_per_proc}


def bench_config(world):
    """The workload's config, printed identically by both arms."""
    return {"workload": WORKLOAD, "dims": list(DIMS), "beta": BETA, "flow_eps": FLOW_EPS,
            "l2": "field 604 MB FP32 > 126 MB L2 (no flush needed)", "parallelism": f"replicas x{world}"}


# ---------------------------------------------------------------------------
# distributed plumbing
# ---------------------------------------------------------------------------
def dist_env():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def max_over_ranks(x: float, world: int):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


# ---------------------------------------------------------------------------
# GPU arm
# ---------------------------------------------------------------------------
def run_gpu(args):
    import torch
    world, rank, local = dist_env()
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))

    cpu_base = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cpu_base = cpu_flow_rate(args.cpu_steps)  # before the first GPU call (spawned processes)

    import glac_b200 as g

    V = int(np.prod(DIMS))
    L = g.Lattice(DIMS, beta=BETA, precision="fp32", n_updates=NHITS, su3_eps=SU3_EPS, flow_eps=FLOW_EPS,
                  seed=20261203, stream_id=rank, reunit_interval=0, device=local)
    stream = torch.cuda.ExternalStream(L.stream)

    def timed(fn, n):
        barrier(world)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(n):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        barrier(world)
        return max_over_ranks(e0.elapsed_time(e1) / 1e3, world)

    # start configuration: Haar hot start + 600 Metropolis sweeps (FP32), timed for link-updates/s
    L.hot_start(20261203)
    L.metropolis(5)
    L.reunitarize()
    tuned = L.autotune(8)  # launch variants timed over 8 repetitions each (flow: measured steps)
    acc_holder = {}
    t_metro = timed(lambda: acc_holder.setdefault("a", L.metropolis(1)), 20)
    L.metropolis(THERM_SWEEPS - 25)
    L.reunitarize()
    start = np.empty((4, V, 18))
    L.get_links(start)
    metro_rate = world * 4 * V * 20 / t_metro
    # Metropolis roofline: compulsory traffic of a (mu, parity) sub-sweep per
    # updated link = the link read and written (2), the three other directions'
    # links of both parities (6) and the other parity's mu links (1): 9 x 72 B
    metro_roofline = {"achieved": round(METRO_BYTES_FP32 * metro_rate / world / 1e9, 1), "unit": "GB/s",
                      "algorithmic_bytes_per_link_update": METRO_BYTES_FP32}

    obs_buf = np.empty((args.steps + 1, 3 + DIMS[3]))

    # clocks sampled from the warm-up through the timed region; the summary
    # takes the samples inside the timed region (NVML polls every 2 ms)
    clk = ClockSampler(local)
    clk.start()
    time.sleep(0.5)
    L.flow(args.warmup, measure=True)
    n0 = L.launch_count
    # timed: K RK3 steps, each followed by the observable measurement (device
    # buffer), all K+1 observable vectors copied back at the end
    tw0 = time.perf_counter()
    t_main = timed(lambda: L.flow(args.steps, out=obs_buf), 1)
    clocks = clk.stop(window=(tw0, time.perf_counter()))
    launches = L.launch_count - n0
    value = world * V * args.steps / t_main

    t_noobs = timed(lambda: L.flow(args.steps, measure=False), 1)
    rate_noobs = world * V * args.steps / t_noobs

    # sustained: measured flow steps over about two seconds of continuous load
    # (the GPU reaches its power cap within that time), clocks sampled meanwhile
    clk_s = ClockSampler(local)
    clk_s.start()
    n_sus = max(100, int(2.0 / (t_main / args.steps)))
    t_sus = timed(lambda: L.flow(n_sus, measure=True), 1)
    sustained = {"site_steps_per_s": world * V * n_sus / t_sus, "steps": n_sus, "seconds": t_sus,
                 "clocks": clk_s.stop()}

    # roofline of the flow-stage kernel: CUDA events around each stage launch on
    # the lattice's stream, averaged over reps RK3 steps
    # roofline of the dominant kernel of the timed region: flow stage 0 with the
    # measurement's clover parts (k_flow_stage0_meas); CUDA events around each
    # launch of measured flow steps on the lattice's stream, right after the
    # timed region, with the SM clock sampled meanwhile
    reps = max(3, min(args.steps, 20))
    clk_st = ClockSampler(local)
    clk_st.start()
    time.sleep(0.5)
    reps = max(reps, 100)  # long enough for several clock samples
    stm = np.array(L.flow_stage_times_measured(reps))
    st = np.array(L.flow_stage_times(reps))
    stage_clocks = clk_st.stop()
    hbm_peak, peak_kind = load_peaks()
    alg_bytes = STAGE0_MEAS_BYTES_FP32 * V
    achieved = alg_bytes / float(stm[0]) / 1e9
    roofline = {"bound": "hbm", "achieved": round(achieved, 1), "peak": hbm_peak, "unit": "GB/s",
                "frac": round(achieved / hbm_peak, 4),
                # dram__bytes_read.sum + dram__bytes_write.sum of one ncu capture of
                # this launch at 32^3x64
                "traffic": NCU_TRAFFIC_STAGE0_MEAS_FP32 if DIMS == (32, 32, 32, 64) else None,
                "kernel": "k_flow_stage0_meas_r128<float, morningstar>",
                "algorithmic_bytes_per_launch": alg_bytes, "peak_source": peak_kind,
                "measured_step_ms": {"stage0_with_clover_parts": round(stm[0] * 1e3, 4),
                                     "measurement_combine_and_reduce": round(stm[1] * 1e3, 4),
                                     "stage1": round(stm[2] * 1e3, 4), "stage2": round(stm[3] * 1e3, 4)},
                "unmeasured_stage_ms": [round(x * 1e3, 4) for x in st],
                "stage_ms_how": (f"CUDA events around each launch over {reps} RK3 steps right after the timed "
                                 f"region; SM clock median {stage_clocks.get('sm_mhz')} MHz meanwhile"),
                "binding_unit": "FP32 FMA pipe (see profiles/)"}
    # the binding unit: FP32 FLOP/s of the same launch against the FP32 peak at the
    # median SM clock sampled while it ran (148 SMs x 128 lanes x 2 FLOP per FMA)
    sm_mhz = stage_clocks.get("sm_mhz") or clocks.get("sm_mhz") or 1965.0
    fp32_peak = SM_COUNT * FP32_LANES_PER_SM * 2 * sm_mhz * 1e6 / 1e12
    if FLOPS_PER_SITE_STAGE0_MEAS_FP32:
        fp32_ach = FLOPS_PER_SITE_STAGE0_MEAS_FP32 * V / float(stm[0]) / 1e12
        roofline["fp32_pipe"] = {"achieved": round(fp32_ach, 2), "peak": round(fp32_peak, 2), "unit": "TFLOP/s",
                                 "frac": round(fp32_ach / fp32_peak, 4),
                                 "flops_per_site": FLOPS_PER_SITE_STAGE0_MEAS_FP32,
                                 "peak_basis": f"148 SMs x 128 FP32 lanes x 2 FLOP x {sm_mhz:.0f} MHz (median while timed)"}
    # Metropolis on the same FP32 pipe: its FMA pipe also runs the Philox
    # integer multiplies, so the FLOP fraction understates how busy the pipe is
    metro_fp32 = FLOPS_PER_LINK_UPDATE_METRO_FP32 * metro_rate / world / 1e12
    metro_fp32_pipe = {"achieved": round(metro_fp32, 2), "peak": round(fp32_peak, 2), "unit": "TFLOP/s",
                       "frac": round(metro_fp32 / fp32_peak, 4),
                       "flops_per_link_update": FLOPS_PER_LINK_UPDATE_METRO_FP32,
                       "binding_unit": "FMA pipe (FP32 and Philox IMAD), 62 % busy, issue-bound (ncu)"}
    # the plain stage-0 launch (flow steps without measurement) for comparison
    plain_fp32 = FLOPS_PER_SITE_STAGE0_FP32 * V / float(st[0]) / 1e12
    roofline["unmeasured_stage0"] = {
        "kernel": "k_flow_stage<float, morningstar, stage 0>", "ms": round(st[0] * 1e3, 4),
        "achieved_GBps": round(STAGE_BYTES_FP32[0] * V / float(st[0]) / 1e9, 1),
        "fp32_pipe_frac": round(plain_fp32 / fp32_peak, 4), "flops_per_site": FLOPS_PER_SITE_STAGE0_FP32}

    # FP64 flow for comparison (same field)
    L64 = g.Lattice(DIMS, beta=BETA, precision="fp64", flow_eps=FLOW_EPS, seed=1, stream_id=rank, device=local)
    L64.set_links(start)
    s64 = torch.cuda.ExternalStream(L64.stream)
    L64.flow(2, measure=True)
    k64 = max(3, args.steps // 4)
    barrier(world)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(s64)
    L64.flow(k64, measure=True)
    e1.record(s64)
    torch.cuda.synchronize()
    t64 = max_over_ranks(e0.elapsed_time(e1) / 1e3, world)
    rate64 = world * V * k64 / t64
    # plain FP64 Metropolis (the reference's proposal at su3_eps) on the same field
    L64m = g.Lattice(DIMS, beta=BETA, precision="fp64", n_updates=NHITS, su3_eps=SU3_EPS, seed=20261203,
                     stream_id=rank, device=local)
    L64m.set_links(start)
    s64m = torch.cuda.ExternalStream(L64m.stream)
    L64m.metropolis(2)
    barrier(world)
    torch.cuda.synchronize()
    e0.record(s64m)
    L64m.metropolis(10)
    e1.record(s64m)
    torch.cuda.synchronize()
    metro64_rate = world * 4 * V * 10 / max_over_ranks(e0.elapsed_time(e1) / 1e3, world)
    L64m.close()
    L64.close()

    # end to end through the C ABI: pinned host field in, host observables out
    host_in = torch.from_numpy(start.reshape(-1)).pin_memory()
    obs_e2e = torch.empty(((args.steps + 1) * (3 + DIMS[3]),), dtype=torch.float64).pin_memory()
    barrier(world)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    L.flow_configuration_ptr(host_in.data_ptr(), args.steps, obs_e2e.data_ptr())
    t_e2e = max_over_ranks(time.perf_counter() - t0, world)
    e2e = {"value": world * V * args.steps / t_e2e, "unit": UNIT,
           "h2d_bytes_per_step": int(host_in.numel() * 8 / args.steps),
           "d2h_bytes_per_step": int(obs_e2e.numel() * 8 / args.steps),
           "how": "glac_flow_configuration: H2D of the FP64 host field, K steps with per-step observables, D2H"}
    obs_last = obs_e2e.numpy().reshape(args.steps + 1, -1)[-1]

    # learned proposal spread on this lattice: ESJ data from 100 plain sweeps,
    # training on the GPU, then the learned sampler's link-updates/s
    learned_extra = None
    eff_q_here = EFF_Q_STUDY
    if not args.no_learned:
        from glac_b200 import learned as lp
        feat, esj, plain = lp.collect_esj(L, 100, 10, 64, lp.DEFAULT_GRID, trials=4)
        net, rep = lp.train_proposal(feat, esj, lp.DEFAULT_GRID, steps=1000, batch=8192, lr=2e-3, seed=1,
                                     esj_plain=plain)
        params = net.params
        net.close()
        del feat, esj, plain
        L.set_option("su2_sign_flips", 0)
        L.set_proposal_net(params, float(lp.DEFAULT_GRID[0]), float(lp.DEFAULT_GRID[-1]))
        L.metropolis(2)
        t_l = timed(lambda: L.metropolis(1), 20)
        L.set_proposal_net(None)
        L.set_option("su2_sign_flips", 1)
        # the second factor of the effective-Q ratio: seconds per sweep with the
        # study's measurements (every 100 sweeps: plaquette, then Q and E of a copy
        # flowed to t = 2) for the plain FP64 and the learned FP32 chains
        from glac_b200 import studies
        cfg = dict(studies.TARGET, dims=DIMS, beta=BETA,
                   sweeps_by={"plain_fp64": EFF_Q_SWEEPS_TIMED, "learned_fp32": EFF_Q_SWEEPS_TIMED})
        sweep_s = {}
        for smp in ("plain_fp64", "learned_fp32"):
            ch = studies.q_chain(start, cfg, smp, 100 + rank, params=params)
            sweep_s[smp] = ch["wall_s"] / ch["sweeps"]
        rate_ratio = sweep_s["plain_fp64"] / sweep_s["learned_fp32"]
        d_ratio, d_err = EFF_Q_DIFFUSION_PER_SWEEP_RATIO
        eff_q_here = dict(EFF_Q_STUDY,
                          seconds_per_sweep_with_measurements_here={k: round(v, 6) for k, v in sweep_s.items()},
                          sweeps_timed_per_sampler=EFF_Q_SWEEPS_TIMED,
                          rate_ratio_measured_here=round(rate_ratio, 4),
                          q_diffusion_per_sweep_ratio_from_study=round(d_ratio, 4),
                          ratio_with_rate_measured_here=round(rate_ratio * d_ratio, 3),
                          ratio_with_rate_measured_here_err=round(rate_ratio * d_err, 3))
        learned_extra = {"metropolis_link_updates_per_s_fp32_learned": world * 4 * V * 20 / t_l,
                         "esj_per_link_update_learned": rep["esj_learned"],
                         "esj_per_link_update_plain": rep["esj_plain_reference_proposal"],
                         "esj_gain_learned_vs_plain": rep["gain_vs_plain"],
                         "esj_gain_learned_vs_best_fixed_spread": rep["gain_vs_best_fixed"],
                         "training_rows": rep["rows_train"], "training_seconds": rep["train_seconds"]}

    # batched ensemble: 64 seeded uneven lattices, 100 sweeps + 200 flow steps as one CUDA graph
    ens_extra = None
    if not args.no_ensemble and world == 1:
        from glac_b200 import ensemble as en
        dims_l, betas_l = en.draw_ensemble(20261203, 64)
        with en.Ensemble(dims_l, betas_l, precision="fp32", seed=20261203) as E:
            E.hot_start(20261203)
            tune_e = E.autotune(2)
            E.run(100, 200)  # capture
            _, obs_e, sec_e = E.run(100, 200)
            # the two phases as graphs of their own, for a rate in each unit
            E.run(100, 0)
            _, _, sec_sweeps = E.run(100, 0)
            E.run(0, 200)
            _, _, sec_flow = E.run(0, 200)
            # the whole schedule as one persistent cooperative launch
            E.run_persistent(100, 200)
            _, obs_p, sec_p = E.run_persistent(100, 200)
        sites_e = int(sum(np.prod(d) for d in dims_l))
        ens_extra = {"lattices": 64, "sites": sites_e, "schedule": "100 sweeps + 200 flow steps with observables",
                     "graph_gpu_s": sec_e,
                     "sweeps_graph_gpu_s": sec_sweeps, "link_updates_per_s": 4 * sites_e * 100 / sec_sweeps,
                     "flow_graph_gpu_s": sec_flow, "flow_site_steps_per_s": sites_e * 200 / sec_flow,
                     "persistent_launch_gpu_s": sec_p,
                     "autotune_chosen": tune_e["chosen"], "plaq_after_flow_mean": float(np.mean([o[-1, 0] for o in obs_e]))}

    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": t_main / args.steps * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded Haar + 600 Metropolis sweeps)",
        "config": bench_config(world),
        "roofline": roofline,
        "cpu_baseline": cpu_base,
        "e2e": e2e,
        "gpu_launches": int(launches),
        "clocks": clocks,
        "extra": {
            "flow_site_steps_per_s_no_obs": rate_noobs,
            "flow_sustained": sustained,
            "flow_site_steps_per_s_fp64_with_obs": rate64,
            "metropolis_link_updates_per_s_fp32": metro_rate,
            "metropolis_roofline_fp32": dict(metro_roofline, peak=hbm_peak,
                                             frac=round(metro_roofline["achieved"] / hbm_peak, 4),
                                             fp32_pipe=metro_fp32_pipe),
            "metropolis_link_updates_per_s_fp64": metro64_rate,
            "learned": learned_extra,
            "eff_Q_samples_study": eff_q_here,
            "ensemble_64_uneven": ens_extra,
            "metropolis_acceptance": acc_holder.get("a"),
            "plaq_after_flow": float(obs_last[0]),
            "autotune": tuned,
        },
    }
    if cpu_base:
        line["extra"]["speedup_vs_cpu_baseline"] = value / cpu_base["value"]
    if rank == 0:
        print(json.dumps(line))
    L.close()
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def run_reference(args):
    """The reference's own CPU path on this host's cores at the benchmark's
    lattice (32^3 x 64): one process per core (as many as host memory holds),
    each flowing and measuring its own lattice; every process runs
    max(1, steps // processes) steps, so the run stays within minutes (one
    32^3 x 64 step of the reference takes minutes on one core).  Warm-up: W
    steps of an 8^3 x 16 lattice in every process, untimed."""
    world, rank, _ = dist_env()
    if rank != 0:
        return
    cores = os.cpu_count() or 1
    V = int(np.prod(DIMS))
    avail = host_memory_available()
    procs = max(1, min(cores, int(0.8 * avail // (REF_BYTES_PER_SITE * V)) if avail else cores))
    per_proc = max(1, args.steps // procs)
    base = cpu_flow_rate(per_proc, DIMS, procs, warm=args.warmup)
    value = base["value"]
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": V / value * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded Haar)", "config": bench_config(world),
            "cpu_baseline": {k: base[k] for k in ("value", "unit", "cores", "kind", "sample")},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "lattice_steps_timed": base["lattice_steps"], "timed_s": base["timed_s"], "wall_s": base["wall_s"],
            "ms_per_step_note": "aggregate: 1e3 x sites / value (time per lattice-step of the whole host)"}
    print(json.dumps(line))


def run_profile(args):
    """Small fixed workload for ncu captures and variant timing: hot start, then
    --steps RK3 steps (with per-step observables unless --no-obs) of one lattice."""
    import torch
    import glac_b200 as g
    dims = tuple(int(x) for x in args.dims.split(","))
    if args.profile == "mlp":
        # batched spread inference (the warp routine, or --tune 1 for tcgen05 tiles) over 2M feature rows
        import torch
        from glac_b200 import learned as lp
        n = 1 << 21
        rng = np.random.default_rng(6)
        X = torch.from_numpy(rng.standard_normal((n, 8)).astype(np.float32)).cuda()
        P = np.zeros(g.MLP_NPARAMS, np.float32)
        P[:256] = rng.standard_normal(256) * 0.5
        P[288:1312] = rng.standard_normal(1024) * 0.25
        P[1344:1376] = rng.standard_normal(32) * 0.3
        with lp.ProposalNet() as net:
            net.params = P
            net.set_forward_mode(int(args.tune or 0))
            for _ in range(max(args.steps, 1)):
                net.forward(X, 0.03, 0.9)
            if args.time_reps:
                torch.cuda.synchronize()
                t0 = time.perf_counter()
                for _ in range(args.time_reps):
                    net.forward(X, 0.03, 0.9)
                sec = (time.perf_counter() - t0) / args.time_reps
                print(json.dumps({"profile": "mlp", "rows": n, "mode": int(args.tune or 0), "ms": sec * 1e3,
                                  "rows_per_s": n / sec, "tflops": n * 2 * (16 * 32 + 32 * 32 + 32 * 16) / sec / 1e12}))
        return
    if args.profile == "ensemble":
        # the seeded uneven ensemble, args.steps sweeps + args.steps flow steps eagerly
        from glac_b200 import ensemble as en
        dl, bl = en.draw_ensemble(20261203, args.ensemble_n)
        with en.Ensemble(dl, bl, precision=args.precision, seed=5) as E:
            E.hot_start(7)
            if args.tune:
                E.tuning = [int(x) for x in args.tune.split(",")]
            E.metropolis(args.steps)
            E.flow(args.steps)
        return
    L = g.Lattice(dims, beta=BETA, precision=args.precision, flow_eps=FLOW_EPS, seed=5, device=0)
    L.hot_start(7)
    if args.fused >= 0:
        L.set_option("fused_measure", int(args.fused))
    L.set_option("fused_combine", int(args.fused_combine))
    if args.tune:
        L.tuning = [int(x) for x in args.tune.split(",")]
    if args.profile == "learned":
        # the learned sampler with a fixed random network (spread varying per link)
        rng = np.random.default_rng(6)
        P = np.zeros(g.MLP_NPARAMS, np.float32)
        P[:256] = rng.standard_normal(256) * 0.5
        P[288:1312] = rng.standard_normal(1024) * 0.25
        P[1344:1376] = rng.standard_normal(32) * 0.3
        L.set_option("su2_sign_flips", 0)
        L.set_proposal_net(P, 0.1, 0.6)
    if args.profile in ("metropolis", "learned"):
        L.metropolis(args.steps)
    else:
        L.flow(args.steps, measure=not args.no_obs)
    L.sync()
    V = int(np.prod(dims))
    if args.time_reps:
        st = torch.cuda.ExternalStream(L.stream)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        if args.profile in ("metropolis", "learned"):
            L.metropolis(args.time_reps)
        else:
            L.flow(args.time_reps, measure=not args.no_obs)
        e1.record(st)
        torch.cuda.synchronize()
        sec = e0.elapsed_time(e1) / 1e3 / args.time_reps
        stages = L.flow_stage_times(5) if args.profile == "flow" else None
        print(json.dumps({"profile": args.profile, "dims": dims, "precision": args.precision, "tune": L.tuning,
                          "fused_measure": int(args.fused), "fused_combine": int(args.fused_combine),
                          "ms_per_step": sec * 1e3,
                          "rate": (4 * V if args.profile in ("metropolis", "learned") else V) / sec,
                          "stage_ms": None if stages is None else [x * 1e3 for x in stages]}))
    L.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=300)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--cpu-steps", type=int, default=1, help="32^3x64 steps per process of the CPU baseline")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-learned", action="store_true", help="skip the learned-proposal leg")
    ap.add_argument("--no-ensemble", action="store_true", help="skip the 64-lattice ensemble leg")
    ap.add_argument("--profile", choices=["flow", "metropolis", "learned", "ensemble", "mlp"],
                    help="small workload for ncu / variant timing")
    ap.add_argument("--ensemble-n", type=int, default=16, help="lattices in the ensemble profile")
    ap.add_argument("--dims", default="32,32,32,64")
    ap.add_argument("--precision", default="fp32")
    ap.add_argument("--no-obs", action="store_true")
    ap.add_argument("--time-reps", type=int, default=0)
    ap.add_argument("--fused", type=int, default=-1,
                    help="profile mode: measurement inside flow stage 0 (1: uncapped kernel, 2: 128-register kernel) "
                         "or a pass of its own (0); default: the library's choice per precision")
    ap.add_argument("--fused-combine", type=int, default=1, help="profile mode: its reduction inside stage 1 (1) or not (0)")
    ap.add_argument("--tune", default="", help="launch variants flow,metropolis,observables (profile mode)")
    args = ap.parse_args()
    if args.profile:
        run_profile(args)
        return
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    else:
        run_gpu(args)


if __name__ == "__main__":
    main()
