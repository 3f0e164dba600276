"""Batched ensemble of independent lattices (glac_ensemble_* in include/glac_b200.h).

Many lattices of uneven sizes and couplings advance together: one launch per
Metropolis sub-sweep, flow stage and observable pass covers all of them, and
``Ensemble.run`` replays the whole schedule (sweeps, then the flow with a
measurement after every step) as one CUDA graph.

``draw_ensemble(seed)`` is the seeded draw of the 64-lattice workload: sizes
uniformly from {8^3x16, 12^3x24, 16^3x32, 24^3x48}, couplings uniformly from
{6.0, 6.1, 6.2, 6.45}.  ``python -m glac_b200.ensemble`` times that workload
(100 sweeps + 200 flow steps) as one graph, eagerly, and as one context per
lattice.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import time

import numpy as np

from . import EXP_FUNCS, PRECISIONS, GlacError, Lattice, _Desc, lib

SIZES = ((8, 8, 8, 16), (12, 12, 12, 24), (16, 16, 16, 32), (24, 24, 24, 48))
BETAS = (6.0, 6.1, 6.2, 6.45)


def draw_ensemble(seed: int = 20261203, n: int = 64):
    """(dims list, betas list) of the seeded uneven ensemble."""
    rng = np.random.default_rng(seed)
    si = rng.integers(0, len(SIZES), n)
    bi = rng.integers(0, len(BETAS), n)
    return [SIZES[k] for k in si], [BETAS[k] for k in bi]


def _bind(L):
    P = C.c_void_p
    L.glac_ensemble_create.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.POINTER(_Desc), C.POINTER(P)]
    L.glac_ensemble_destroy.argtypes = [P]
    L.glac_ensemble_destroy.restype = None
    L.glac_ensemble_last_error.argtypes = [P]
    L.glac_ensemble_last_error.restype = C.c_char_p
    L.glac_ensemble_global_error.restype = C.c_char_p
    L.glac_ensemble_launch_count.argtypes = [P]
    L.glac_ensemble_launch_count.restype = C.c_uint64
    L.glac_ensemble_set_option.argtypes = [P, C.c_char_p, C.c_long]
    L.glac_ensemble_hot_start.argtypes = [P, C.c_uint64]
    L.glac_ensemble_set_links.argtypes = [P, C.c_int, C.c_void_p]
    L.glac_ensemble_get_links.argtypes = [P, C.c_int, C.c_void_p]
    L.glac_ensemble_metropolis.argtypes = [P, C.c_int, C.c_void_p]
    L.glac_ensemble_obs_count.argtypes = [P, C.c_int]
    L.glac_ensemble_obs_count.restype = C.c_longlong
    L.glac_ensemble_flow.argtypes = [P, C.c_int, C.c_void_p]
    L.glac_ensemble_run.argtypes = [P, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.POINTER(C.c_double)]
    L.glac_ensemble_run_persistent.argtypes = [P, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.POINTER(C.c_double)]
    L.glac_ensemble_autotune.argtypes = [P, C.c_int, C.c_void_p]
    L.glac_ensemble_get_tuning.argtypes = [P, C.c_void_p]
    L.glac_ensemble_set_tuning.argtypes = [P, C.c_void_p]
    return L


class Ensemble:
    """Independent lattices advanced together on one GPU."""

    def __init__(self, dims_list, betas, precision="fp32", n_updates=10, su3_eps=0.24, flow_eps=0.01, seed=1,
                 stream_id=0, device=0):
        L = _bind(lib())
        self.dims = [tuple(int(x) for x in d) for d in dims_list]
        self.betas = [float(b) for b in betas]
        if len(self.dims) != len(self.betas):
            raise ValueError("one beta per lattice")
        d = _Desc()
        d.dims = (C.c_int * 4)(4, 4, 4, 4)
        d.beta = 6.0
        d.precision = PRECISIONS[precision] if isinstance(precision, str) else int(precision)
        d.n_updates = int(n_updates)
        d.su3_eps = float(su3_eps)
        d.flow_eps = float(flow_eps)
        d.exp_func = EXP_FUNCS["morningstar"]
        d.seed = int(seed) & 0xFFFFFFFFFFFFFFFF
        d.stream_id = int(stream_id) & 0xFFFFFFFF
        d.reunit_interval = 0
        d.device = int(device)
        dims = np.ascontiguousarray(np.array(self.dims, np.int32).reshape(-1))
        betas_a = np.ascontiguousarray(self.betas, np.float64)
        self._h = C.c_void_p()
        st = L.glac_ensemble_create(len(self.dims), dims.ctypes.data, betas_a.ctypes.data, C.byref(d),
                                    C.byref(self._h))
        if st != 0:
            raise GlacError(st, L.glac_ensemble_global_error().decode())
        self.n = len(self.dims)
        self.V = [int(np.prod(x)) for x in self.dims]

    def _ck(self, st):
        if st != 0:
            raise GlacError(st, lib().glac_ensemble_last_error(self._h).decode())

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            lib().glac_ensemble_destroy(self._h)
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

    @property
    def launch_count(self) -> int:
        return int(lib().glac_ensemble_launch_count(self._h))

    def set_option(self, key, value):
        self._ck(lib().glac_ensemble_set_option(self._h, key.encode(), int(value)))

    def hot_start(self, seed):
        self._ck(lib().glac_ensemble_hot_start(self._h, int(seed)))

    def set_links(self, i, links):
        i = self._index(i)
        a = np.ascontiguousarray(links, np.float64)
        if a.size != 4 * self.V[i] * 18:
            raise ValueError("field size")
        self._ck(lib().glac_ensemble_set_links(self._h, int(i), a.ctypes.data))

    def _index(self, i):
        if not 0 <= int(i) < self.n:
            raise GlacError(1, f"lattice index {i} out of range (ensemble of {self.n})")
        return int(i)

    def get_links(self, i):
        i = self._index(i)
        a = np.empty((4, self.V[i], 18))
        self._ck(lib().glac_ensemble_get_links(self._h, int(i), a.ctypes.data))
        return a

    def metropolis(self, n_sweeps):
        acc = np.empty(self.n)
        self._ck(lib().glac_ensemble_metropolis(self._h, int(n_sweeps), acc.ctypes.data))
        return acc

    def _split(self, flat, n_steps):
        out, o = [], 0
        for d in self.dims:
            k = (n_steps + 1) * (3 + d[3])
            out.append(flat[o:o + k].reshape(n_steps + 1, 3 + d[3]))
            o += k
        return out

    def flow(self, n_steps):
        """Per lattice: (n_steps + 1, 3 + Nt) measurements of a flowed copy of the chain."""
        flat = np.empty(lib().glac_ensemble_obs_count(self._h, int(n_steps)))
        self._ck(lib().glac_ensemble_flow(self._h, int(n_steps), flat.ctypes.data))
        return self._split(flat, n_steps)

    def run(self, n_sweeps, n_steps):
        """Sweeps then flow as one CUDA graph: (acceptance, per-lattice measurements, GPU seconds)."""
        acc = np.empty(self.n)
        flat = np.empty(lib().glac_ensemble_obs_count(self._h, int(n_steps)))
        sec = C.c_double(0.0)
        self._ck(lib().glac_ensemble_run(self._h, int(n_sweeps), int(n_steps), acc.ctypes.data, flat.ctypes.data,
                                         C.byref(sec)))
        return acc, self._split(flat, n_steps), sec.value

    def run_persistent(self, n_sweeps, n_steps):
        """The same schedule as run(), as one persistent cooperative launch (FP32):
        (acceptance, per-lattice measurements, GPU seconds)."""
        acc = np.empty(self.n)
        flat = np.empty(lib().glac_ensemble_obs_count(self._h, int(n_steps)))
        sec = C.c_double(0.0)
        self._ck(lib().glac_ensemble_run_persistent(self._h, int(n_sweeps), int(n_steps), acc.ctypes.data,
                                                    flat.ctypes.data, C.byref(sec)))
        return acc, self._split(flat, n_steps), sec.value

    def autotune(self, reps=2):
        rep = np.zeros(12)
        self._ck(lib().glac_ensemble_autotune(self._h, int(reps), rep.ctypes.data))
        return {"flow": rep[0:4].tolist(), "metropolis": rep[4:8].tolist(), "observables": rep[8:12].tolist(),
                "chosen": self.tuning}

    @property
    def tuning(self):
        v = (C.c_int * 3)()
        self._ck(lib().glac_ensemble_get_tuning(self._h, v))
        return list(v)

    @tuning.setter
    def tuning(self, v):
        self._ck(lib().glac_ensemble_set_tuning(self._h, (C.c_int * 3)(*[int(x) for x in v])))


def timing_study(seed=20261203, n=64, sweeps=100, steps=200, precision="fp32", separate=True):
    """Seconds for the ensemble workload as one graph, eagerly, and (optionally) one context per lattice."""
    dims, betas = draw_ensemble(seed, n)
    out = dict(n=n, sites=int(sum(np.prod(d) for d in dims)), sweeps=sweeps, steps=steps, precision=precision,
               sizes={str(s): int(sum(1 for d in dims if d == s)) for s in SIZES},
               betas={str(b): int(sum(1 for x in betas if x == b)) for b in BETAS})
    with Ensemble(dims, betas, precision=precision, seed=seed) as E:
        E.hot_start(seed)
        out["autotune"] = E.autotune(2)
        E.run(sweeps, steps)  # capture + warm-up
        acc, obs, gpu_s = E.run(sweeps, steps)
        t0 = time.perf_counter()
        E.metropolis(sweeps)
        E.flow(steps)
        out["eager_wall_s"] = time.perf_counter() - t0
        out["graph_gpu_s"] = gpu_s
        out["acceptance_mean"] = float(acc.mean())
        out["plaq_after_flow_mean"] = float(np.mean([o[-1, 0] for o in obs]))
    if separate:
        ctxs = []
        for i, (d, b) in enumerate(zip(dims, betas)):
            L = Lattice(d, beta=b, precision=precision, seed=seed, stream_id=i)
            L.hot_start(seed)
            ctxs.append(L)
        for L in ctxs:
            L.sync()
        t0 = time.perf_counter()
        for L in ctxs:  # one lattice after another, as separate jobs on one GPU would run
            L.metropolis(sweeps)
            L.flow(steps)
        for L in ctxs:
            L.sync()
        out["separate_wall_s"] = time.perf_counter() - t0
        for L in ctxs:
            L.close()
    units = out["sites"] * (4 * sweeps + steps)
    out["graph_site_units_per_s"] = units / out["graph_gpu_s"]
    return out


def _main():
    ap = argparse.ArgumentParser(prog="python -m glac_b200.ensemble")
    ap.add_argument("--n", type=int, default=64)
    ap.add_argument("--sweeps", type=int, default=100)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--precision", default="fp32")
    ap.add_argument("--no-separate", action="store_true")
    a = ap.parse_args()
    print(json.dumps(timing_study(n=a.n, sweeps=a.sweeps, steps=a.steps, precision=a.precision,
                                  separate=not a.no_separate)))


if __name__ == "__main__":
    _main()
