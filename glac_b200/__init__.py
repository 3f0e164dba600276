"""glac_b200 -- B200 (sm_100a) implementation of GLAC's pure-gauge SU(3) hot path.

This module is the Python binding of the C ABI in ``include/glac_b200.h``
(library ``glac_b200/libglac_b200.so``).  There is no CPU fallback: if the
library is missing or no CUDA device is usable, every call raises.

Field layout on the host: float64 array of shape (4, V, 18) -- for each
direction mu the V SU(3) matrices (18 doubles, re/im row-major) in the
reference's site order x + Nx(y + Ny(z + Nz t)) (GLAC/math/lattice.h,
GLAC/parallelization/index.h:32-35).
Observable vectors: [plaq, topc, energy, topct[0..Nt-1]]
(GLAC/observables/mastersamplertopcxyz.cpp:223-234).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libglac_b200.so")

GLAC_OK, GLAC_ERR_ARG, GLAC_ERR_CUDA, GLAC_ERR_TIMEOUT, GLAC_ERR_NONFINITE, GLAC_ERR_IO, GLAC_ERR_STATE = range(7)
FP64, FP32 = 0, 1
EXP_FUNCS = {"morningstar": 0, "luscher": 1, "taylor2": 2, "taylor4": 3}
PRECISIONS = {"fp64": FP64, "fp32": FP32, "double": FP64, "float": FP32}


MLP_NPARAMS = 1377  # GLAC_MLP_NPARAMS


class GlacError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"glac status {status}: {message}")
        self.status = status


class _Desc(C.Structure):
    _fields_ = [
        ("dims", C.c_int * 4),
        ("beta", C.c_double),
        ("precision", C.c_int),
        ("n_updates", C.c_int),
        ("su3_eps", C.c_double),
        ("flow_eps", C.c_double),
        ("exp_func", C.c_int),
        ("seed", C.c_uint64),
        ("stream_id", C.c_uint32),
        ("reunit_interval", C.c_int),
        ("device", C.c_int),
    ]


_lib = None
_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_u8 = np.ctypeslib.ndpointer(dtype=np.uint8, flags="C_CONTIGUOUS")


def build(force: bool = False) -> str:
    """Compile libglac_b200.so for sm_100a in place (nvcc; no GPU needed)."""
    args = ["make", "-s", "-C", HERE, "-j4"]
    if force:
        subprocess.run(["make", "-s", "-C", HERE, "clean"], check=True)
    subprocess.run(args, check=True)
    return LIB_PATH


def lib() -> C.CDLL:
    """The loaded C ABI library (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"{LIB_PATH} is missing: run glac_b200.build() (or `make -C glac_b200`)")
    L = C.CDLL(LIB_PATH)
    P = C.c_void_p
    L.glac_create.argtypes = [C.POINTER(_Desc), C.POINTER(P)]
    L.glac_destroy.argtypes = [P]
    L.glac_destroy.restype = None
    L.glac_last_error.argtypes = [P]
    L.glac_last_error.restype = C.c_char_p
    L.glac_global_error.restype = C.c_char_p
    L.glac_io_error.restype = C.c_char_p
    L.glac_stream.argtypes = [P]
    L.glac_stream.restype = C.c_void_p
    L.glac_sync.argtypes = [P]
    L.glac_launch_count.argtypes = [P]
    L.glac_launch_count.restype = C.c_uint64
    L.glac_set_option.argtypes = [P, C.c_char_p, C.c_long]
    L.glac_cold_start.argtypes = [P]
    L.glac_hot_start.argtypes = [P, C.c_uint64]
    L.glac_set_links.argtypes = [P, C.c_void_p]
    L.glac_get_links.argtypes = [P, C.c_void_p]
    L.glac_set_links_device.argtypes = [P, C.c_void_p]
    L.glac_get_links_device.argtypes = [P, C.c_void_p]
    L.glac_reunitarize.argtypes = [P]
    L.glac_unitarity_violation.argtypes = [P, C.POINTER(C.c_double)]
    L.glac_metropolis.argtypes = [P, C.c_int, C.POINTER(C.c_double)]
    L.glac_flow.argtypes = [P, C.c_int, C.c_void_p]
    L.glac_measure.argtypes = [P, C.c_void_p]
    L.glac_flow_configuration.argtypes = [P, C.c_void_p, C.c_int, C.c_void_p]
    L.glac_flow_stage_times.argtypes = [P, C.c_int, _dp]
    L.glac_flow_stage_times_measured.argtypes = [P, C.c_int, _dp]
    L.glac_autotune.argtypes = [P, C.c_int, C.c_void_p]
    L.glac_get_tuning.argtypes = [P, C.c_void_p]
    L.glac_set_tuning.argtypes = [P, C.c_void_p]
    L.glac_staples.argtypes = [P, _dp]
    L.glac_force.argtypes = [P, _dp]
    L.glac_exp_batch.argtypes = [C.c_int, C.c_int, _dp, C.c_long, _dp]
    L.glac_delta_s_batch.argtypes = [C.c_int, C.c_double, C.c_long, _dp, _dp, _dp, _dp]
    L.glac_accept_fed.argtypes = [C.c_int, C.c_double, C.c_long, C.c_int, _dp, _dp, _dp, _dp, _u8]
    L.glac_read_field.argtypes = [C.c_char_p, C.c_int * 4, C.c_int, _dp]
    L.glac_write_field.argtypes = [C.c_char_p, C.c_int * 4, _dp]
    # learned proposal spread
    L.glac_copy_field.argtypes = [P, P]
    L.glac_measure_density.argtypes = [P, C.c_void_p, C.c_void_p, C.c_void_p]
    L.glac_measure_weinberg.argtypes = [P, C.c_void_p]
    L.glac_get_sweep.argtypes = [P, C.POINTER(C.c_uint32)]
    L.glac_set_sweep.argtypes = [P, C.c_uint32]
    L.glac_set_proposal_net.argtypes = [P, C.c_void_p, C.c_double, C.c_double]
    L.glac_esj_data.argtypes = [P, C.c_int, _dp, C.c_int, C.c_int, C.c_uint32, C.c_void_p, C.c_void_p, C.c_void_p,
                                C.c_longlong, C.POINTER(C.c_longlong)]
    L.glac_mlp_create.argtypes = [C.c_int, C.POINTER(P)]
    L.glac_mlp_destroy.argtypes = [P]
    L.glac_mlp_destroy.restype = None
    L.glac_mlp_last_error.argtypes = [P]
    L.glac_mlp_last_error.restype = C.c_char_p
    L.glac_mlp_set_params.argtypes = [P, C.c_void_p]
    L.glac_mlp_get_params.argtypes = [P, C.c_void_p]
    L.glac_mlp_init.argtypes = [P, C.c_uint64, C.c_double, C.c_double, C.c_double]
    L.glac_mlp_forward.argtypes = [P, C.c_void_p, C.c_longlong, C.c_double, C.c_double, C.c_void_p]
    L.glac_mlp_set_forward_mode.argtypes = [P, C.c_int]
    L.glac_mlp_test_tc_wait.argtypes = [P, C.c_ulonglong, C.c_int]
    L.glac_mlp_loss_grad.argtypes = [P, C.c_void_p, C.c_void_p, C.c_longlong, C.c_int, _dp,
                                     C.POINTER(C.c_double), C.c_void_p]
    L.glac_mlp_train.argtypes = [P, C.c_void_p, C.c_void_p, C.c_longlong, C.c_int, _dp, C.c_int, C.c_longlong,
                                 C.c_double, C.c_void_p]
    _lib = L
    return L


def _check_global(status: int) -> None:
    if status != GLAC_OK:
        raise GlacError(status, lib().glac_global_error().decode())


def _as_field(links, V):
    a = np.ascontiguousarray(links, dtype=np.float64)
    if a.size != 4 * V * 18:
        raise ValueError(f"field must hold 4*V*18 = {4 * V * 18} doubles, got {a.size}")
    return a


class Lattice:
    """One lattice on one GPU: the device state behind the reference's
    System / Flow / Correlator objects (GLAC/system.h, GLAC/flow/flow.h,
    GLAC/observables/correlator.h)."""

    def __init__(self, dims, beta=6.0, precision="fp64", n_updates=10, su3_eps=0.24, flow_eps=0.01,
                 exp_func="morningstar", seed=1, stream_id=0, reunit_interval=0, device=0):
        L = lib()
        d = _Desc()
        dims = [int(x) for x in (dims if len(dims) == 4 else (dims[0],) * 3 + (dims[1],))]
        d.dims = (C.c_int * 4)(*dims)
        d.beta = float(beta)
        d.precision = PRECISIONS[precision] if isinstance(precision, str) else int(precision)
        d.n_updates = int(n_updates)
        d.su3_eps = float(su3_eps)
        d.flow_eps = float(flow_eps)
        d.exp_func = EXP_FUNCS[exp_func] if isinstance(exp_func, str) else int(exp_func)
        d.seed = int(seed) & 0xFFFFFFFFFFFFFFFF
        d.stream_id = int(stream_id) & 0xFFFFFFFF
        d.reunit_interval = int(reunit_interval)
        d.device = int(device)
        self._desc = d
        self._ctx = C.c_void_p()
        _check_global(L.glac_create(C.byref(d), C.byref(self._ctx)))
        self.dims = tuple(dims)
        self.V = int(np.prod(dims))
        self.Nt = dims[3]
        self.precision = d.precision
        self.beta = float(beta)
        self.flow_eps = float(flow_eps)

    # -- plumbing --------------------------------------------------------
    def _ck(self, status):
        if status != GLAC_OK:
            raise GlacError(status, lib().glac_last_error(self._ctx).decode())

    def close(self):
        if getattr(self, "_ctx", None) and self._ctx.value:
            lib().glac_destroy(self._ctx)
            self._ctx = C.c_void_p()

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
    def stream(self) -> int:
        """cudaStream_t of this lattice (for torch.cuda.ExternalStream)."""
        return lib().glac_stream(self._ctx) or 0

    @property
    def launch_count(self) -> int:
        return int(lib().glac_launch_count(self._ctx))

    def sync(self):
        self._ck(lib().glac_sync(self._ctx))

    def set_option(self, key: str, value: int):
        self._ck(lib().glac_set_option(self._ctx, key.encode(), int(value)))

    # -- field -------------------------------------------------------------
    def cold_start(self):
        self._ck(lib().glac_cold_start(self._ctx))

    def hot_start(self, seed: int):
        self._ck(lib().glac_hot_start(self._ctx, int(seed) & 0xFFFFFFFFFFFFFFFF))

    def set_links(self, links):
        a = _as_field(links, self.V)
        self._ck(lib().glac_set_links(self._ctx, a.ctypes.data))

    def get_links(self, out=None):
        if out is None:
            out = np.empty((4, self.V, 18), np.float64)
        self._ck(lib().glac_get_links(self._ctx, out.ctypes.data))
        return out

    def set_links_ptr(self, host_ptr: int):
        """Host pointer variant (e.g. a pinned torch tensor's data_ptr())."""
        self._ck(lib().glac_set_links(self._ctx, C.c_void_p(host_ptr)))

    def set_links_device(self, dev_ptr: int):
        self._ck(lib().glac_set_links_device(self._ctx, C.c_void_p(dev_ptr)))

    def get_links_device(self, dev_ptr: int):
        self._ck(lib().glac_get_links_device(self._ctx, C.c_void_p(dev_ptr)))

    def reunitarize(self):
        self._ck(lib().glac_reunitarize(self._ctx))

    def unitarity_violation(self) -> float:
        v = C.c_double()
        self._ck(lib().glac_unitarity_violation(self._ctx, C.byref(v)))
        return v.value

    # -- hot path ------------------------------------------------------------
    def metropolis(self, n_sweeps: int) -> float:
        acc = C.c_double()
        self._ck(lib().glac_metropolis(self._ctx, int(n_sweeps), C.byref(acc)))
        return acc.value

    def flow(self, n_steps: int, measure: bool = True, out=None):
        if not measure:
            self._ck(lib().glac_flow(self._ctx, int(n_steps), None))
            return None
        if out is None:
            out = np.empty((n_steps + 1, 3 + self.Nt), np.float64)
        self._ck(lib().glac_flow(self._ctx, int(n_steps), out.ctypes.data))
        return out

    def autotune(self, reps: int = 3):
        """Pick the fastest launch variant of each kernel family on this lattice;
        returns the timing table {family: [seconds per call per variant]}."""
        rep = np.zeros(12)
        self._ck(lib().glac_autotune(self._ctx, int(reps), rep.ctypes.data))
        rep = rep.reshape(3, 4)
        return {"flow": rep[0].tolist(), "metropolis": rep[1].tolist(), "observables": rep[2].tolist(),
                "chosen": self.tuning}

    @property
    def tuning(self):
        v = np.zeros(3, np.int32)
        self._ck(lib().glac_get_tuning(self._ctx, v.ctypes.data))
        return v.tolist()

    @tuning.setter
    def tuning(self, variants):
        v = np.ascontiguousarray(variants, np.int32)
        self._ck(lib().glac_set_tuning(self._ctx, v.ctypes.data))

    def flow_stage_times(self, n_steps: int):
        out = np.zeros(3)
        self._ck(lib().glac_flow_stage_times(self._ctx, int(n_steps), out))
        return out

    def flow_stage_times_measured(self, n_steps: int):
        """Seconds per launch of [stage 0 with the clover parts, the measurement's
        reduction, stage 1, stage 2] over n_steps measured flow steps."""
        out = np.zeros(4)
        self._ck(lib().glac_flow_stage_times_measured(self._ctx, int(n_steps), out))
        return out

    def flow_configuration_ptr(self, host_ptr: int, n_steps: int, obs_ptr: int):
        self._ck(lib().glac_flow_configuration(self._ctx, C.c_void_p(host_ptr), int(n_steps), C.c_void_p(obs_ptr)))

    def measure(self, out=None):
        if out is None:
            out = np.empty(3 + self.Nt, np.float64)
        self._ck(lib().glac_measure(self._ctx, out.ctypes.data))
        return out

    def measure_ptr(self, host_ptr: int):
        self._ck(lib().glac_measure(self._ctx, C.c_void_p(host_ptr)))

    # -- test exports ----------------------------------------------------------
    def staples(self):
        out = np.empty((4, self.V, 18), np.float64)
        self._ck(lib().glac_staples(self._ctx, out))
        return out

    def set_proposal_net(self, params=None, eps_min=0.0, eps_max=1.0):
        """Learned proposal spread from now on (params: GLAC_MLP_NPARAMS floats), or None for su3_eps."""
        if params is None:
            self._ck(lib().glac_set_proposal_net(self._ctx, None, 0.0, 0.0))
            return
        p = np.ascontiguousarray(params, np.float32)
        if p.size != MLP_NPARAMS:
            raise ValueError(f"need {MLP_NPARAMS} parameters")
        self._ck(lib().glac_set_proposal_net(self._ctx, p.ctypes.data, float(eps_min), float(eps_max)))

    def esj_data_ptr(self, eps_grid, trials, stride, snapshot, feat_ptr, esj_ptr, ids_ptr, capacity) -> int:
        """Expected-squared-jump rows into device buffers (pointers); returns the row count."""
        g = np.ascontiguousarray(eps_grid, np.float64)
        n = C.c_longlong(0)
        self._ck(lib().glac_esj_data(self._ctx, g.size, g, int(trials), int(stride), int(snapshot), feat_ptr,
                                     esj_ptr if g.size else None, ids_ptr, int(capacity), C.byref(n)))
        return n.value

    def measure_density(self):
        """(observables, q density, e density): per-site fields of length V in the host site order."""
        obs = np.empty(3 + self.Nt)
        q, e = np.empty(self.V), np.empty(self.V)
        self._ck(lib().glac_measure_density(self._ctx, obs.ctypes.data, q.ctypes.data, e.ctypes.data))
        return obs, q, e

    def measure_weinberg(self):
        """SuperSampler observables: [plaq, topc, energy, weinberg, topct[Nt], weinbergt[Nt]]."""
        out = np.empty(4 + 2 * self.Nt)
        self._ck(lib().glac_measure_weinberg(self._ctx, out.ctypes.data))
        return out

    @property
    def sweep(self) -> int:
        """Philox sweep counter (advanced by every Metropolis sweep)."""
        v = C.c_uint32(0)
        self._ck(lib().glac_get_sweep(self._ctx, C.byref(v)))
        return v.value

    @sweep.setter
    def sweep(self, v: int):
        self._ck(lib().glac_set_sweep(self._ctx, int(v)))

    def copy_from(self, other: "Lattice"):
        """Device copy of another context's field (same dimensions and precision)."""
        self._ck(lib().glac_copy_field(self._ctx, other._ctx))

    def esj_rows(self, stride) -> int:
        return 8 * ((self.V // 2) // int(stride))

    def force(self):
        out = np.empty((4, self.V, 18), np.float64)
        self._ck(lib().glac_force(self._ctx, out))
        return out


def exp_batch(mats, precision="fp64", exp_func="morningstar"):
    """Device exponential of traceless anti-Hermitian 3x3 matrices (18 doubles each)."""
    m = np.ascontiguousarray(mats, np.float64).reshape(-1, 18)
    out = np.empty_like(m)
    p = PRECISIONS[precision] if isinstance(precision, str) else int(precision)
    k = EXP_FUNCS[exp_func] if isinstance(exp_func, str) else int(exp_func)
    _check_global(lib().glac_exp_batch(p, k, m, m.shape[0], out))
    return out.reshape(np.shape(mats))


def delta_s_batch(U, Up, A, beta, precision="fp64"):
    """Device dS = -(beta/3) ReTr[(U' - U) A] for n triples of matrices."""
    U = np.ascontiguousarray(U, np.float64).reshape(-1, 18)
    out = np.empty(U.shape[0], np.float64)
    p = PRECISIONS[precision] if isinstance(precision, str) else int(precision)
    _check_global(lib().glac_delta_s_batch(p, float(beta), U.shape[0], U,
                                           np.ascontiguousarray(Up, np.float64).reshape(-1, 18),
                                           np.ascontiguousarray(A, np.float64).reshape(-1, 18), out))
    return out


def accept_fed(U, A, X, r, beta, precision="fp64"):
    """Metropolis accept step on the device with given proposals and uniforms."""
    U = np.array(U, np.float64, copy=True, order="C").reshape(-1, 18)
    nl = U.shape[0]
    r = np.ascontiguousarray(r, np.float64).reshape(nl, -1)
    nh = r.shape[1]
    acc = np.zeros(nl * nh, np.uint8)
    p = PRECISIONS[precision] if isinstance(precision, str) else int(precision)
    _check_global(lib().glac_accept_fed(p, float(beta), nl, nh, U, np.ascontiguousarray(A, np.float64),
                                        np.ascontiguousarray(X, np.float64), r, acc))
    return U, acc.reshape(nl, nh)


def read_field(path, dims, chroma=False):
    """GLAC .bin (or Chroma byte-swapped) configuration -> (4, V, 18) array."""
    V = int(np.prod(dims))
    out = np.empty((4, V, 18), np.float64)
    st = lib().glac_read_field(os.fsencode(path), (C.c_int * 4)(*dims), int(chroma), out)
    if st != GLAC_OK:
        raise GlacError(st, lib().glac_io_error().decode())
    return out


def write_field(path, dims, links):
    V = int(np.prod(dims))
    a = _as_field(links, V).reshape(4, V, 18)
    st = lib().glac_write_field(os.fsencode(path), (C.c_int * 4)(*dims), a)
    if st != GLAC_OK:
        raise GlacError(st, lib().glac_io_error().decode())


__all__ = [
    "Lattice", "exp_batch", "delta_s_batch", "accept_fed", "read_field", "write_field", "build", "lib", "GlacError",
]
