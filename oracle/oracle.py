"""ctypes access to the two CPU checkers.

TEST INFRASTRUCTURE ONLY: imported by tests/, ``__graft_entry__.smoke()`` and
the CPU-baseline leg of ``bench.py``.  The product (``glac_b200``) never
imports this module.

* :class:`Oracle` -- the project's C restatement (``oracle/liboracle.so``,
  source ``oracle/glac_oracle.c``), always available once built.
* :class:`Reference` -- the reference GLAC sources compiled into
  ``oracle/_ref/libglacref.so`` (portable, -march=x86-64-v3) and
  ``oracle/_ref/native/libglacref.so`` (the reference's own -O3 -march=native,
  for the CPU that built it; used only on a host whose ISA flags include that
  CPU's, see :func:`ref_library`).  Recipe ``oracle/Makefile``.  Built only
  where the reference tree exists ($GLAC_REF_SRC, default ../reference/GLAC
  beside the repository); the prebuilt libraries travel with the repository
  copy to other machines.

Field layout for every call: float64 array of shape (4, V, 18), sites in
lexicographic order x + Nx(y + Ny(z + Nz t)) (GLAC/parallelization/index.h:32-35).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libglacref.so")
REF_NATIVE_SO = os.path.join(HERE, "_ref", "native", "libglacref.so")
REF_NATIVE_FLAGS = os.path.join(HERE, "_ref", "native", "cpu_flags.txt")
REF_SRC = os.environ.get("GLAC_REF_SRC", os.path.normpath(os.path.join(HERE, "..", "..", "reference", "GLAC")))

_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_u8 = np.ctypeslib.ndpointer(dtype=np.uint8, flags="C_CONTIGUOUS")
_i32 = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_u32 = np.ctypeslib.ndpointer(dtype=np.uint32, flags="C_CONTIGUOUS")


def build(ref: bool = True) -> None:
    """Compile the C restatement, and the reference libraries when its sources exist."""
    targets = ["oracle"]
    if ref and os.path.isdir(REF_SRC):
        targets += ["ref", "ref-native", "ref-bin"]
        if os.path.exists(os.path.join(HERE, "..", "glac_b200", "libglac_b200.so")):
            targets.append("ref-bin-bound")
    subprocess.run(["make", "-s", "-C", HERE, "-j8", f"REF_SRC={REF_SRC}", *targets], check=True)


def _cpu_flags(path="/proc/cpuinfo"):
    try:
        with open(path) as f:
            for line in f:
                if line.startswith("flags"):
                    return set(line.split(":", 1)[1].split())
    except OSError:
        pass
    return set()


def ref_library():
    """(path, build) of the reference library to load on this host.

    The -march=native build when it exists and this CPU has every ISA flag of
    the CPU that compiled it (so it cannot hit an unsupported instruction),
    else the portable -march=x86-64-v3 build.
    """
    if os.path.exists(REF_NATIVE_SO) and os.path.exists(REF_NATIVE_FLAGS):
        with open(REF_NATIVE_FLAGS) as f:
            need = _isa_flags(f.read().split())
        if need and need <= _isa_flags(_cpu_flags()):
            return REF_NATIVE_SO, "-O3 -march=native"
    return REF_SO, "-O3 -march=x86-64-v3"


# /proc/cpuinfo flags that name instruction-set extensions a compiler may emit
# (the rest -- hypervisor, clock and power features -- differ between hosts
# with the same instruction set)
_ISA_PREFIXES = ("sse", "ssse", "avx", "fma", "f16c", "bmi", "amx", "movbe", "popcnt", "abm", "adx", "sha",
                 "vaes", "vpclmul", "gfni", "aes", "pclmul", "cx16", "lzcnt", "rdrand", "rdseed", "clflushopt",
                 "clwb", "xsave", "movdir", "serialize", "prefetchw", "3dnowprefetch")


def _isa_flags(flags):
    return {f for f in flags if f.startswith(_ISA_PREFIXES)}


def _dims(N):
    N = [int(n) for n in N]
    if len(N) != 4:
        raise ValueError("N must have 4 entries (Nx, Ny, Nz, Nt)")
    return (C.c_int * 4)(*N), int(np.prod(N))


class Oracle:
    """The C restatement of the reference path (plus the project's Philox/Haar parts)."""

    def __init__(self, path: str = ORACLE_SO):
        if not os.path.exists(path):
            build(ref=False)
        lib = C.CDLL(path)
        lib.oracle_philox4x32_10.argtypes = [_u32, _u32, _u32]
        lib.oracle_su3_mul.argtypes = [_dp, _dp, _dp]
        lib.oracle_su3_dagger.argtypes = [_dp, _dp]
        lib.oracle_retr_mul.argtypes = [_dp, _dp]
        lib.oracle_retr_mul.restype = C.c_double
        lib.oracle_staples.argtypes = [C.c_int * 4, _dp, _dp]
        lib.oracle_delta_s.argtypes = [_dp, _dp, _dp, C.c_double]
        lib.oracle_delta_s.restype = C.c_double
        lib.oracle_force.argtypes = [C.c_int * 4, _dp, _dp]
        lib.oracle_exp.argtypes = [C.c_int, C.c_int, _dp, C.c_long, _dp]
        lib.oracle_flow.argtypes = [C.c_int * 4, _dp, C.c_double, C.c_int, C.c_int]
        lib.oracle_observables.argtypes = [C.c_int * 4, _dp, _dp]
        lib.oracle_plaquette.argtypes = [C.c_int * 4, _dp]
        lib.oracle_plaquette.restype = C.c_double
        lib.oracle_rst_multiply.argtypes = [_dp, _dp, _dp, C.c_int, _dp]
        lib.oracle_su2_near_unity.argtypes = [_dp, C.c_double, _dp]
        lib.oracle_accept_fed.argtypes = [C.c_long, C.c_int, C.c_double, _dp, _dp, _dp, _dp, _u8]
        lib.oracle_metropolis_sweep.argtypes = [C.c_int * 4, _dp, C.c_double, C.c_double, C.c_int,
                                                C.c_uint64, C.c_uint32, C.c_uint32, C.c_int]
        lib.oracle_metropolis_sweep.restype = C.c_uint64
        lib.oracle_haar_field.argtypes = [C.c_int * 4, _dp, C.c_uint64, C.c_uint32]
        lib.oracle_reunitarize.argtypes = [_dp, C.c_long]
        lib.oracle_density.argtypes = [C.c_int * 4, _dp, _dp, _dp]
        lib.oracle_weinberg.argtypes = [C.c_int * 4, _dp, _dp]
        lib.oracle_esj_link.argtypes = [_dp, _dp, C.c_double, C.c_int, C.c_int, _dp, C.c_int, C.c_uint64,
                                        C.c_uint32, C.c_uint32, C.c_uint32, C.c_int, _dp]
        self.lib = lib

    def philox(self, ctr, key):
        out = np.zeros(4, np.uint32)
        self.lib.oracle_philox4x32_10(np.ascontiguousarray(ctr, np.uint32),
                                      np.ascontiguousarray(key, np.uint32), out)
        return out

    def su3_mul(self, A, B):
        out = np.zeros(18)
        self.lib.oracle_su3_mul(np.ascontiguousarray(A, np.float64), np.ascontiguousarray(B, np.float64), out)
        return out

    def su3_dagger(self, A):
        out = np.zeros(18)
        self.lib.oracle_su3_dagger(np.ascontiguousarray(A, np.float64), out)
        return out

    def retr_mul(self, A, B):
        return self.lib.oracle_retr_mul(np.ascontiguousarray(A, np.float64), np.ascontiguousarray(B, np.float64))

    def staples(self, N, links):
        n, V = _dims(N)
        out = np.zeros((4, V, 18))
        self.lib.oracle_staples(n, np.ascontiguousarray(links, np.float64), out)
        return out

    def delta_s(self, U, Up, A, beta):
        return self.lib.oracle_delta_s(*(np.ascontiguousarray(a, np.float64) for a in (U, Up, A)), beta)

    def force(self, N, links):
        n, V = _dims(N)
        out = np.zeros((4, V, 18))
        self.lib.oracle_force(n, np.ascontiguousarray(links, np.float64), out)
        return out

    def exp(self, mats, kind=0, degree=16):
        m = np.ascontiguousarray(mats, np.float64).reshape(-1, 18)
        out = np.zeros_like(m)
        self.lib.oracle_exp(kind, degree, m, m.shape[0], out)
        return out.reshape(np.shape(mats))

    def flow(self, N, links, eps, nsteps, expkind=0):
        n, _ = _dims(N)
        out = np.array(links, np.float64, copy=True, order="C")
        self.lib.oracle_flow(n, out, eps, nsteps, expkind)
        return out

    def observables(self, N, links):
        n, _ = _dims(N)
        out = np.zeros(3 + int(N[3]))
        self.lib.oracle_observables(n, np.ascontiguousarray(links, np.float64), out)
        return out

    def plaquette(self, N, links):
        n, _ = _dims(N)
        return self.lib.oracle_plaquette(n, np.ascontiguousarray(links, np.float64))

    def rst_multiply(self, r8, s8, t8, inverse=False):
        out = np.zeros(18)
        self.lib.oracle_rst_multiply(*(np.ascontiguousarray(a, np.float64) for a in (r8, s8, t8)),
                                     int(inverse), out)
        return out

    def accept_fed(self, U, A, X, r, beta):
        U = np.array(U, np.float64, copy=True, order="C").reshape(-1, 18)
        nl = U.shape[0]
        nh = int(np.size(r) // nl)
        acc = np.zeros(nl * nh, np.uint8)
        self.lib.oracle_accept_fed(nl, nh, beta, U, np.ascontiguousarray(A, np.float64),
                                   np.ascontiguousarray(X, np.float64), np.ascontiguousarray(r, np.float64), acc)
        return U, acc.reshape(nl, nh)

    def metropolis_sweep(self, N, links, beta, eps, nhits, seed, stream, sweep, flips=True):
        n, _ = _dims(N)
        out = np.array(links, np.float64, copy=True, order="C")
        acc = self.lib.oracle_metropolis_sweep(n, out, beta, eps, nhits, seed, stream, sweep, int(bool(flips)))
        return out, int(acc)

    def weinberg(self, N, links):
        """SuperSampler observables [plaq, topc, energy, weinberg, topct[Nt], weinbergt[Nt]]."""
        n, _ = _dims(N)
        out = np.zeros(4 + 2 * int(N[3]))
        self.lib.oracle_weinberg(n, np.ascontiguousarray(links, np.float64), out)
        return out

    def density(self, N, links):
        """Per-site (q, e) densities of LatticeActionChargeDensity, V doubles each."""
        n, V = _dims(N)
        q, e = np.zeros(V), np.zeros(V)
        self.lib.oracle_density(n, np.ascontiguousarray(links, np.float64), q, e)
        return q, e

    def esj_link(self, U, A, beta, nhits, eps_grid, trials, seed, link_id, snapshot, stream, flips=True):
        """Expected squared jump of one link for each spread on the grid."""
        g = np.ascontiguousarray(eps_grid, np.float64)
        J = np.zeros(g.size)
        self.lib.oracle_esj_link(np.ascontiguousarray(U, np.float64), np.ascontiguousarray(A, np.float64),
                                 float(beta), int(nhits), g.size, g, int(trials), int(seed), int(link_id),
                                 int(snapshot), int(stream), int(bool(flips)), J)
        return J

    def haar_field(self, N, seed, stream=0):
        n, V = _dims(N)
        out = np.zeros((4, V, 18))
        self.lib.oracle_haar_field(n, out, seed, stream)
        return out

    def reunitarize(self, mats):
        m = np.array(mats, np.float64, copy=True, order="C")
        self.lib.oracle_reunitarize(m, m.size // 18)
        return m


class Reference:
    """The reference's own classes, compiled from its sources (see oracle/Makefile)."""

    def __init__(self, path: str | None = None):
        if path is None:
            if not os.path.exists(REF_SO) and os.path.isdir(REF_SRC):
                build(ref=True)
            path, self.build_flags = ref_library()
        else:
            self.build_flags = "given path"
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} is not built and the reference sources are absent")
        self.path = path
        lib = C.CDLL(path)
        lib.ref_configure.argtypes = [C.c_int, C.c_int, C.c_double, C.c_double, C.c_double, C.c_char_p,
                                      C.c_double, C.c_double, C.c_int, C.c_int]
        lib.ref_staples.argtypes = [_dp, _dp]
        lib.ref_delta_s.argtypes = [_dp, _dp, _dp]
        lib.ref_delta_s.restype = C.c_double
        lib.ref_action_derivative.argtypes = [_dp, _dp]
        lib.ref_exp.argtypes = [C.c_int, C.c_int, _dp, C.c_long, _dp]
        lib.ref_flow.argtypes = [_dp, C.c_int]
        lib.ref_observables.argtypes = [_dp, _dp]
        lib.ref_observables_nt.argtypes = [_dp, _dp]
        lib.ref_plaquette.argtypes = [_dp]
        lib.ref_plaquette.restype = C.c_double
        lib.ref_generate.argtypes = [C.c_int, C.c_long, _dp]
        lib.ref_rst_multiply.argtypes = [_dp, _dp, _dp, C.c_int, _dp]
        lib.ref_metropolis.argtypes = [_dp, C.c_int]
        lib.ref_metropolis.restype = C.c_double
        lib.ref_metropolis_trace.argtypes = [_dp, _dp, _dp, _dp, _dp, _u8, _i32]
        lib.ref_metropolis_trace.restype = C.c_long
        lib.ref_load_field.argtypes = [C.c_char_p, C.c_int, _dp]
        lib.ref_write_field.argtypes = [_dp, C.c_char_p, C.c_char_p, C.c_int]
        lib.ref_time_flow.argtypes = [_dp, C.c_int]
        lib.ref_time_flow.restype = C.c_double
        lib.ref_time_flow_measure.argtypes = [_dp, C.c_int]
        lib.ref_time_flow_measure.restype = C.c_double
        lib.ref_density.argtypes = [_dp, _dp, _dp, _dp]
        lib.ref_supersampler.argtypes = [_dp, _dp]
        lib.ref_metropolis_chain.argtypes = [_dp, C.c_int, _dp]
        lib.ref_metropolis_chain.restype = C.c_double
        lib.ref_time_metropolis.argtypes = [_dp, C.c_int, C.POINTER(C.c_double)]
        lib.ref_time_metropolis.restype = C.c_double
        lib.ref_time_observables.argtypes = [_dp, C.c_int]
        lib.ref_time_observables.restype = C.c_double
        self.lib = lib
        self.N = None
        self.nupdates = 10

    def configure(self, Ns, Nt, beta=6.0, su3eps=0.24, flow_eps=0.01, exp_func="morningstar",
                  metropolis_seed=1.0, matrix_seed=2.0, nupdates=10, nflows=0):
        self.lib.ref_configure(int(Ns), int(Nt), beta, su3eps, flow_eps, exp_func.encode(),
                               float(metropolis_seed), float(matrix_seed), int(nupdates), int(nflows))
        self.N = (int(Ns), int(Ns), int(Ns), int(Nt))
        self.nupdates = int(nupdates)
        return self

    @property
    def V(self):
        return int(np.prod(self.N))

    def staples(self, links):
        out = np.zeros((4, self.V, 18))
        self.lib.ref_staples(np.ascontiguousarray(links, np.float64), out)
        return out

    def delta_s(self, U, Up, A):
        return self.lib.ref_delta_s(*(np.ascontiguousarray(a, np.float64) for a in (U, Up, A)))

    def force(self, links):
        out = np.zeros((4, self.V, 18))
        self.lib.ref_action_derivative(np.ascontiguousarray(links, np.float64), out)
        return out

    def exp(self, mats, kind=0, degree=16):
        m = np.ascontiguousarray(mats, np.float64).reshape(-1, 18)
        out = np.zeros_like(m)
        self.lib.ref_exp(kind, degree, m, m.shape[0], out)
        return out.reshape(np.shape(mats))

    def flow(self, links, nsteps):
        out = np.array(links, np.float64, copy=True, order="C")
        self.lib.ref_flow(out, int(nsteps))
        return out

    def observables(self, links):
        out = np.zeros(3 + self.N[3])
        self.lib.ref_observables(np.ascontiguousarray(links, np.float64), out)
        return out

    def observables_nt(self, links):
        out = np.zeros(3)
        self.lib.ref_observables_nt(np.ascontiguousarray(links, np.float64), out)
        return out

    def plaquette(self, links):
        return self.lib.ref_plaquette(np.ascontiguousarray(links, np.float64))

    def generate(self, n, kind=0):
        out = np.zeros((n, 18))
        self.lib.ref_generate(kind, n, out)
        return out

    def rst_multiply(self, r8, s8, t8, inverse=False):
        out = np.zeros(18)
        self.lib.ref_rst_multiply(*(np.ascontiguousarray(a, np.float64) for a in (r8, s8, t8)),
                                  int(inverse), out)
        return out

    def metropolis(self, links, nsweeps):
        out = np.array(links, np.float64, copy=True, order="C")
        acc = self.lib.ref_metropolis(out, int(nsweeps))
        return out, acc

    def supersampler(self, links):
        """The reference's SuperSampler: [plaq, topc, energy, weinberg, topct[Nt], weinbergt[Nt]]."""
        out = np.zeros(4 + 2 * self.N[3])
        self.lib.ref_supersampler(np.ascontiguousarray(links, np.float64), out)
        return out

    def density(self, links):
        """(q, e, [plaq, topc, energy]) of the reference's LatticeActionChargeDensity."""
        q, e, o = np.zeros(self.V), np.zeros(self.V), np.zeros(3)
        self.lib.ref_density(np.ascontiguousarray(links, np.float64), q, e, o)
        return q, e, o

    def metropolis_chain(self, links, nsweeps):
        """nsweeps sweeps of one System: (links after, plaquette per sweep, acceptance)."""
        out = np.array(links, np.float64, copy=True, order="C")
        plaq = np.zeros(int(nsweeps))
        acc = self.lib.ref_metropolis_chain(out, int(nsweeps), plaq)
        return out, plaq, acc

    def metropolis_trace(self, links):
        nl, nh = 4 * self.V, self.nupdates
        out = np.array(links, np.float64, copy=True, order="C")
        Ub = np.zeros((nl, 18))
        A = np.zeros((nl, 18))
        X = np.zeros((nl, nh, 18))
        r = np.zeros((nl, nh))
        acc = np.zeros((nl, nh), np.uint8)
        order = np.zeros((nl, 2), np.int32)
        self.lib.ref_metropolis_trace(out, Ub, A, X, r, acc, order)
        return dict(links=out, U_before=Ub, staples=A, X=X, r=r, accept=acc, order=order)

    def load_field(self, path, chroma=False):
        out = np.zeros((4, self.V, 18))
        self.lib.ref_load_field(os.fsencode(path), int(chroma), out)
        return out

    def write_field(self, links, directory, batch, config_number=0):
        d = directory if directory.endswith("/") else directory + "/"
        os.makedirs(os.path.join(d, batch, "field_configurations"), exist_ok=True)
        self.lib.ref_write_field(np.ascontiguousarray(links, np.float64), d.encode(), batch.encode(),
                                 int(config_number))

    def time_flow(self, links, nsteps):
        out = np.array(links, np.float64, copy=True, order="C")
        return self.lib.ref_time_flow(out, int(nsteps))

    def time_flow_measure(self, links, nsteps):
        out = np.array(links, np.float64, copy=True, order="C")
        return self.lib.ref_time_flow_measure(out, int(nsteps))

    def time_metropolis(self, links, nsweeps):
        out = np.array(links, np.float64, copy=True, order="C")
        acc = C.c_double(0.0)
        dt = self.lib.ref_time_metropolis(out, int(nsweeps), C.byref(acc))
        return dt, acc.value

    def time_observables(self, links, nmeas):
        return self.lib.ref_time_observables(np.ascontiguousarray(links, np.float64), int(nmeas))
