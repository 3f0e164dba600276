"""The reference's operator names over the device implementation.

Thin Python mirrors of GLAC's C++ interface for this path, so that callers
(and tests written like the reference's own) use the same names and
argument meanings: ``WilsonGaugeAction`` (GLAC/actions/action.h:49-68),
``Flow`` (GLAC/flow/flow.h:42), ``SU3Exp`` (GLAC/math/exponentiation/su3exp.h:32),
``MasterSamplerTopcXYZ`` / ``Plaquette`` (GLAC/observables/correlator.h:46-67).
All arithmetic runs in the CUDA library; nothing here computes on the CPU.
"""
from __future__ import annotations

import numpy as np


class WilsonGaugeAction:
    """Staple, Delta S and flow force of the Wilson gauge action
    (GLAC/actions/wilsongaugeaction.cpp:24-86)."""

    def __init__(self, beta: float):
        self.beta = float(beta)
        self._staple = None
        self._cache = None

    def computeStaple(self, lattice, i, j, k, l, mu):  # noqa: N802 (reference name)
        if self._cache is None or self._cache[0] is not lattice:
            self._cache = (lattice, lattice.staples())
        Nx, Ny, Nz, _ = lattice.dims
        site = i + Nx * (j + Ny * (k + Nz * l))
        self._staple = self._cache[1][mu, site].copy()

    def invalidate(self):
        self._cache = None

    def getDeltaAction(self, U, UPrime, precision="fp64"):  # noqa: N802
        from . import delta_s_batch
        return float(delta_s_batch(np.reshape(U, (1, 18)), np.reshape(UPrime, (1, 18)),
                                   np.reshape(self._staple, (1, 18)), self.beta, precision)[0])

    def getActionDerivative(self, lattice, mu):  # noqa: N802
        return lattice.force()[mu]


class SU3Exp:
    """Exponential of traceless anti-Hermitian matrices (morningstar by default)."""

    def __init__(self, name: str = "morningstar", precision: str = "fp64"):
        self.name, self.precision = name, precision

    def exp(self, Q):
        from . import exp_batch
        return exp_batch(Q, self.precision, self.name)


class Flow:
    """Luscher RK3 gradient flow with step flowEpsilon (GLAC/flow/flow.cpp:43-73)."""

    def __init__(self, lattice):
        self.lattice = lattice

    def flowField(self, lattice=None):  # noqa: N802
        (lattice or self.lattice).flow(1, measure=False)


class MasterSamplerTopcXYZ:
    """plaq, topc, energy and topct per call (GLAC/observables/mastersamplertopcxyz.cpp:236-384)."""

    def __init__(self, n_obs: int, Nt: int):
        self.obs = np.zeros((n_obs, 3 + Nt))

    def calculate(self, lattice, iObs):  # noqa: N803
        self.obs[iObs] = lattice.measure()

    def getObservablesVector(self, iObs):  # noqa: N802,N803
        return self.obs[iObs].copy()


class Plaquette:
    """Plaquette alone (GLAC/observables/plaquette.cpp:26-40)."""

    def __init__(self, n_obs: int):
        self.obs = np.zeros(n_obs)

    def calculate(self, lattice, iObs):  # noqa: N803
        self.obs[iObs] = lattice.measure()[0]
