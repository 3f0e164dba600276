"""Monte Carlo error analysis for Markov-chain time series.

The reference leaves autocorrelation analysis to an external package, so this
module restates the published Gamma method (U. Wolff, "Monte Carlo errors with
less errors", Comput. Phys. Commun. 156 (2004) 143-153, Sections 3 and 4) for a
primary observable:

* autocorrelation function Gamma(t) = <(a_i - abar)(a_{i+t} - abar)>;
* integrated autocorrelation time tau_int(W) = 1/2 + sum_{t=1..W} rho(t);
* automatic window: the first W with g(W) = exp(-W/tau(W)) - tau(W)/sqrt(W N) < 0,
  tau(W) = S / ln((2 tau_int(W) + 1) / (2 tau_int(W) - 1)), S = 1.5 by default;
* bias correction of Gamma by C_F(W)/N, error of tau_int from the Madras-Sokal
  formula d tau ~= tau * sqrt((4W + 2)/N), error of the mean sqrt(C_F/N).

For several independent chains (replicas) of one algorithm, Wolff Section 3.3:
Gamma(t) is averaged over the replicas about the grand mean, with N the total
number of samples (gamma_method_replicas), and a delete-one-replica jackknife
gives errors of derived quantities (jackknife).

Also binned (jackknife-free) errors for several chains, used when chains are
short compared with their autocorrelation.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np


@dataclass
class GammaResult:
    mean: float
    error: float          # statistical error of the mean, autocorrelation included
    tau_int: float        # integrated autocorrelation time in units of the series spacing
    tau_error: float
    window: int
    n: int

    @property
    def n_eff(self) -> float:
        """Effectively independent samples, N / (2 tau_int)."""
        return self.n / (2.0 * self.tau_int)


def autocorrelation(a: np.ndarray) -> np.ndarray:
    """Gamma(t) for t = 0..N-1 (FFT, zero-padded, normalised by N - t)."""
    a = np.asarray(a, np.float64)
    n = a.size
    d = a - a.mean()
    m = 1 << (2 * n - 1).bit_length()
    f = np.fft.rfft(d, m)
    g = np.fft.irfft(f * np.conj(f), m)[:n]
    return g / (n - np.arange(n))


def _window(G: np.ndarray, n: int, S: float) -> int:
    """Wolff's automatic window for the autocorrelation function G of n samples."""
    wmax = G.size - 1
    tint = 0.5
    for w in range(1, wmax + 1):
        tint += G[w] / G[0]
        if tint <= 0.5:
            tau = 1e-12  # decorrelated faster than a step: stop at once
        else:
            tau = S / np.log((2 * tint + 1) / (2 * tint - 1))
        if np.exp(-w / tau) - tau / np.sqrt(w * n) < 0:
            return w
    return wmax


def gamma_method_replicas(chains, S: float = 1.5) -> GammaResult:
    """The Gamma method for R independent replicas of one chain (Wolff, Section 3.3).

    Gamma(t) = sum_r sum_i (a_ri - abar)(a_r,i+t - abar) / sum_r (N_r - t),
    abar the grand mean; window, bias correction and errors as in
    gamma_method with N = sum_r N_r.  (The mean over replicas of unequal
    length is weighted by N_r.)
    """
    chains = [np.asarray(c, np.float64).ravel() for c in chains]
    if len(chains) == 1:
        return gamma_method(chains[0], S)
    n = sum(c.size for c in chains)
    if min(c.size for c in chains) < 4:
        raise ValueError("every replica needs at least 4 samples")
    abar = float(sum(c.sum() for c in chains) / n)
    tmax = min(c.size for c in chains) // 2
    num = np.zeros(tmax + 1)
    den = np.zeros(tmax + 1)
    for c in chains:
        d = c - abar
        m = 1 << (2 * d.size - 1).bit_length()
        f = np.fft.rfft(d, m)
        g = np.fft.irfft(f * np.conj(f), m)[:tmax + 1]
        num += g
        den += d.size - np.arange(tmax + 1)
    G = num / den
    if G[0] <= 0.0:
        return GammaResult(abar, 0.0, 0.5, 0.0, 0, n)
    W = _window(G, n, S)
    CF = G[0] + 2.0 * G[1:W + 1].sum()
    Gc = G[:W + 1] + CF / n
    CF = Gc[0] + 2.0 * Gc[1:].sum()
    tau_int = max(CF / (2.0 * Gc[0]), 0.5)
    tau_err = tau_int * np.sqrt((4.0 * W + 2.0) / n)
    return GammaResult(abar, float(np.sqrt(max(CF, 0.0) / n)), float(tau_int), float(tau_err), int(W), n)


def jackknife(values_by_replica_removed):
    """Jackknife error from the R delete-one-replica estimates of a quantity."""
    v = np.asarray(values_by_replica_removed, np.float64)
    R = v.size
    if R < 2:
        return float("nan")
    return float(np.sqrt((R - 1) / R * np.sum((v - v.mean()) ** 2)))


def gamma_method(a, S: float = 1.5) -> GammaResult:
    """Wolff's Gamma method with automatic windowing for one chain."""
    a = np.asarray(a, np.float64).ravel()
    n = a.size
    if n < 4:
        raise ValueError("gamma_method needs at least 4 samples")
    G = autocorrelation(a)
    if G[0] <= 0.0:  # constant series
        return GammaResult(float(a.mean()), 0.0, 0.5, 0.0, 0, n)
    wmax = n // 2
    W = wmax
    tint = 0.5
    for w in range(1, wmax + 1):
        tint += G[w] / G[0]
        if tint <= 0.5:
            tau = 1e-12  # decorrelated faster than a step: stop at once
        else:
            tau = S / np.log((2 * tint + 1) / (2 * tint - 1))
        g = np.exp(-w / tau) - tau / np.sqrt(w * n)
        if g < 0:
            W = w
            break
    CF = G[0] + 2.0 * G[1:W + 1].sum()
    # bias correction of the autocorrelation function (Wolff eq. 49)
    Gc = G[:W + 1] + CF / n
    CF = Gc[0] + 2.0 * Gc[1:].sum()
    tau_int = max(CF / (2.0 * Gc[0]), 0.5)
    tau_err = tau_int * np.sqrt((4.0 * W + 2.0) / n)
    err = np.sqrt(max(CF, 0.0) / n)
    return GammaResult(float(a.mean()), float(err), float(tau_int), float(tau_err), int(W), n)


def binned_mean(chains, nbins: int = 20):
    """Mean and error of several chains by equal-length bins (bins treated as independent)."""
    means = []
    for c in chains:
        c = np.asarray(c, np.float64).ravel()
        L = c.size // nbins
        if L == 0:
            raise ValueError("chain shorter than the number of bins")
        means.append(c[: L * nbins].reshape(nbins, L).mean(axis=1))
    b = np.concatenate(means)
    return float(b.mean()), float(b.std(ddof=1) / np.sqrt(b.size))


def ar1(n: int, rho: float, seed: int = 0) -> np.ndarray:
    """AR(1) test series x_{i+1} = rho x_i + e_i; its tau_int is (1+rho)/(2(1-rho))."""
    rng = np.random.default_rng(seed)
    e = rng.standard_normal(n)
    x = np.empty(n)
    x[0] = e[0] / np.sqrt(1 - rho * rho)
    for i in range(1, n):
        x[i] = rho * x[i - 1] + e[i]
    return x
