"""The Gamma-method error analysis (glac_b200.analysis) on series with known answers."""
import numpy as np
import pytest

from glac_b200.analysis import ar1, autocorrelation, binned_mean, gamma_method


@pytest.mark.parametrize("rho", [0.0, 0.5, 0.9])
def test_tau_int_of_ar1(rho):
    r = gamma_method(ar1(100_000, rho, seed=3))
    want = (1 + rho) / (2 * (1 - rho))
    assert abs(r.tau_int - want) < 4 * r.tau_error + 1e-9
    # error of the mean of AR(1): sqrt(2 tau_int var / N), var = 1/(1-rho^2)
    want_err = np.sqrt(2 * want / (1 - rho * rho) / r.n)
    assert abs(r.error / want_err - 1) < 0.1


def test_autocorrelation_matches_direct_sum():
    a = ar1(500, 0.7, seed=1)
    d = a - a.mean()
    G = autocorrelation(a)
    for t in (0, 1, 5, 40):
        assert np.isclose(G[t], np.dot(d[: a.size - t], d[t:]) / (a.size - t))


def test_constant_series_and_bins():
    r = gamma_method(np.full(100, 2.5))
    assert r.mean == 2.5 and r.error == 0.0 and r.tau_int == 0.5
    m, e = binned_mean([np.arange(100.0), np.arange(100.0)], 10)
    assert m == pytest.approx(49.5) and e > 0
    with pytest.raises(ValueError):
        gamma_method([1.0, 2.0])


def test_replica_gamma_method_on_ar1():
    # four independent AR(1) replicas: the pooled estimate finds the known tau_int
    from glac_b200.analysis import gamma_method_replicas, jackknife
    rho = 0.8
    chains = [ar1(20_000, rho, seed=10 + r) for r in range(4)]
    r = gamma_method_replicas(chains)
    want = (1 + rho) / (2 * (1 - rho))
    assert r.n == 80_000
    assert abs(r.tau_int - want) < 4 * r.tau_error
    # delete-one-replica jackknife of tau_int: an error of the size Madras-Sokal gives
    loo = [gamma_method_replicas(chains[:k] + chains[k + 1:]).tau_int for k in range(4)]
    je = jackknife(loo)
    assert 0.2 * r.tau_error < je < 5 * r.tau_error
    # one replica: the single-chain method
    assert gamma_method_replicas(chains[:1]).tau_int == gamma_method(chains[0]).tau_int
