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


def _study_runs(samplers, replicas, n_meas, meas_every=100, seed=0):
    """Synthetic chains in the layout glac_b200.studies.target_run writes: Q is
    an AR(1) series with per-measurement correlation rho (the same stationary
    variance for every sampler), plaquette and E are white noise."""
    chains = []
    for si, (name, rho, sweep_s) in enumerate(samplers):
        for r in range(replicas):
            q = ar1(n_meas, rho, seed=seed + 1000 * si + r) * np.sqrt(1 - rho * rho) * 6.0
            g = np.random.default_rng(seed + 7 + 1000 * si + r)
            chains.append(dict(sampler=name, replica=r, meas_every=meas_every, sweeps=n_meas * meas_every,
                               wall_s=n_meas * meas_every * sweep_s, acceptance=0.2, Q=q.tolist(),
                               plaq=(0.61 + 1e-4 * g.standard_normal(n_meas)).tolist(),
                               E=(-2.0 + 1e-3 * g.standard_normal(n_meas)).tolist()))
    return [dict(config={"synthetic": True}, chains=chains)]


def test_q_diffusion_estimator_on_known_chains():
    # Two samplers of known tau_int,Q and cost: "plain_fp64" decorrelates over
    # 3000 sweeps at 9.6 ms a sweep, "learned_fp32" over 1000 sweeps at 3.9 ms.
    # For AR(1), <(Q_{i+k} - Q_i)^2> = 2 var (1 - rho^k) exactly, so the
    # diffusion ratio at lag k has a known expectation, which lies below the
    # ratio of effective samples per second (1 - rho^k is concave in the
    # decorrelation rate): the estimator can only understate the faster sampler.
    from glac_b200.studies import target_combine
    every = 100
    rho_a, rho_b = np.exp(-every / 3000.0), np.exp(-every / 1000.0)
    res = target_combine(_study_runs([("plain_fp64", rho_a, 9.6e-3), ("learned_fp32", rho_b, 3.9e-3)],
                                     replicas=48, n_meas=600))["samplers"]
    tau = lambda rho: (1 + rho) / (2 * (1 - rho))
    true_ratio = (tau(rho_a) * 9.6e-3) / (tau(rho_b) * 3.9e-3)
    for lag in (200, 500, 1000):
        k = lag // every
        expect = ((1 - rho_b ** k) / 3.9e-3) / ((1 - rho_a ** k) / 9.6e-3)
        got = res["learned_fp32"][f"eff_Q_ratio_vs_plain_fp64_diffusion_{lag}"]
        err = res["learned_fp32"][f"eff_Q_ratio_vs_plain_fp64_diffusion_{lag}_err"]
        assert expect < true_ratio
        assert abs(got - expect) < 4 * err and err < 0.1 * expect, (lag, got, expect, err)
    # the replica Gamma method finds tau_int,Q of each sampler (in sweeps)
    for name, rho in (("plain_fp64", rho_a), ("learned_fp32", rho_b)):
        assert abs(res[name]["tau_Q"] - tau(rho) * every) < 4 * res[name]["tau_Q_err"]
    assert res["plain_fp64"]["eff_Q_ratio_vs_plain_fp64"] == 1.0
