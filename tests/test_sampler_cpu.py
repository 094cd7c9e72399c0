"""The sampler's host pieces without a GPU: acor of the product library
against the oracle restatement, bit for bit, and the oracle stretch move
against the known posterior of a Gaussian."""
import numpy as np
import pytest


def _ar1(n, rho, seed):
    rng = np.random.default_rng(seed)
    x = np.empty(n)
    x[0] = rng.standard_normal()
    for i in range(1, n):
        x[i] = rho * x[i - 1] + np.sqrt(1 - rho * rho) * rng.standard_normal()
    return x.astype(np.float32)


@pytest.mark.parametrize("n,rho", [(30, 0.0), (200, 0.0), (1000, 0.5),
                                   (4000, 0.9), (5001, 0.97), (80, 0.9),
                                   (120, 0.95), (300, 0.98)])
def test_acor_matches_oracle(built_lib, n, rho):
    import sampler_oracle as so
    from pofd_affine_b200.mcmc import acor
    x = _ar1(n, rho, 3)
    m, s, t, ok = acor(x)
    om, os_, ot, st = so.acor(x.copy())
    assert ok == (st == 0)
    assert m == om
    if ok:
        assert s == os_ and t == ot
    if ok and n >= 4000 and rho <= 0.9:
        # AR(1): tau = (1 + rho) / (1 - rho)
        assert abs(t / ((1 + rho) / (1 - rho)) - 1) < 0.35


def test_philox_known_answer():
    """Philox4x32-10 known-answer vectors of the Random123 distribution
    (kat_vectors: counter/key all zeros, all ones, and the pi digits)."""
    import sampler_oracle as so
    assert so.philox4x32_10((0, 0, 0, 0), (0, 0)) == (
        0x6627e8d5, 0xe169c58d, 0xbc57ac4c, 0x9b00dbd8)
    assert so.philox4x32_10((0xffffffff,) * 4, (0xffffffff,) * 2) == (
        0x408f276d, 0x41c83b0e, 0xa20bc7c6, 0x6d5451fd)
    assert so.philox4x32_10((0x243f6a88, 0x85a308d3, 0x13198a2e, 0x03707344),
                            (0xa4093822, 0x299f31d0)) == (
        0xd16cfe09, 0x94fdcceb, 0x5001e420, 0x24126ea1)


def test_oracle_stretch_samples_gaussian():
    import sampler_oracle as so
    rng = np.random.default_rng(0)
    k = 3
    A = rng.normal(size=(k, k))
    cov = A @ A.T + k * np.eye(k)
    mu = np.array([1.0, -2.0, 0.5])
    icov = np.linalg.inv(cov)

    def ll(th):
        d = th.astype(np.float64) - mu
        return -0.5 * np.einsum("ij,jk,ik->i", d, icov, d), np.zeros(len(th), int)

    nw = 16
    w = (mu + rng.normal(size=(nw, k))).astype(np.float32)
    ch, _, nacc = so.stretch_run(w, np.full(nw, -np.inf), ll, 600, seed=5)
    s = ch[100:].reshape(-1, k)
    assert np.all(np.abs(s.mean(0) - mu) < 0.5 * np.sqrt(np.diag(cov)))
    assert np.all(np.abs(np.diag(np.cov(s.T)) / np.diag(cov) - 1) < 0.35)
    assert 0.2 < nacc.sum() / (600 * nw) < 0.9


@pytest.mark.parametrize("rho", [0.5, 0.9, 0.97])
def test_integrated_time_on_ar1_ensembles(rho):
    """Sokal-window integrated time against the exact tau = (1 + rho) /
    (1 - rho) of AR(1) walkers, within 10 % on chains of > 100 tau."""
    from pofd_affine_b200.mcmc import integrated_time
    rng = np.random.default_rng(int(rho * 100))
    nsteps, nw = 8000, 32
    x = np.empty((nsteps, nw, 2))
    e = rng.normal(size=(nsteps, nw, 2))
    x[0] = e[0] / np.sqrt(1 - rho * rho)
    for t in range(1, nsteps):
        x[t] = rho * x[t - 1] + e[t]
    x[:, :, 1] = 3.0  # a fixed parameter
    tau, win, conv = integrated_time(x)
    exact = (1 + rho) / (1 - rho)
    assert conv[0] and abs(tau[0] / exact - 1) < 0.1, (tau[0], exact)
    assert np.isnan(tau[1])
    assert win[0] >= 5 * tau[0]


def test_host_mcmc_baseline_runs():
    """The host plain-method baseline of the benchmark (oracle sampler over
    the oracle likelihood, thread farm) on a short chain of the 1D plain
    fit: every walker moves, the chain stays inside the knot limits and the
    effective-sample bookkeeping is finite."""
    import bench
    r = bench.cpu_mcmc_1d(nthreads=2, nburn=5, nsteps=20, nwalkers=8)
    assert r["evals"] == 8 * 26
    assert 0.05 < r["acceptance"] < 0.95
    assert np.isfinite(r["tau_max"]) and r["ess"] > 0
    assert 0 < r["likelihood_s"] <= r["wall_s"]


def test_oracle_limit_policy_reject_stays_inside():
    """The oracle's reject-outside limit policy (the product's opt-in
    policy): a wide stretch with a limit through the posterior's middle
    never leaves the limits and never raises, and only steps inside the
    limits are accepted."""
    import sampler_oracle as so

    def ll(th):
        d = th.astype(np.float64)
        return -0.5 * (d * d).sum(1), np.zeros(len(th), int)
    w = np.abs(np.random.default_rng(0).normal(size=(8, 2))).astype(np.float32)
    lo = np.array([0.0, -np.inf], np.float32)
    hi = np.array([np.inf, np.inf], np.float32)
    ch, _, na = so.stretch_run(w, np.full(8, -np.inf), ll, 60, seed=3,
                               scalefac=5.0, lo=lo, hi=hi,
                               reject_outside=True)
    assert ch[..., 0].min() >= 0.0
    assert 0 < na.sum() < 8 * 60
