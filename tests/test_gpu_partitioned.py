"""Partitioned h2 on the device (ldsc_h2_partitioned) against the oracle's
fit_h2_partitioned (src/regressions.rs:553-630, 1121-1226).

Tolerance: the device forms each block's weighted Gram in its own summation
order and solves by Gaussian elimination where the reference uses faer's LU
(the oracle numpy's), so estimates, delete values, h2 figures and the
jackknife covariance agree to a relative 1e-8 (entries near zero: 1e-8 of the
largest of their array); counts and block numbers are exact.  With ~100
near-collinear columns the solves lose digits with the condition number, and
the bound scales with it.
"""
import math

import numpy as np
import pytest

from oracle import regress_oracle as R

pytestmark = pytest.mark.gpu

RTOL = 1e-8


def _annot_ld(m, k, seed):
    rng = np.random.default_rng(seed)
    base = 1.0 + rng.gamma(2.0, 15.0, m)
    frac = rng.dirichlet(np.ones(k), size=m) * rng.uniform(0.5, 1.5, (m, k))
    l2 = base[:, None] * frac
    wld = np.maximum(base * rng.uniform(0.8, 1.2, m), 0.5)
    return l2, wld


def _traits(l2, m_vec, n_traits, seed, per_snp=False):
    """chi2 = (sqrt(N s_i) b_i + e_i)^2, s_i = sum_k tau_k l2_ik (E chi2 = 1 + N s_i)."""
    rng = np.random.default_rng(seed)
    m, k = l2.shape
    tau = rng.uniform(0.0, 1.0, (n_traits, k)) * (0.4 / np.sum(m_vec))
    if per_snp:
        n = rng.uniform(5e4, 2e5, (n_traits, m))
    else:
        n = np.exp(rng.uniform(np.log(2e4), np.log(3e5), n_traits))
    nn = n if per_snp else n[:, None]
    s = np.maximum(tau @ l2.T, 0.0)
    z = np.sqrt(nn * s) * rng.standard_normal((n_traits, m)) + rng.standard_normal((n_traits, m))
    return z * z, n


def _check(got, want, k):
    assert got.n_obs == want["n_obs"] and got.n_blocks == want["n_blocks"]
    np.testing.assert_allclose(got.est, want["est"], rtol=RTOL, atol=RTOL * np.abs(want["est"]).max())
    np.testing.assert_allclose(got.delete_values, want["delete_values"], rtol=RTOL,
                               atol=RTOL * np.abs(want["delete_values"]).max())
    np.testing.assert_allclose(got.cov, want["cov"], rtol=RTOL, atol=RTOL * np.abs(want["cov"]).max())
    np.testing.assert_allclose(got.h2_annot, want["h2_annot"], rtol=RTOL,
                               atol=RTOL * np.abs(want["h2_annot"]).max())
    for key in ("h2_total", "h2_total_se", "n_mean", "mean_chi2"):
        assert got.__dict__[key] == pytest.approx(want[key], rel=RTOL), key
    if math.isnan(want["intercept_se"]):
        assert got.intercept == want["intercept"] and math.isnan(got.intercept_se)
    else:
        assert got.intercept == pytest.approx(want["intercept"], rel=RTOL)
        assert got.intercept_se == pytest.approx(want["intercept_se"], rel=RTOL)


@pytest.mark.parametrize("k", [2, 5])
def test_partitioned_scalar_n(ctx, k):
    from ldsc_b200.partitioned import h2_partitioned
    m = 40_000
    l2, wld = _annot_ld(m, k, 21 + k)
    m_vec = np.linspace(2e4, 8e4, k)
    chi2, n = _traits(l2, m_vec, 3, 31 + k)
    fits = h2_partitioned(ctx, chi2, n, l2, wld, m_vec, 200)
    for t in range(3):
        _check(fits[t], R.fit_h2_partitioned(chi2[t], l2, wld, n[t], m_vec, 200), k)


def test_partitioned_per_snp_n_with_dropped_snps(ctx):
    from ldsc_b200.partitioned import h2_partitioned
    m, k = 30_000, 4
    l2, wld = _annot_ld(m, k, 41)
    m_vec = np.array([1e4, 3e4, 5e3, 2e4])
    chi2, n = _traits(l2, m_vec, 2, 42, per_snp=True)
    rng = np.random.default_rng(43)
    chi2[0, rng.choice(m, 50, replace=False)] = np.nan       # missing chi2
    chi2[1, rng.choice(m, 30, replace=False)] = 5e3           # above the default cut
    fits = h2_partitioned(ctx, chi2, n, l2, wld, m_vec, 200)
    for t in range(2):
        want = R.fit_h2_partitioned(chi2[t], l2, wld, n[t], m_vec, 200)
        assert want["n_obs"] < m
        _check(fits[t], want, k)


def test_partitioned_missing_n_runs_that_trait_alone(ctx):
    from ldsc_b200.partitioned import h2_partitioned
    m, k = 20_000, 3
    l2, wld = _annot_ld(m, k, 44)
    m_vec = np.array([1e4, 1e4, 1e4])
    chi2, n = _traits(l2, m_vec, 2, 45, per_snp=True)
    n[1, [5, 17, 9000]] = np.nan
    fits = h2_partitioned(ctx, chi2, n, l2, wld, m_vec, 100)
    for t in range(2):
        _check(fits[t], R.fit_h2_partitioned(chi2[t], l2, wld, n[t], m_vec, 100), k)


@pytest.mark.parametrize("mode", ["intercept_h2", "no_intercept"])
def test_partitioned_constrained_intercept(ctx, mode):
    from ldsc_b200.partitioned import h2_partitioned
    m, k = 25_000, 3
    l2, wld = _annot_ld(m, k, 51)
    m_vec = np.array([2e4, 1e4, 3e4])
    chi2, n = _traits(l2, m_vec, 2, 52)
    kw = {"intercept_h2": 1.013} if mode == "intercept_h2" else {"no_intercept": True}
    fits = h2_partitioned(ctx, chi2, n, l2, wld, m_vec, 150, **kw)
    for t in range(2):
        want = R.fit_h2_partitioned(chi2[t], l2, wld, n[t], m_vec, 150, **kw)
        assert fits[t].est.shape == (k,)
        _check(fits[t], want, k)


def test_partitioned_fewer_snps_than_blocks(ctx):
    """A trait with fewer kept SNPs than --n-blocks uses one block per SNP
    (src/regressions.rs:1151) while the others keep 200."""
    from ldsc_b200.partitioned import h2_partitioned
    m, k = 5_000, 2
    l2, wld = _annot_ld(m, k, 61)
    m_vec = np.array([3e3, 2e3])
    chi2, n = _traits(l2, m_vec, 3, 62)
    chi2[1, 120:] = 1e6                       # 120 SNPs below the cut
    fits = h2_partitioned(ctx, chi2, n, l2, wld, m_vec, 200)
    for t in range(3):
        want = R.fit_h2_partitioned(chi2[t], l2, wld, n[t], m_vec, 200)
        if t == 1:
            assert want["n_obs"] <= 120 and want["n_blocks"] == want["n_obs"]
        else:
            assert want["n_blocks"] == 200
        _check(fits[t], want, k)


@pytest.mark.parametrize("k,fixed", [(63, False), (64, True), (127, False), (159, False)])
def test_partitioned_many_annotations(ctx, k, fixed):
    """Gram tile edges (P + 1 = 65, 65, 129) and the largest system (P = 160)."""
    from ldsc_b200.partitioned import h2_partitioned
    m = 12_000
    l2, wld = _annot_ld(m, k, 70 + k)
    m_vec = np.full(k, 1e3)
    chi2, n = _traits(l2, m_vec, 1, 80 + k)
    kw = {"no_intercept": True} if fixed else {}
    got = h2_partitioned(ctx, chi2[0], n[0], l2, wld, m_vec, 60, **kw)
    want = R.fit_h2_partitioned(chi2[0], l2, wld, n[0], m_vec, 60, **kw)
    # many near-collinear columns: the solves lose digits with the condition number
    cond = np.linalg.cond(want["cov"])
    tol = min(1e-4, 1e-13 * max(cond, 1.0))
    np.testing.assert_allclose(got.est, want["est"], rtol=max(RTOL, tol), atol=max(RTOL, tol) * np.abs(want["est"]).max())
    assert got.h2_total == pytest.approx(want["h2_total"], rel=max(RTOL, tol))


def test_partitioned_too_many_annotations_is_an_error(ctx):
    from ldsc_b200.api import LdscError
    from ldsc_b200.partitioned import h2_partitioned
    m, k = 2_000, 160
    l2, wld = _annot_ld(m, k, 90)
    with pytest.raises(LdscError):
        h2_partitioned(ctx, np.ones(m), 1e4, l2, wld, np.full(k, 10.0), 20)


def test_partitioned_device_tensors_equal_host_arrays(ctx):
    """Device pointers (the l2 run's (K, n_snp) output layout) give the same
    fit as host arrays: the same kernels on the same values."""
    import torch
    from ldsc_b200.partitioned import default_chisq_max, h2_partitioned, h2_partitioned_device
    m, k = 20_000, 4
    l2, wld = _annot_ld(m, k, 95)
    m_vec = np.array([2e4, 1e4, 5e3, 8e3])
    chi2, n = _traits(l2, m_vec, 3, 96)
    host = h2_partitioned(ctx, chi2, n, l2, wld, m_vec, 200)
    cmax = [default_chisq_max(chi2[t], n[t]) for t in range(3)]
    dev = h2_partitioned_device(ctx, torch.from_numpy(chi2).cuda(), torch.from_numpy(n).cuda(),
                                torch.from_numpy(np.ascontiguousarray(l2.T)).cuda(), torch.from_numpy(wld).cuda(),
                                m_vec, cmax, 200)
    for a, b in zip(host, dev):
        np.testing.assert_array_equal(a.est, b.est)
        np.testing.assert_array_equal(a.cov, b.cov)
        assert a.h2_total == b.h2_total and a.n_obs == b.n_obs


def test_partitioned_errors(ctx):
    """Every SNP above the chi2 cut, and an M vector of the wrong length, are
    errors (run_h2 stops on both: src/regressions.rs:530-533, 1131-1136)."""
    from ldsc_b200.api import LdscError
    from ldsc_b200.partitioned import h2_partitioned
    m, k = 3_000, 2
    l2, wld = _annot_ld(m, k, 97)
    with pytest.raises(LdscError):
        h2_partitioned(ctx, np.full(m, 500.0), 1e4, l2, wld, [1e3, 1e3], 20)
    with pytest.raises(ValueError):
        h2_partitioned(ctx, np.ones(m), 1e4, l2, wld, [1e3, 1e3, 1e3], 20)


def test_partitioned_trait_chunks_equal_single_calls(ctx):
    """A batch whose block Grams exceed one launch's budget (K = 159: 25
    traits per launch) runs in trait chunks; each trait's fit equals its fit
    alone, bit for bit."""
    from ldsc_b200.partitioned import h2_partitioned
    m, k, T = 6_000, 159, 30
    l2, wld = _annot_ld(m, k, 98)
    m_vec = np.full(k, 100.0)
    chi2, n = _traits(l2, m_vec, T, 99)
    batch = h2_partitioned(ctx, chi2, n, l2, wld, m_vec, 200)
    for t in (0, 24, 25, 29):
        one = h2_partitioned(ctx, chi2[t], n[t], l2, wld, m_vec, 200)
        np.testing.assert_array_equal(batch[t].est, one.est)
        np.testing.assert_array_equal(batch[t].delete_values, one.delete_values)
