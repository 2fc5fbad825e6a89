"""The regression oracle against closed-form cases (CPU only).

The reference carries no known-answer fixture for the regressions, so the
oracle is pinned by cases whose answers follow from the algebra: a noise-free
LD-score model returns its generating parameters, the fast jackknife equals
explicit delete-one-block refits, and the separators follow
src/h2.rs:31-58 by hand.
"""
import math

import numpy as np
import pytest

from oracle import regress_oracle as R


def test_separators_by_hand():
    assert R.get_separators(10, 3) == [0, 3, 6, 10]
    assert R.get_separators(7, 7) == list(range(8))
    mask = np.array([True, False, True, True, False, True, True])
    # 5 kept rows, blocks [0,2,5) over kept indices -> positions in the full vector
    assert R.update_separators([0, 2, 5], mask) == [0, 3, 7]


def test_jackknife_se_cov_by_hand():
    est = np.array([2.0])
    dele = np.array([[1.0], [2.0], [3.0]])
    se, cov = R.jackknife_se_cov(est, dele)
    pseudo = 3 * 2.0 - 2 * dele[:, 0]            # 4, 2, 0
    want = np.sum((pseudo - pseudo.mean()) ** 2) / (2 * 3)
    assert cov[0, 0] == pytest.approx(want)
    assert se[0] == pytest.approx(math.sqrt(want))


def test_fast_jackknife_matches_explicit_refits():
    rng = np.random.default_rng(4)
    x = np.stack([rng.gamma(2, 3, 300), np.ones(300)], axis=1)
    y = 0.7 * x[:, 0] + 1.3 + rng.standard_normal(300)
    jk = R.jackknife_fast(x, y, 12)
    seps = jk["separators"]
    for b in range(12):
        keep = np.ones(300, bool)
        keep[seps[b]:seps[b + 1]] = False
        ref = np.linalg.lstsq(x[keep], y[keep], rcond=None)[0]
        np.testing.assert_allclose(jk["delete_values"][b], ref, rtol=1e-10)
    np.testing.assert_allclose(jk["est"], np.linalg.lstsq(x, y, rcond=None)[0], rtol=1e-10)


@pytest.mark.parametrize("per_snp_n", [False, True])
def test_noise_free_model_returns_its_parameters(per_snp_n):
    rng = np.random.default_rng(5)
    m = 4000
    ld = 1.0 + rng.gamma(2.0, 15.0, m)
    n = rng.uniform(2e4, 6e4, m) if per_snp_n else np.full(m, 3e4)
    h2, a = 0.31, 1.07
    chi2 = a + n * h2 * ld / m
    r = R.run_h2(chi2, ld, ld, n, m, 50)
    assert r["h2"] == pytest.approx(h2, rel=1e-10)
    assert r["intercept"] == pytest.approx(a, rel=1e-10)
    assert r["h2_se"] < 1e-8 and r["intercept_se"] < 1e-8
    fixed = R.run_h2(chi2, ld, ld, n, m, 50, fixed_intercept=a)
    assert fixed["h2"] == pytest.approx(h2, rel=1e-10)
    assert math.isnan(fixed["intercept_se"]) and math.isnan(fixed["ratio"])
    assert r["ratio"] == pytest.approx((a - 1) / (chi2.mean() - 1), rel=1e-9)
    assert r["lambda_gc"] == pytest.approx(np.median(chi2) / 0.4549)


def test_noise_free_gencov_returns_its_parameters():
    rng = np.random.default_rng(6)
    m = 3000
    ld = 1.0 + rng.gamma(2.0, 15.0, m)
    n1, n2, rho, ci = 4e4, 2.5e4, 0.12, 0.03
    prod = ci + math.sqrt(n1 * n2) * rho * ld / m
    z1 = np.sqrt(np.abs(prod)) * np.sign(prod)
    z2 = np.sqrt(np.abs(prod))
    h = dict(h2=0.3, intercept=1.0)
    g = R.run_gencov(z1, z2, ld, ld, n1, n2, m, 40, h, h)
    assert g["tot"] == pytest.approx(rho, rel=1e-9)
    assert g["intercept"] == pytest.approx(ci, rel=1e-8)


def test_ratio_jackknife_nan_becomes_zero_se():
    # f64::max(NaN, 0) is 0 in the reference, so a NaN pseudovalue gives se 0
    assert R.ratio_jackknife(0.5, np.array([1.0, 2.0, 3.0]), np.array([1.0, 0.0, 2.0])) == 0.0


def test_two_step_runs_and_stays_near_one_step():
    rng = np.random.default_rng(7)
    m = 6000
    ld = 1.0 + rng.gamma(2.0, 15.0, m)
    n, big_m = 5e4, 1e6      # mean chi2 near 1.3, few SNPs above the cut
    z = np.sqrt(n * 0.2 * ld / big_m) * rng.standard_normal(m) + rng.standard_normal(m)
    chi2 = z * z
    one = R.run_h2(chi2, ld, ld, n, big_m, 100)
    two = R.run_h2(chi2, ld, ld, n, big_m, 100, two_step=30.0)
    assert abs(one["h2"] - two["h2"]) < 4 * one["h2_se"]
    assert np.isfinite(two["h2_se"]) and np.isfinite(two["intercept_se"])


def test_rg_recovers_a_strong_correlation():
    from ldsc_b200.synth import gwas_pairs
    rng = np.random.default_rng(8)
    m = 20000
    ld = 1.0 + rng.gamma(2.0, 20.0, m)
    z1, z2, n1, n2, rg = gwas_pairs(ld, m, 2, seed=9)
    for p in range(2):
        r = R.run_rg(z1[p], z2[p], ld, ld, n1[p], n2[p], m, 100)
        assert abs(r["rg"] - rg[p]) < 5 * r["rg_se"] + 0.02
        assert r["p"] == pytest.approx(math.erfc(abs(r["z"]) / math.sqrt(2)))
