"""Partitioned h2: the oracle against closed-form cases, and the host-side
report code (ldsc_b200.partitioned) against the oracle (CPU only).

The reference carries no known-answer fixture for partitioned h2
(src/regressions.rs:1121-1493), so the oracle is pinned by algebra: a
noise-free K-annotation model returns its per-annotation coefficients, the
chi2 cut equals dropping those SNPs, and with disjoint annotations the
overlap figures reduce to the plain proportions.
"""
import math

import numpy as np
import pytest

from oracle import regress_oracle as R


def _annot_ld(m, k, seed):
    rng = np.random.default_rng(seed)
    base = 1.0 + rng.gamma(2.0, 15.0, m)
    frac = rng.dirichlet(np.ones(k), size=m) * rng.uniform(0.5, 1.5, (m, k))
    l2 = base[:, None] * frac
    wld = np.maximum(base * rng.uniform(0.8, 1.2, m), 0.5)
    return l2, wld


@pytest.mark.parametrize("per_snp_n", [False, True])
def test_noise_free_partitioned_model_returns_its_coefficients(per_snp_n):
    rng = np.random.default_rng(11)
    m, k = 5000, 4
    l2, wld = _annot_ld(m, k, 3)
    n = rng.uniform(2e4, 6e4, m) if per_snp_n else np.full(m, 3e4)
    tau = np.array([2e-6, 5e-7, 0.0, 1.2e-6])
    a = 1.04
    chi2 = a + n * (l2 @ tau)
    m_vec = np.array([1e4, 2e4, 3e4, 4e4])
    f = R.fit_h2_partitioned(chi2, l2, wld, n, m_vec, 40)
    assert f["n_obs"] == m and f["n_blocks"] == 40
    np.testing.assert_allclose(f["est"][:k] / f["n_mean"], tau, rtol=1e-9, atol=1e-15)
    assert f["intercept"] == pytest.approx(a, rel=1e-10)
    np.testing.assert_allclose(f["h2_annot"], tau * m_vec, rtol=1e-9, atol=1e-12)
    assert f["h2_total"] == pytest.approx(float(np.sum(tau * m_vec)), rel=1e-9)
    assert f["h2_total_se"] < 1e-8 and f["intercept_se"] < 1e-8


def test_fixed_intercept_noise_free():
    m, k = 3000, 3
    l2, wld = _annot_ld(m, k, 4)
    tau = np.array([1e-6, 3e-6, 2e-7])
    chi2 = 1.0 + 5e4 * (l2 @ tau)
    f = R.fit_h2_partitioned(chi2, l2, wld, 5e4, [1e4, 1e4, 1e4], 30, no_intercept=True)
    assert f["est"].shape == (k,) and f["intercept"] == 1.0 and math.isnan(f["intercept_se"])
    np.testing.assert_allclose(f["est"] / f["n_mean"], tau, rtol=1e-9)


def test_chisq_cut_equals_dropping_the_snps():
    rng = np.random.default_rng(12)
    m, k = 2000, 3
    l2, wld = _annot_ld(m, k, 5)
    chi2 = rng.chisquare(1, m) * 1.5
    n = np.full(m, 2e4)            # default cut-off max(0.001 * 2e4, 80) = 80
    m_vec = [5e3, 5e3, 5e3]
    want = R.fit_h2_partitioned(chi2, l2, wld, n, m_vec, 25)
    bad = np.array([7, 100, 1500])
    chi2b = chi2.copy()
    chi2b[bad[:2]] = [80.0, 400.0]  # not below the cut
    chi2b[bad[2]] = np.nan
    got = R.fit_h2_partitioned(chi2b, l2, wld, n, m_vec, 25)
    keep = np.setdiff1d(np.arange(m), bad)
    ref = R.fit_h2_partitioned(chi2[keep], l2[keep], wld[keep], n[keep], m_vec, 25)
    assert got["n_obs"] == m - 3
    for key in ("est", "cov", "delete_values", "h2_annot"):
        np.testing.assert_array_equal(got[key], ref[key])
    assert want["n_obs"] == m


def test_overlap_figures_disjoint_annotations():
    rng = np.random.default_rng(13)
    m, k = 3000, 3
    l2, wld = _annot_ld(m, k, 6)
    chi2 = 1.0 + rng.chisquare(1, m) * (1 + l2.sum(1) / 50)
    m_vec = np.array([2e3, 5e3, 3e3])
    f = R.fit_h2_partitioned(chi2, l2, wld, 4e4, m_vec, 30)
    fig = R.overlap_figures(f, np.diag(m_vec), float(m_vec.sum()))
    prop = f["h2_annot"] / f["h2_total"]
    np.testing.assert_allclose(fig["prop_h2"], prop, rtol=1e-12)
    np.testing.assert_allclose(fig["prop_m"], m_vec / m_vec.sum(), rtol=1e-15)
    np.testing.assert_allclose(fig["enrichment"], prop / (m_vec / m_vec.sum()), rtol=1e-12)
    np.testing.assert_allclose(fig["coef"], f["est"][:k] / f["n_mean"], rtol=1e-15)


def _product_fit(f):
    from ldsc_b200.partitioned import PartitionedFit
    return PartitionedFit(est=f["est"], cov=f["cov"], delete_values=f["delete_values"], m_vec=f["m_vec"],
                          n_mean=f["n_mean"], h2_annot=f["h2_annot"], h2_total=f["h2_total"],
                          h2_total_se=f["h2_total_se"], intercept=f["intercept"], intercept_se=f["intercept_se"],
                          mean_chi2=f["mean_chi2"], n_obs=f["n_obs"], n_blocks=f["n_blocks"])


def test_host_overlap_figures_match_oracle():
    from ldsc_b200 import partitioned as P
    rng = np.random.default_rng(14)
    m, k = 4000, 4
    l2, wld = _annot_ld(m, k, 7)
    chi2 = rng.chisquare(1, m) * (1 + l2 @ np.array([0.02, 0.01, 0.0, 0.03]))
    m_vec = np.array([4e3, 2e3, 1e3, 6e3])
    f = R.fit_h2_partitioned(chi2, l2, wld, 5e4, m_vec, 50)
    ov = np.diag(m_vec).copy()
    ov[0, 1] = ov[1, 0] = 500.0
    ov[2, 3] = ov[3, 2] = 800.0
    m_tot = 9e3
    want = R.overlap_figures(f, ov, m_tot)
    got = P.overlap_figures(_product_fit(f), ov, m_tot)
    for key in want:
        np.testing.assert_allclose(got[key], want[key], rtol=1e-12, atol=1e-15, err_msg=key)


def test_results_file_layout(tmp_path):
    from ldsc_b200 import partitioned as P
    rng = np.random.default_rng(15)
    m, k = 2000, 2
    l2, wld = _annot_ld(m, k, 8)
    chi2 = rng.chisquare(1, m) * (1 + l2.sum(1) / 40)
    m_vec = np.array([1e3, 1e3])
    f = _product_fit(R.fit_h2_partitioned(chi2, l2, wld, 3e4, m_vec, 20))
    # m_tot == M_0: category 0's difference row is skipped, its SE is 0 -> "NA"
    path = P.write_overlap_results(str(tmp_path / "o"), f, ["A", "B"], np.diag(m_vec), 1e3, True)
    lines = open(path).read().splitlines()
    assert lines[0].split("\t") == ["Category", "Prop._SNPs", "Prop._h2", "Prop._h2_std_error", "Enrichment",
                                    "Enrichment_std_error", "Enrichment_p", "Coefficient",
                                    "Coefficient_std_error", "Coefficient_z-score"]
    row = lines[1].split("\t")
    assert row[0] == "A" and row[6] == "NA" and row[1] == "1.000000"
    assert "e" in row[7] and "e-0" not in row[7]


def test_rust_exponent_format():
    from ldsc_b200.partitioned import _rust_exp
    assert _rust_exp(1.23456789e-5, 4) == "1.2346e-5"
    assert _rust_exp(300.0, 4) == "3.0000e2"
    assert _rust_exp(0.0, 4) == "0.0000e0"
    assert _rust_exp(-2.5e10, 6) == "-2.500000e10"
    assert _rust_exp(float("nan"), 4) == "NaN"


def test_default_chisq_max():
    from ldsc_b200.partitioned import default_chisq_max
    assert default_chisq_max(np.ones(3), np.array([1e4, 2e5, np.nan])) == pytest.approx(200.0)
    assert default_chisq_max(np.array([1.0, np.nan]), np.array([1e4, 9e5])) == 80.0
