"""Batched h2 / rg regressions on the device against the regression oracle
(src/h2.rs:258-458, src/regressions.rs:1612-2052, 2389-2465).

Tolerance: the device sums each jackknife block in its own order and solves
the 2 x 2 normal equations where the reference solves by QR, so estimates and
standard errors agree to a relative 1e-8; lambda_GC (an order statistic) is
exact.
"""
import math

import numpy as np
import pytest

from oracle import regress_oracle as R

pytestmark = pytest.mark.gpu

RTOL = 1e-8


def _ld(m, seed):
    rng = np.random.default_rng(seed)
    ld = 1.0 + rng.gamma(2.0, 20.0, m)
    wld = np.maximum(ld * rng.uniform(0.8, 1.2, m), 0.5)
    return ld, wld


def _close(a, b, rtol=RTOL, atol=0.0):
    if math.isnan(b):
        return math.isnan(a)
    return abs(a - b) <= atol + rtol * abs(b)


def _check_h2(got, want, fixed=False):
    for k in ("h2", "h2_se", "mean_chi2"):
        assert _close(got[k], want[k]), (k, got[k], want[k])
    assert got["lambda_gc"] == want["lambda_gc"]
    if fixed:
        assert got["intercept"] == want["intercept"] and math.isnan(got["intercept_se"])
        assert math.isnan(got["ratio"])
    else:
        for k in ("intercept", "intercept_se", "ratio", "ratio_se"):
            assert _close(got[k], want[k], atol=1e-12), (k, got[k], want[k])


@pytest.mark.parametrize("m", [50_001, 50_000])   # odd / even count for the median
def test_h2_batch_scalar_n(ctx, m):
    from ldsc_b200.api import h2_batch
    from ldsc_b200.synth import gwas_traits
    ld, wld = _ld(m, 1)
    big_m = 1e6
    chi2, n, _ = gwas_traits(ld, big_m, 5, seed=m)
    got = h2_batch(ctx, chi2, n, ld, wld, big_m, 200)
    for t in range(5):
        _check_h2(got[t], R.run_h2(chi2[t], ld, wld, n[t], big_m, 200))


def _lgc_case(kind, rng):
    if kind == "small_odd":          # fewer keys than the shared-memory capacity
        return rng.chisquare(1, 7)
    if kind == "at_capacity":
        return rng.chisquare(1, 2048)
    if kind == "above_capacity":
        return rng.chisquare(1, 2050)
    if kind == "split_octaves":      # the middle ranks fall in different buckets of the first digit
        return rng.permutation(np.concatenate([rng.uniform(1.0, 2.0, 5000), rng.uniform(4.0, 8.0, 5000)]))
    if kind == "all_equal":          # the prefix never narrows: every digit is taken
        return np.full(10_000, 3.0)
    if kind == "few_values":         # ties far above the capacity, odd count
        return rng.integers(0, 6, 50_001).astype(np.float64)
    if kind == "signed_zeros":       # y enters as given: negative values, -0.0 and 0.0 order exactly
        return rng.choice(np.array([-1.5, -0.0, 0.0, 2.5]), 20_000)
    raise ValueError(kind)


@pytest.mark.parametrize("kind", ["small_odd", "at_capacity", "above_capacity", "split_octaves", "all_equal",
                                  "few_values", "signed_zeros"])
def test_lambda_gc_median_edge_cases(ctx, kind):
    """lambda_GC = median(chi2) / 0.4549 (src/h2.rs:394-414) is an exact order
    statistic: equal to numpy's median on ties, split buckets, capacity edges
    and signed zeros."""
    from ldsc_b200.api import h2_batch
    rng = np.random.default_rng(sum(map(ord, kind)))
    chi2 = _lgc_case(kind, rng)
    m = len(chi2)
    ld, wld = _ld(m, 21)
    got = h2_batch(ctx, np.stack([chi2, chi2[::-1].copy()]), [1e5, 1e5], ld, wld, 1e6, min(5, m - 1))
    want = np.median(chi2) / 0.4549
    for t in range(2):
        assert got[t]["lambda_gc"] == want, (kind, t, got[t]["lambda_gc"], want)


def test_h2_batch_per_snp_n_and_fixed_intercept(ctx):
    from ldsc_b200.api import h2_batch
    from ldsc_b200.synth import gwas_traits
    m = 30_000
    ld, wld = _ld(m, 2)
    chi2, n, _ = gwas_traits(ld, 5e5, 3, seed=3)
    rng = np.random.default_rng(4)
    nv = n[:, None] * rng.uniform(0.7, 1.0, (3, m))
    got = h2_batch(ctx, chi2, nv, ld, wld, 5e5, 100)
    for t in range(3):
        _check_h2(got[t], R.run_h2(chi2[t], ld, wld, nv[t], 5e5, 100))
    got = h2_batch(ctx, chi2, n, ld, wld, 5e5, 100, intercept=1.02)
    for t in range(3):
        _check_h2(got[t], R.run_h2(chi2[t], ld, wld, n[t], 5e5, 100, fixed_intercept=1.02), fixed=True)


def test_h2_batch_more_blocks_than_snps_clamps(ctx):
    from ldsc_b200.api import h2_batch
    from ldsc_b200.synth import gwas_traits
    m = 150
    ld, wld = _ld(m, 5)
    chi2, n, _ = gwas_traits(ld, 1e5, 2, seed=6)
    got = h2_batch(ctx, chi2, n, ld, wld, 1e5, 200)
    for t in range(2):
        _check_h2(got[t], R.run_h2(chi2[t], ld, wld, n[t], 1e5, 200))


def test_h2_batch_many_traits(ctx):
    from ldsc_b200.api import h2_batch
    from ldsc_b200.synth import gwas_traits
    m = 20_000
    ld, wld = _ld(m, 7)
    chi2, n, _ = gwas_traits(ld, 1e6, 64, seed=8)
    got = h2_batch(ctx, chi2, n, ld, wld, 1e6, 200)
    for t in (0, 17, 63):
        _check_h2(got[t], R.run_h2(chi2[t], ld, wld, n[t], 1e6, 200))


def test_h2_batch_device_pointers(ctx):
    import torch
    from ldsc_b200 import _lib as L
    from ldsc_b200.api import h2_batch
    from ldsc_b200.synth import gwas_traits
    import ctypes as C
    m = 10_000
    ld, wld = _ld(m, 9)
    chi2, n, _ = gwas_traits(ld, 1e6, 2, seed=10)
    host = h2_batch(ctx, chi2, n, ld, wld, 1e6, 50)
    dev = {k: torch.from_numpy(np.ascontiguousarray(v, dtype=np.float64)).cuda()
           for k, v in dict(chi2=chi2, n=n, ld=ld, wld=wld).items()}
    torch.cuda.synchronize()
    args = L.H2Args(n_snp=m, n_traits=2, n_blocks=50, chi2=dev["chi2"].data_ptr(), n_per_snp=None,
                    n_scalar=dev["n"].data_ptr(), ref_l2=dev["ld"].data_ptr(), w_l2=dev["wld"].data_ptr(),
                    m_snps=1e6, fixed_intercept=0, intercept=0.0, want_lambda_gc=1, device_pointers=1)
    out = (L.H2Result * 2)()
    ctx.check(ctx.lib.ldsc_h2_batch(ctx.h, C.byref(args), C.cast(out, C.c_void_p)))
    for t in range(2):
        for f, _ in L.H2Result._fields_:
            a, b = getattr(out[t], f), host[t][f]
            assert (math.isnan(a) and math.isnan(b)) or a == b, f


def test_rg_batch(ctx):
    from ldsc_b200.api import rg_batch
    from ldsc_b200.synth import gwas_pairs
    m = 40_000
    ld, wld = _ld(m, 11)
    z1, z2, n1, n2, _ = gwas_pairs(ld, 2e5, 4, seed=12)
    got = rg_batch(ctx, z1, z2, n1, n2, ld, wld, 2e5, 200)
    for p in range(4):
        want = R.run_rg(z1[p], z2[p], ld, wld, n1[p], n2[p], 2e5, 200)
        for k in ("rg", "rg_se", "gencov", "gencov_se", "gencov_intercept", "gencov_intercept_se",
                  "h2_1", "h2_1_se", "h2_2", "h2_2_se", "mean_z1z2", "z"):
            assert _close(got[p][k], want[k], rtol=1e-7, atol=1e-12), (p, k, got[p][k], want[k])
        assert _close(got[p]["p"], want["p"], rtol=1e-5, atol=1e-300)


def test_rg_negative_h2_gives_nan(ctx):
    from ldsc_b200.api import rg_batch
    m = 5000
    ld, wld = _ld(m, 13)
    rng = np.random.default_rng(14)
    # trait 1's chi^2 falls with LD score: its fitted h2 is negative
    z1 = np.sqrt(np.maximum(1.2 - 0.004 * ld, 0.05)) * rng.standard_normal(m)
    z2 = rng.standard_normal(m)
    got = rg_batch(ctx, z1[None], z2[None], 1e5, 1e5, ld, wld, 1e6, 50)[0]
    want = R.run_rg(z1, z2, ld, wld, 1e5, 1e5, 1e6, 50)
    assert want["h2_1"] < 0 and math.isnan(want["rg"])
    assert math.isnan(got["rg"])
    assert _close(got["h2_1"], want["h2_1"], rtol=1e-7, atol=1e-12)
    assert got["z"] == math.inf and got["p"] == 0.0


def test_regression_errors(ctx):
    from ldsc_b200.api import LdscError, h2_batch
    ld = np.ones(10)
    with pytest.raises(LdscError, match="n_blocks"):
        h2_batch(ctx, np.ones((1, 10)), [1e4], ld, ld, 10.0, 1)
    with pytest.raises(LdscError, match="M must be"):
        h2_batch(ctx, np.ones((1, 10)), [1e4], ld, ld, 0.0, 5)


@pytest.mark.parametrize("cutoff", [30.0, 8.0])
def test_h2_batch_two_step(ctx, cutoff):
    """--two-step (src/h2.rs:319-393): intercept from chi2 < cutoff, slope
    refit on all SNPs, combined delete values."""
    from ldsc_b200.api import h2_batch
    from ldsc_b200.synth import gwas_traits
    m = 40_000
    ld, wld = _ld(m, 15)
    chi2, n, _ = gwas_traits(ld, 2e5, 4, seed=16)
    got = h2_batch(ctx, chi2, n, ld, wld, 2e5, 200, two_step=cutoff)
    for t in range(4):
        want = R.run_h2(chi2[t], ld, wld, n[t], 2e5, 200, two_step=cutoff)
        for k in ("h2", "h2_se", "intercept", "intercept_se", "mean_chi2", "ratio", "ratio_se"):
            assert _close(got[t][k], want[k], atol=1e-12), (t, k, got[t][k], want[k])
        assert got[t]["lambda_gc"] == want["lambda_gc"]


def test_h2_batch_two_step_errors(ctx):
    from ldsc_b200.api import LdscError, h2_batch
    m = 1000
    ld, wld = _ld(m, 17)
    chi2 = np.full((1, m), 50.0)
    chi2[0, :100] = 1.0                                  # 100 SNPs below the cutoff, 200 blocks asked
    with pytest.raises(LdscError, match="More blocks than data points"):
        h2_batch(ctx, chi2, [1e5], ld, wld, 1e6, 200, two_step=30.0)
    with pytest.raises(LdscError, match="constrained intercept"):
        h2_batch(ctx, chi2, [1e5], ld, wld, 1e6, 50, two_step=30.0, intercept=1.0)
