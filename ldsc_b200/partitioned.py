"""Partitioned (stratified) h2: run_h2's K > 1 branch (src/regressions.rs:561-630).

The fit itself -- weights from the summed LD score, the weighted Gram of the
K-column design per jackknife block, the block-deleted solves and the
jackknife covariance -- runs on the device (`ldsc_h2_partitioned`).  The
reports built from it are K x K host arithmetic, as in the reference:
print_partitioned_summary (src/regressions.rs:1228-1260),
print_jackknife_diagnostics (src/regressions.rs:2610-2638) and
write_overlap_results (src/regressions.rs:1262-1493).
"""
from __future__ import annotations

import ctypes as C
import dataclasses
import math
from typing import List, Optional, Sequence

import numpy as np

from . import _lib as L
from .api import LdscError
from .io import rust_f64


@dataclasses.dataclass
class PartitionedFit:
    """PartitionedFit (src/regressions.rs:1054-1065) plus the total's SE."""
    est: np.ndarray            # P: coefficient x nbar per annotation, then the intercept (free only)
    cov: np.ndarray            # P x P jackknife covariance of est
    delete_values: np.ndarray  # n_blocks x P
    m_vec: np.ndarray          # K
    n_mean: float
    h2_annot: np.ndarray       # K
    h2_total: float
    h2_total_se: float
    intercept: float
    intercept_se: float        # NaN when constrained
    mean_chi2: float
    n_obs: int
    n_blocks: int

    @property
    def coef(self) -> np.ndarray:
        return self.est[:len(self.m_vec)] / self.n_mean


def default_chisq_max(chi2: np.ndarray, n: np.ndarray) -> float:
    """run_h2's K > 1 cut-off max(0.001 max N, 80), N over the SNPs whose chi2
    and N are present (src/regressions.rs:577-593)."""
    chi2 = np.asarray(chi2, dtype=np.float64)
    n = np.broadcast_to(np.asarray(n, dtype=np.float64), chi2.shape)
    ok = ~np.isnan(chi2) & ~np.isnan(n)
    max_n = 0.0
    if ok.any():
        mx = float(np.max(n[ok]))
        max_n = mx if mx > 0.0 else 0.0
    return max(0.001 * max_n, 80.0)


def _call(ctx, chi2, n, ref_l2, w_l2, m_vec, n_blocks, fixed, chisq_max, device=None) -> List[PartitionedFit]:
    """One ldsc_h2_partitioned call.  Host arrays, or with device = (T, m, K,
    per_snp, ref_ld) the first four arguments are device pointers (ints)."""
    if device is None:
        T, m = chi2.shape
        K = ref_l2.shape[1]
        per_snp = n.ndim == 2
        ptrs = (chi2.ctypes.data, n.ctypes.data, ref_l2.ctypes.data, w_l2.ctypes.data)
        ref_ld = m
    else:
        T, m, K, per_snp, ref_ld = device
        ptrs = (chi2, n, ref_l2, w_l2)
    P = K + (0 if fixed is not None else 1)
    cmax = np.ascontiguousarray(chisq_max, dtype=np.float64)
    est = np.zeros((T, P))
    cov = np.zeros((T, P, P))
    dv = np.zeros((T, n_blocks, P))
    h2a = np.zeros((T, K))
    args = L.H2PArgs(n_snp=m, n_traits=T, n_annot=K, n_blocks=n_blocks, chi2=ptrs[0],
                     n_per_snp=ptrs[1] if per_snp else None, n_scalar=None if per_snp else ptrs[1],
                     ref_l2=ptrs[2], ref_ld=ref_ld, w_l2=ptrs[3], m_vec=m_vec.ctypes.data,
                     fixed_intercept=int(fixed is not None), intercept=float(fixed or 0.0),
                     chisq_max=cmax.ctypes.data, device_pointers=int(device is not None), est=est.ctypes.data,
                     cov=cov.ctypes.data, delete_values=dv.ctypes.data, h2_annot=h2a.ctypes.data)
    out = (L.H2PResult * T)()
    ctx.check(ctx.lib.ldsc_h2_partitioned(ctx.h, C.byref(args), C.cast(out, C.c_void_p)))
    fits = []
    for t, r in enumerate(out):
        nb = int(r.n_blocks)
        fits.append(PartitionedFit(est=est[t], cov=cov[t], delete_values=dv[t, :nb], m_vec=m_vec.copy(),
                                   n_mean=r.n_mean, h2_annot=h2a[t], h2_total=r.h2_total, h2_total_se=r.h2_total_se,
                                   intercept=r.intercept, intercept_se=r.intercept_se, mean_chi2=r.mean_chi2,
                                   n_obs=int(r.n_obs), n_blocks=nb))
    return fits


def h2_partitioned(ctx, chi2, n, ref_l2, w_l2, m_vec, n_blocks: int = 200, intercept_h2: Optional[float] = None,
                   no_intercept: bool = False, chisq_max: Optional[float] = None):
    """Partitioned h2 of one trait (chi2: n_snp) or many (chi2: T x n_snp)
    against the n_snp x K LD scores `ref_l2`.  n: scalar / T scalars, or per
    SNP (n_snp or T x n_snp).  SNPs with a missing chi2 or N are dropped, then
    those with chi2 >= chisq_max (default: run_h2's K > 1 rule per trait).
    Returns a PartitionedFit (a list of them for 2-D chi2)."""
    single = np.ndim(chi2) == 1
    chi2 = np.ascontiguousarray(np.atleast_2d(chi2), dtype=np.float64)
    T, m = chi2.shape
    ref_l2 = np.asarray(ref_l2, dtype=np.float64)
    if ref_l2.ndim == 1:
        ref_l2 = ref_l2[:, None]
    if ref_l2.shape[0] != m:
        raise ValueError(f"ref_l2 has {ref_l2.shape[0]} rows for {m} SNPs")
    ref_l2 = np.asfortranarray(ref_l2)
    w_l2 = np.ascontiguousarray(w_l2, dtype=np.float64)
    m_vec = np.ascontiguousarray(np.atleast_1d(m_vec), dtype=np.float64)
    if m_vec.shape[0] != ref_l2.shape[1]:
        raise ValueError(f"M vector length {m_vec.shape[0]} does not match K={ref_l2.shape[1]}")
    fixed = intercept_h2 if intercept_h2 is not None else (1.0 if no_intercept else None)
    n = np.asarray(n, dtype=np.float64)
    # per-SNP sample sizes: n_snp values for one trait, T x n_snp for many
    per_snp = n.ndim == 2 or (n.ndim == 1 and single and n.shape[0] == m)
    if per_snp:
        n = np.ascontiguousarray(np.broadcast_to(n, (T, m)))
    else:
        n = np.ascontiguousarray(np.broadcast_to(n, (T,)))
    nfull = n if per_snp else np.broadcast_to(n[:, None], (T, m))
    if chisq_max is None:
        cmax = np.array([default_chisq_max(chi2[t], nfull[t]) for t in range(T)])
    else:
        cmax = np.full(T, float(chisq_max))
    fits: List[Optional[PartitionedFit]] = [None] * T
    # traits with a missing N drop those SNPs on the host and run alone
    bad = [t for t in range(T) if per_snp and np.isnan(n[t]).any()]
    good = [t for t in range(T) if t not in bad]
    if good:
        sub = _call(ctx, np.ascontiguousarray(chi2[good]), np.ascontiguousarray(n[good]), ref_l2, w_l2, m_vec,
                    n_blocks, fixed, cmax[good])
        for t, f in zip(good, sub):
            fits[t] = f
    for t in bad:
        keep = ~np.isnan(n[t])
        f = _call(ctx, np.ascontiguousarray(chi2[t:t + 1, keep]), np.ascontiguousarray(n[t:t + 1, keep]),
                  np.asfortranarray(ref_l2[keep]), np.ascontiguousarray(w_l2[keep]), m_vec, n_blocks, fixed,
                  cmax[t:t + 1])
        fits[t] = f[0]
    return fits[0] if single else fits


def h2_partitioned_device(ctx, chi2, n, ref_l2, w_l2, m_vec, chisq_max, n_blocks: int = 200,
                          intercept_h2: Optional[float] = None, no_intercept: bool = False) -> List[PartitionedFit]:
    """Partitioned h2 on device-resident CUDA tensors: chi2 (T, n_snp), n
    (T,) scalar sample sizes or (T, n_snp), ref_l2 (K, n_snp) row-major (=
    n_snp x K column-major, as the l2 run's device output), w_l2 (n_snp,),
    all float64.  chisq_max: T cut-offs (host); the caller applies any
    missing-N filter."""
    T, m = int(chi2.shape[0]), int(chi2.shape[1])
    K = int(ref_l2.shape[0])
    for t, shape in ((chi2, (T, m)), (ref_l2, (K, m)), (w_l2, (m,))):
        if tuple(t.shape) != shape or not t.is_contiguous() or not t.is_cuda:
            raise LdscError(L.LDSC_E_INVALID, "h2_partitioned_device wants contiguous float64 CUDA tensors")
    per_snp = n.dim() == 2
    if tuple(n.shape) != ((T, m) if per_snp else (T,)) or not n.is_cuda:
        raise LdscError(L.LDSC_E_INVALID, "n must be a (T,) or (T, n_snp) float64 CUDA tensor")
    fixed = intercept_h2 if intercept_h2 is not None else (1.0 if no_intercept else None)
    m_vec = np.ascontiguousarray(np.atleast_1d(m_vec), dtype=np.float64)
    cmax = np.broadcast_to(np.asarray(chisq_max, dtype=np.float64), (T,))
    return _call(ctx, chi2.data_ptr(), n.data_ptr(), ref_l2.data_ptr(), w_l2.data_ptr(), m_vec, n_blocks, fixed,
                 cmax, device=(T, m, K, per_snp, m))


def _rust_exp(v: float, prec: int) -> str:
    """Rust's `{:.Ne}` of an f64: mantissa with N decimals, exponent without
    sign padding (1.2346e-5, 3.0000e2)."""
    if math.isnan(v):
        return "NaN"
    if math.isinf(v):
        return "inf" if v > 0 else "-inf"
    s = f"{v:.{prec}e}"
    mant, exp = s.split("e")
    return f"{mant}e{int(exp)}"


def _f(v: float, prec: int) -> str:
    """Rust's `{:.N}` of an f64 (NaN / inf spelled as Rust does)."""
    if math.isnan(v):
        return "NaN"
    if math.isinf(v):
        return "inf" if v > 0 else "-inf"
    return f"{v:.{prec}f}"


def print_partitioned_summary(fit: PartitionedFit, names: Sequence[str], print_coefficients: bool = False,
                              overlap_annot: bool = False) -> None:
    """print_partitioned_summary (src/regressions.rs:1228-1260)."""
    print(f"Total observed-scale h2: {_f(fit.h2_total, 4)}")
    print(f"Intercept: {_f(fit.intercept, 4)}")
    if print_coefficients and not overlap_annot:
        m_total = float(np.sum(fit.m_vec))
        print()
        print(f"{'Category':<35} {'Prop_h2':>10} {'Prop_SNPs':>10} {'Enrichment':>12} {'Coefficient':>14}")
        print("-" * 83)
        for j, name in enumerate(names):
            prop_h2 = fit.h2_annot[j] / fit.h2_total if abs(fit.h2_total) > 1e-12 else float("nan")
            prop_m = fit.m_vec[j] / m_total
            enr = prop_h2 / prop_m if prop_m > 1e-12 else float("nan")
            coeff = fit.est[j] / fit.n_mean
            print(f"{name:<35} {_f(prop_h2, 4):>10} {_f(prop_m, 4):>10} {_f(enr, 4):>12} "
                  f"{_rust_exp(coeff, 4):>14}")
        print()


def print_jackknife_diagnostics(fit: PartitionedFit, print_cov: bool, print_delete_vals: bool) -> None:
    """print_jackknife_diagnostics (src/regressions.rs:2610-2638)."""
    if print_cov:
        p = fit.cov.shape[0]
        print(f"\nJackknife covariance matrix ({p}×{p}):")
        for i in range(p):
            print("  " + "  ".join(_rust_exp(float(v), 6) for v in fit.cov[i]))
    if print_delete_vals:
        dv = fit.delete_values
        print(f"\nJackknife delete values ({dv.shape[0]} blocks × {dv.shape[1]} params):")
        for b in range(dv.shape[0]):
            print(f"  Block {b:3}: " + "  ".join(_f(float(v), 6) for v in dv[b]))


def _ratio_jackknife_cov(est: np.ndarray, numer: np.ndarray, denom: np.ndarray) -> np.ndarray:
    """ratio_jackknife's covariance (src/regressions.rs:1067-1120)."""
    nb = numer.shape[0]
    with np.errstate(divide="ignore", invalid="ignore"):
        pseudo = np.where(denom == 0.0, np.nan, nb * est[None, :] - (nb - 1.0) * (numer / denom))
    c = pseudo - pseudo.sum(axis=0) / nb
    cov = c.T @ c
    scale = (nb - 1.0) * nb
    return cov / scale if scale > 0.0 else cov


def _se(diag: np.ndarray) -> np.ndarray:
    # f64::max(v, 0.0).sqrt(): NaN -> 0
    d = np.where(diag > 0.0, diag, 0.0)
    return np.sqrt(d)


def overlap_figures(fit: PartitionedFit, overlap: np.ndarray, m_tot: float) -> dict:
    """The per-category figures of write_overlap_results
    (src/regressions.rs:1262-1440): Prop._SNPs, Prop._h2 and its SE,
    Enrichment and its SE, the t statistic of the coefficient difference
    (diff_na where its SE is 0), the coefficients and their SEs."""
    k = len(fit.m_vec)
    overlap = np.asarray(overlap, dtype=np.float64)
    if overlap.shape != (k, k):
        raise ValueError(f"Overlap matrix shape {overlap.shape[0]}x{overlap.shape[1]} does not match K={k}")
    m_vec, nm = fit.m_vec, fit.n_mean
    coef = fit.est[:k] / nm
    coef_cov = fit.cov[:k, :k] / (nm * nm)
    coef_se = _se(np.diag(coef_cov))
    if abs(fit.h2_total) > 1e-12:
        prop = fit.h2_annot / fit.h2_total
    else:
        prop = np.full(k, np.nan)
    numer = m_vec[None, :] * fit.delete_values[:, :k] / nm
    denom = np.repeat(numer.sum(axis=1, keepdims=True), k, axis=1)
    prop_cov = _ratio_jackknife_cov(prop, numer, denom)
    overlap_prop = overlap / m_vec[None, :]
    prop_h2 = overlap_prop @ prop
    prop_h2_se = _se(np.diag(overlap_prop @ prop_cov @ overlap_prop.T))
    prop_m = m_vec / m_tot if m_tot > 0 else np.full(k, np.nan)
    diff = np.zeros((k, k))
    for i in range(k):
        if abs(m_tot - m_vec[i]) < 1e-12:
            continue
        diff[i] = overlap[i] / m_vec[i] - (m_vec - overlap[i]) / (m_tot - m_vec[i])
    diff_est = diff @ coef
    diff_se = _se(np.diag(diff @ coef_cov @ diff.T))
    with np.errstate(divide="ignore", invalid="ignore"):
        t = np.abs(diff_est / diff_se)
    return dict(prop_m=prop_m, prop_h2=prop_h2, prop_h2_se=prop_h2_se, enrichment=prop_h2 / prop_m,
                enrichment_se=prop_h2_se / prop_m, diff_t=t, diff_na=diff_se == 0.0, coef=coef, coef_se=coef_se)


def write_overlap_results(out_prefix: str, fit: PartitionedFit, names: Sequence[str], overlap: np.ndarray,
                          m_tot: float, print_coefficients: bool = False) -> str:
    """`{out}.results` of --overlap-annot (src/regressions.rs:1440-1493).
    Enrichment_p is the two-sided Student t (n_blocks degrees of freedom)
    p-value of the coefficient difference, "NA" where its SE is 0."""
    from scipy.stats import t as student_t
    fig = overlap_figures(fit, overlap, m_tot)
    path = f"{out_prefix}.results"
    with open(path, "w") as f:
        head = "Category\tProp._SNPs\tProp._h2\tProp._h2_std_error\tEnrichment\tEnrichment_std_error\tEnrichment_p"
        if print_coefficients:
            head += "\tCoefficient\tCoefficient_std_error\tCoefficient_z-score"
        f.write(head + "\n")
        for i, name in enumerate(names):
            p = "NA" if fig["diff_na"][i] else rust_f64(float(2.0 * student_t.sf(fig["diff_t"][i], fit.n_blocks)))
            row = [name] + [_f(float(fig[c][i]), 6) for c in ("prop_m", "prop_h2", "prop_h2_se", "enrichment",
                                                              "enrichment_se")] + [p]
            if print_coefficients:
                cs = fig["coef_se"][i]
                z = float("nan") if cs == 0.0 else fig["coef"][i] / cs
                row += [_rust_exp(float(fig["coef"][i]), 6), _rust_exp(float(cs), 6), _f(float(z), 6)]
            f.write("\t".join(row) + "\n")
    print(f"Results printed to {path}")
    return path
