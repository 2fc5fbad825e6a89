"""CPU restatement of the LD-score regressions -- TEST INFRASTRUCTURE ONLY.

Follows, step for step:
  get_separators / update_separators     src/h2.rs:31-58
  weight_xy / wls (QR least squares)     src/h2.rs:60-92
  jackknife_fast (LU solves)             src/h2.rs:100-183
  ldsc_weights / aggregate               src/h2.rs:185-218
  combine_twostep                        src/h2.rs:220-256
  run_h2_ldsc (incl. --two-step)         src/h2.rs:258-433
  irwls_ldsc                             src/h2.rs:435-458
  jackknife_se_cov                       src/jackknife.rs:10-59
  ratio_jackknife                        src/regressions.rs:1067-1120
  gencov_weights / run_gencov_ldsc       src/regressions.rs:1612-1645, 1828-2052
  rg, z, p                               src/regressions.rs:2389-2465
  run_h2's K > 1 filters                 src/regressions.rs:553-593
  fit_h2_partitioned                     src/regressions.rs:1121-1226
  total_from_jknife                      src/regressions.rs:1565-1610
  write_overlap_results (the figures)    src/regressions.rs:1262-1440
faer's QR and LU are replaced by numpy's (same factorisations, different
rounding order).
"""
from __future__ import annotations

import math

import numpy as np


def get_separators(n, n_blocks):
    seps = [int(math.floor(i * n / n_blocks)) for i in range(n_blocks + 1)]
    seps[-1] = n
    return seps


def update_separators(seps, mask):
    maplist = np.nonzero(mask)[0]
    out = [0] + [int(maplist[s]) for s in seps[1:-1]] + [len(mask)]
    return out


def weight_xy(x, y, w):
    if np.any(w <= 0):
        raise ValueError("weights must be > 0")
    wi = w / w.sum()
    return x * wi[:, None], y * wi


def wls(x, y, w):
    xw, yw = weight_xy(x, y, w)
    q, r = np.linalg.qr(xw)
    return np.linalg.solve(r, q.T @ yw)


def jackknife_se_cov(est, delete_values):
    nb, p = delete_values.shape
    pseudo = est[None, :] * nb - delete_values * (nb - 1)
    centered = pseudo - pseudo.mean(axis=0)
    cov = centered.T @ centered / ((nb - 1.0) * nb)
    return np.sqrt(np.diag(cov)), cov


def jackknife_fast(x, y, n_blocks, separators=None):
    n, p = x.shape
    seps = list(separators) if separators is not None else get_separators(n, n_blocks)
    nb = len(seps) - 1
    if nb > n:
        raise ValueError("More blocks than data points.")
    xty = np.zeros((nb, p))
    xtx = np.zeros((nb, p, p))
    for i in range(nb):
        xb, yb = x[seps[i]:seps[i + 1]], y[seps[i]:seps[i + 1]]
        xty[i] = xb.T @ yb
        xtx[i] = xb.T @ xb
    est = np.linalg.solve(xtx.sum(0), xty.sum(0))
    dele = np.array([np.linalg.solve(xtx.sum(0) - xtx[i], xty.sum(0) - xty[i]) for i in range(nb)])
    se, cov = jackknife_se_cov(est, dele)
    return dict(est=est, se=se, cov=cov, delete_values=dele, separators=seps)


def ldsc_weights(ld, w_ld, n_vec, m, hsq, intercept):
    hsq = min(max(hsq, 0.0), 1.0)
    ld = np.maximum(ld, 1.0)
    w = np.maximum(w_ld, 1.0)
    c = hsq * n_vec / m
    return 1.0 / (2.0 * (intercept + c * ld) ** 2) / w


def gencov_weights(ld, w_ld, n1, n2, m, h1, h2, rho_g, int_g, int_h1, int_h2):
    h1 = min(max(h1, 0.0), 1.0)
    h2 = min(max(h2, 0.0), 1.0)
    ld = np.maximum(ld, 1.0)
    w = np.maximum(w_ld, 1.0)
    a = n1 * h1 * ld / m + int_h1
    b = n2 * h2 * ld / m + int_h2
    c = np.sqrt(n1 * n2) * rho_g * ld / m + int_g
    return 1.0 / (a * b + c * c) / w


def aggregate(y, x, n_vec, m, intercept):
    return m * (y.mean() - intercept) / (x * n_vec).mean()


def irwls(x, y, initial_w, update, n_blocks, separators=None):
    w = np.sqrt(initial_w)
    for _ in range(2):
        coef = wls(x, y, w)
        w = np.sqrt(update(coef))
    xw, yw = weight_xy(x, y, w)
    return jackknife_fast(xw, yw, n_blocks, separators)


def combine_twostep(s1, s2, c):
    nb = s1["delete_values"].shape[0]
    step1_int = s1["est"][1]
    est = np.array([s2["est"][0], step1_int])
    dele = np.zeros((nb, 2))
    dele[:, 1] = s1["delete_values"][:, 1]
    dele[:, 0] = s2["delete_values"][:, 0] - c * (s1["delete_values"][:, 1] - step1_int)
    se, cov = jackknife_se_cov(est, dele)
    return dict(est=est, se=se, cov=cov, delete_values=dele, separators=s2["separators"])


def run_h2(chi2, ref_l2, w_l2, n_vec, m, n_blocks=200, two_step=None, fixed_intercept=None):
    """run_h2_ldsc: returns dict(h2, h2_se, intercept, intercept_se, mean_chi2,
    lambda_gc, ratio, ratio_se, tot_delete)."""
    chi2 = np.asarray(chi2, float)
    n_blocks = min(n_blocks, len(chi2))
    n_vec = np.broadcast_to(np.asarray(n_vec, float), chi2.shape).copy()
    n = len(chi2)
    nbar = n_vec.mean()
    int0 = 1.0 if fixed_intercept is None else fixed_intercept
    agg = aggregate(chi2, ref_l2, n_vec, m, int0)
    initial_w = ldsc_weights(ref_l2, w_l2, n_vec, m, agg, int0)
    x0 = n_vec * ref_l2 / nbar
    if fixed_intercept is not None:
        y_reg, x_reg = chi2 - fixed_intercept, x0[:, None]
    else:
        y_reg, x_reg = chi2, np.stack([x0, np.ones(n)], axis=1)
    if two_step is not None:
        mask = chi2 < two_step
        x1, y1, w1, n1 = x_reg[mask], y_reg[mask], w_l2[mask], n_vec[mask]
        x1c0 = x1[:, 0]
        upd1 = lambda c: ldsc_weights(x1c0, w1, n1, m, m * c[0] / nbar, c[1])  # noqa: E731
        s1 = irwls(x1, y1, initial_w[mask], upd1, n_blocks)
        step1_int = s1["est"][1]
        y2, x2 = y_reg - step1_int, x_reg[:, :1]
        upd2 = lambda c: ldsc_weights(ref_l2, w_l2, n_vec, m, m * c[0] / nbar, step1_int)  # noqa: E731
        seps = update_separators(s1["separators"], mask)
        s2 = irwls(x2, y2, initial_w, upd2, n_blocks, seps)
        cc = np.sum(initial_w * x2[:, 0]) / np.sum(initial_w * x2[:, 0] ** 2)
        jk = combine_twostep(s1, s2, cc)
    else:
        upd = lambda c: ldsc_weights(ref_l2, w_l2, n_vec, m, m * c[0] / nbar,  # noqa: E731
                                     fixed_intercept if fixed_intercept is not None else c[1])
        jk = irwls(x_reg, y_reg, initial_w, upd, n_blocks)
    h2 = m * jk["est"][0] / nbar
    h2_se = math.sqrt(m * m * jk["cov"][0, 0] / nbar ** 2)
    if fixed_intercept is not None:
        intercept, intercept_se = fixed_intercept, float("nan")
    else:
        intercept, intercept_se = jk["est"][1], jk["se"][1]
    mean_chi2 = chi2.mean()
    lam = np.median(chi2) / 0.4549
    if mean_chi2 > 1.0 and fixed_intercept is None:
        ratio, ratio_se = (intercept - 1) / (mean_chi2 - 1), intercept_se / (mean_chi2 - 1)
    else:
        ratio = ratio_se = float("nan")
    return dict(h2=h2, h2_se=h2_se, intercept=intercept, intercept_se=intercept_se, mean_chi2=mean_chi2,
                lambda_gc=lam, ratio=ratio, ratio_se=ratio_se,
                tot_delete=m * jk["delete_values"][:, 0] / nbar, est=jk["est"])


def run_gencov(z1, z2, ref_l2, w_l2, n1, n2, m, n_blocks, hsq1, hsq2):
    n = len(z1)
    n1 = np.broadcast_to(np.asarray(n1, float), (n,))
    n2 = np.broadcast_to(np.asarray(n2, float), (n,))
    sq = np.sqrt(n1 * n2)
    nbar = sq.mean()
    prod = z1 * z2
    agg = aggregate(prod, ref_l2, sq, m, 0.0)
    iw = gencov_weights(ref_l2, w_l2, n1, n2, m, hsq1["h2"], hsq2["h2"], agg, 0.0, hsq1["intercept"],
                        hsq2["intercept"])
    x = np.stack([sq * ref_l2 / nbar, np.ones(n)], axis=1)
    upd = lambda c: gencov_weights(ref_l2, w_l2, n1, n2, m, hsq1["h2"], hsq2["h2"],  # noqa: E731
                                   m * c[0] / nbar, c[1], hsq1["intercept"], hsq2["intercept"])
    jk = irwls(x, prod, iw, upd, n_blocks)
    return dict(tot=m * jk["est"][0] / nbar, tot_se=math.sqrt(_rmax0(m * m * jk["cov"][0, 0] / nbar ** 2)),
                intercept=jk["est"][1], intercept_se=jk["se"][1], mean_z1z2=prod.mean(),
                tot_delete=m * jk["delete_values"][:, 0] / nbar)


def _rmax0(v):
    """f64::max(v, 0.0): the non-NaN operand wins, so NaN -> 0."""
    return v if v > 0.0 else 0.0


def ratio_jackknife(est, numer_delete, denom_delete):
    nb = len(numer_delete)
    with np.errstate(divide="ignore", invalid="ignore"):
        pseudo = np.where(denom_delete == 0, np.nan, nb * est - (nb - 1) * (numer_delete / denom_delete))
    centered = pseudo - pseudo.mean()
    cov = centered @ centered / ((nb - 1.0) * nb)
    return math.sqrt(_rmax0(cov))


def run_rg(z1, z2, ref_l2, w_l2, n1, n2, m, n_blocks=200):
    n_blocks = min(n_blocks, len(z1))
    h1 = run_h2(np.maximum(z1 * z1, 0), ref_l2, w_l2, n1, m, n_blocks)
    h2 = run_h2(np.maximum(z2 * z2, 0), ref_l2, w_l2, n2, m, n_blocks)
    g = run_gencov(z1, z2, ref_l2, w_l2, n1, n2, m, n_blocks, h1, h2)
    if h1["h2"] > 0 and h2["h2"] > 0:
        rg = g["tot"] / math.sqrt(h1["h2"] * h2["h2"])
        pr = h1["tot_delete"] * h2["tot_delete"]
        with np.errstate(invalid="ignore"):
            den = np.where(np.isfinite(pr) & (pr >= 0), np.sqrt(np.abs(pr)), np.nan)
        rg_se = ratio_jackknife(rg, g["tot_delete"], den)
    else:
        rg = rg_se = float("nan")
    if math.isfinite(rg_se) and rg_se != 0.0:
        z = rg / rg_se
        p = math.erfc(abs(z) / math.sqrt(2.0)) if math.isfinite(z) else 0.0
    else:
        z, p = float("inf"), 0.0
    return dict(rg=rg, rg_se=rg_se, z=z, p=p, gencov=g["tot"], gencov_se=g["tot_se"], gencov_intercept=g["intercept"],
                gencov_intercept_se=g["intercept_se"], h2_1=h1["h2"], h2_1_se=h1["h2_se"], h2_2=h2["h2"],
                h2_2_se=h2["h2_se"], mean_z1z2=g["mean_z1z2"])


def fit_h2_partitioned(chi2, ref_l2_k, w_l2, n_vec, m_vec, n_blocks=200, intercept_h2=None, no_intercept=False,
                       chisq_max=None):
    """run_h2's K > 1 branch: drop NaN chi2 / N, drop chi2 >= chisq_max
    (default max(0.001 max N, 80)), then fit_h2_partitioned.  ref_l2_k: n x K."""
    chi2 = np.asarray(chi2, float)
    x_raw = np.asarray(ref_l2_k, float).reshape(len(chi2), -1)
    w_l2 = np.asarray(w_l2, float)
    n_vec = np.broadcast_to(np.asarray(n_vec, float), chi2.shape).copy()
    valid = ~np.isnan(chi2) & ~np.isnan(n_vec)
    chi2, x_raw, w_l2, n_vec = chi2[valid], x_raw[valid], w_l2[valid], n_vec[valid]
    if chisq_max is None:
        chisq_max = max(0.001 * max(float(n_vec.max(initial=0.0)), 0.0), 80.0)
    keep = chi2 < chisq_max
    chi2, x_raw, w_l2, n_vec = chi2[keep], x_raw[keep], w_l2[keep], n_vec[keep]
    n_obs, k = x_raw.shape
    n_mean = n_vec.mean()
    m_vec = np.asarray(m_vec, float)
    m_total = float(np.sum(m_vec))
    nb = min(n_obs, n_blocks)
    x_tot = np.zeros(n_obs)
    for j in range(k):
        x_tot = x_tot + x_raw[:, j]
    fixed = intercept_h2 if intercept_h2 is not None else (1.0 if no_intercept else None)
    y_reg = chi2 - fixed if fixed is not None else chi2.copy()
    scale = n_vec / n_mean
    x_reg = x_raw * scale[:, None]
    if fixed is None:
        x_reg = np.concatenate([x_reg, np.ones((n_obs, 1))], axis=1)
    agg_int = fixed if fixed is not None else 1.0
    hsq = aggregate(chi2, x_tot, n_vec, m_total, agg_int)
    initial_w = ldsc_weights(x_tot, w_l2, n_vec, m_total, hsq, agg_int)
    xw, yw = weight_xy(x_reg, y_reg, np.sqrt(initial_w))
    jk = jackknife_fast(xw, yw, nb)
    coef = jk["est"][:k] / n_mean
    h2_annot = coef * m_vec
    h2_total = float(np.sum(h2_annot))
    intercept = fixed if fixed is not None else float(jk["est"][k])
    intercept_se = float("nan") if fixed is not None else float(math.sqrt(_rmax0(jk["cov"][k, k])))
    coef_cov = jk["cov"][:k, :k] / (n_mean * n_mean)
    tot_cov = 0.0
    for i in range(k):
        for j in range(k):
            tot_cov += m_vec[i] * m_vec[j] * coef_cov[i, j]
    return dict(est=jk["est"], cov=jk["cov"], delete_values=jk["delete_values"], m_vec=m_vec, n_mean=n_mean,
                h2_annot=h2_annot, h2_total=h2_total, h2_total_se=math.sqrt(_rmax0(tot_cov)), intercept=intercept,
                intercept_se=intercept_se, n_obs=n_obs, n_blocks=nb, mean_chi2=float(chi2.mean()))


def _ratio_jackknife_mat(est, numer, denom):
    nb, k = numer.shape
    pseudo = np.zeros((nb, k))
    for b in range(nb):
        for j in range(k):
            pseudo[b, j] = float("nan") if denom[b, j] == 0.0 else \
                nb * est[j] - (nb - 1.0) * (numer[b, j] / denom[b, j])
    mean = pseudo.sum(axis=0) / nb
    c = pseudo - mean
    cov = c.T @ c
    scale = (nb - 1.0) * nb
    if scale > 0.0:
        cov = cov / scale
    return cov


def overlap_figures(fit, overlap, m_tot):
    """The per-category figures of write_overlap_results (before formatting):
    prop_m, prop_h2, prop_h2_se, enrichment, enrichment_se, t statistic of the
    coefficient difference (diff_na where its SE is 0), coef, coef_se."""
    k = len(fit["m_vec"])
    m_vec = fit["m_vec"]
    n_mean = fit["n_mean"]
    coef = fit["est"][:k] / n_mean
    coef_cov = fit["cov"][:k, :k] / (n_mean * n_mean)
    coef_se = np.sqrt(np.array([_rmax0(coef_cov[j, j]) for j in range(k)]))
    h2_total = fit["h2_total"]
    prop = np.array([h / h2_total if abs(h2_total) > 1e-12 else float("nan") for h in fit["h2_annot"]])
    dv = fit["delete_values"]
    nb = dv.shape[0]
    numer = np.zeros((nb, k))
    for b in range(nb):
        for j in range(k):
            numer[b, j] = m_vec[j] * dv[b, j] / n_mean
    denom = np.zeros((nb, k))
    for b in range(nb):
        denom[b, :] = numer[b, :].sum()
    prop_cov = _ratio_jackknife_mat(prop, numer, denom)
    overlap_prop = np.zeros((k, k))
    for i in range(k):
        for j in range(k):
            overlap_prop[i, j] = overlap[i, j] / m_vec[j]
    prop_h2_overlap = overlap_prop @ prop
    var = overlap_prop @ prop_cov @ overlap_prop.T
    prop_h2_overlap_se = np.sqrt(np.array([_rmax0(var[j, j]) for j in range(k)]))
    prop_m = np.array([m / m_tot if m_tot > 0 else float("nan") for m in m_vec])
    enrichment = prop_h2_overlap / prop_m
    enrichment_se = prop_h2_overlap_se / prop_m
    diff = np.zeros((k, k))
    for i in range(k):
        if abs(m_tot - m_vec[i]) < 1e-12:
            continue
        for j in range(k):
            diff[i, j] = overlap[i, j] / m_vec[i] - (m_vec[j] - overlap[i, j]) / (m_tot - m_vec[i])
    diff_est = diff @ coef
    diff_cov = diff @ coef_cov @ diff.T
    diff_se = np.sqrt(np.array([_rmax0(diff_cov[j, j]) for j in range(k)]))
    na = np.array([diff_se[i] == 0.0 for i in range(k)])
    with np.errstate(divide="ignore", invalid="ignore"):
        t = np.array([abs(diff_est[i] / diff_se[i]) for i in range(k)])
    return dict(prop_m=prop_m, prop_h2=prop_h2_overlap, prop_h2_se=prop_h2_overlap_se, enrichment=enrichment,
                enrichment_se=enrichment_se, diff_t=t, diff_na=na, coef=coef, coef_se=coef_se)
