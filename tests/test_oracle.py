"""Pin the CPU oracle: the reference's own known answers, its scatter tests,
and the brute-force definition of l2 on small panels."""
import os

import numpy as np
import pytest

from conftest import brute_force_l2
from oracle import OracleL2Args, block_lefts, oracle_l2, scatter_column_f32

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def py_left_limits(chr_, cm, bp, mode, wind, half, chunk, masking, per_chr):
    """Independent restatement of the pair set: masked -> block_left;
    chunked -> chunk start minus its rounded-up window (src/l2/compute.rs:1164-1184,1288-1299)."""
    bl, _ = block_lefts(chr_, cm, bp, mode, wind, half)
    m = len(chr_)
    left = np.zeros(m, dtype=np.int64)
    groups = []
    s = 0
    while s < m:
        e = s + 1
        if per_chr:
            while e < m and chr_[e] == chr_[s]:
                e += 1
        else:
            e = m
        groups.append((s, e))
        s = e
    for g0, g1 in groups:
        for cs in range(g0, g1, chunk):
            ce = min(cs + chunk, g1)
            dist = cs - bl[cs]
            b = 0 if dist == 0 else -(-dist // chunk) * chunk
            b = min(b, cs - g0)
            for j in range(cs, ce):
                left[j] = bl[j] if masking else cs - b
    return left


def test_micro_known_answer():
    """src/l2/mod.rs:1191-1225: l2 = [2, 2], MAF = [0.5, 0.5] within 1e-9."""
    z = np.load(os.path.join(GOLDEN, "micro.npz"))
    a = OracleL2Args(bed_body=z["bed"][3:], n_file_indiv=4, chr=z["chr"], cm=z["cm"], bp=z["bp"],
                     mode="kb", wind=100.0, chunk_c=2, per_chr=False)
    l2, maf, pairs, _ = oracle_l2(a)
    np.testing.assert_allclose(l2[:, 0], z["l2"], atol=1e-9)
    np.testing.assert_allclose(maf, z["maf"], atol=1e-9)
    assert pairs == 1


def test_chunk_size_zero_is_an_error():
    z = np.load(os.path.join(GOLDEN, "micro.npz"))
    a = OracleL2Args(bed_body=z["bed"][3:], n_file_indiv=4, chr=z["chr"], cm=z["cm"], bp=z["bp"],
                     mode="kb", wind=100.0, chunk_c=0)
    with pytest.raises(ValueError, match="chunk_size must be >= 1"):
        oracle_l2(a)


def test_sketch_out_of_bounds_is_an_error():
    z = np.load(os.path.join(GOLDEN, "small_panel.npz"))
    n = int(z["n_indiv"])
    a = OracleL2Args(bed_body=z["body"], n_file_indiv=n, chr=z["chr"], cm=z["cm"], bp=z["bp"],
                     sketch_d=n, use_f32=True)
    with pytest.raises(ValueError, match="out of bounds"):
        oracle_l2(a)


CASES = [
    ("cm", 1.0, 0, 50, False, True, None, None),
    ("cm", 1.0, 0, 50, True, True, None, None),
    ("cm", 1.0, 0, 64, False, False, None, None),
    ("kb", 500.0, 0, 40, False, True, None, None),
    ("snp", 0.0, 25, 30, True, True, None, None),
    ("cm", 1.0, 0, 50, False, True, "annot3", None),
    ("cm", 1.0, 0, 50, True, True, None, 1.0),
]


@pytest.mark.parametrize("mode,wind,half,chunk,masking,per_chr,annot,pq", CASES)
def test_oracle_matches_brute_force(mode, wind, half, chunk, masking, per_chr, annot, pq):
    z = np.load(os.path.join(GOLDEN, "small_panel.npz"))
    body, n = z["body"], int(z["n_indiv"])
    chr_, cm, bp = z["chr"], z["cm"], z["bp"]
    A = None
    if annot:
        from golden.make_golden import annot3
        A = annot3(len(chr_))
    a = OracleL2Args(bed_body=body, n_file_indiv=n, chr=chr_, cm=cm, bp=bp, mode=mode, wind=wind,
                     wind_snp=half, chunk_c=chunk, masking=masking, per_chr=per_chr, annot=A,
                     pq_exp=pq)
    l2, maf, pairs, _ = oracle_l2(a)
    left = py_left_limits(chr_, cm, bp, mode, wind, half, chunk, masking, per_chr)
    assert pairs == int(np.sum(np.arange(len(chr_)) - left))
    pqv = None
    if pq is not None:
        pqv = (maf * (1 - maf)) ** pq
    ref, ref_maf = brute_force_l2(body, n, chr_, cm, bp, left, annot=A, pq=pqv)
    np.testing.assert_allclose(maf, ref_maf, atol=1e-15)
    scale = np.maximum(np.abs(ref), 1.0)
    assert np.max(np.abs(l2 - ref) / scale) < 1e-10


@pytest.mark.parametrize("masking,chunk", [(True, 200), (False, 50)])
def test_oracle_wide_panel_matches_brute_force(masking, chunk):
    """700 individuals (several 256-individual slices of the chunk Grams, with
    a ragged last slice) and windows wider than one 64-column macro tile, so
    the blocked and packed Gram kernels' slice and tile edges are all
    crossed."""
    from ldsc_b200 import synth
    spec = synth.PanelSpec(n_indiv=700, chrom_sizes=[320], chrom_cm=[2.0], founders=20, miss=0.02, seed=5)
    body = synth.bed_body(spec)
    chr_, cm, bp = synth.positions(spec)
    a = OracleL2Args(bed_body=body, n_file_indiv=spec.n_indiv, chr=chr_, cm=cm, bp=bp, chunk_c=chunk,
                     masking=masking)
    l2, maf, pairs, _ = oracle_l2(a)
    left = py_left_limits(chr_, cm, bp, "cm", 1.0, 0, chunk, masking, True)
    assert int(np.max(np.arange(len(chr_)) - left)) > 64
    ref, ref_maf = brute_force_l2(body, spec.n_indiv, chr_, cm, bp, left)
    np.testing.assert_allclose(maf, ref_maf, atol=1e-15)
    assert np.max(np.abs(l2 - ref) / np.maximum(np.abs(ref), 1.0)) < 1e-10


def test_oracle_keep_subset_matches_brute_force():
    z = np.load(os.path.join(GOLDEN, "small_panel.npz"))
    body, n = z["body"], int(z["n_indiv"])
    chr_, cm, bp = z["chr"], z["cm"], z["bp"]
    keep = np.arange(3, n, 2, dtype=np.int64)
    a = OracleL2Args(bed_body=body, n_file_indiv=n, chr=chr_, cm=cm, bp=bp, chunk_c=50,
                     iid_idx=keep)
    l2, maf, _, _ = oracle_l2(a)
    left = py_left_limits(chr_, cm, bp, "cm", 1.0, 0, 50, False, True)
    ref, ref_maf = brute_force_l2(body, n, chr_, cm, bp, left, iid=keep)
    np.testing.assert_allclose(maf, ref_maf, atol=1e-15)
    assert np.max(np.abs(l2 - ref) / np.maximum(np.abs(ref), 1.0)) < 1e-10


def test_oracle_f32_within_reference_tolerance():
    """--fast-f32 vs f64 (scripts/verify_parity_all.sh: f32 within 2e-2)."""
    z = np.load(os.path.join(GOLDEN, "small_panel.npz"))
    assert np.max(np.abs(z["l2_cm1_f32"] - z["l2_cm1_chunk50"])) < 2e-2


def test_oracle_reproduces_golden():
    from golden.make_golden import MODES, oracle_args
    z = np.load(os.path.join(GOLDEN, "small_panel.npz"))
    for name in MODES:
        l2, maf, pairs, _ = oracle_l2(oracle_args(name, z["body"], int(z["n_indiv"]), z["chr"], z["cm"], z["bp"]))
        np.testing.assert_allclose(l2, z[f"l2_{name}"], rtol=1e-12, atol=1e-12)
        assert pairs == int(z[f"pairs_{name}"])


# ---- port of the reference's CountSketch scatter tests (src/wasm_simd.rs:2810-3180) ----

def lcg_bed_fixture(seed, c, n_indiv):
    """make_bed_fixture: 6% missing, 31% each real code."""
    bpr = (n_indiv + 3) // 4
    state = seed
    raw = np.zeros(c * bpr, dtype=np.uint8)
    mask = (1 << 64) - 1
    for j in range(c):
        for b in range(bpr):
            byte = 0
            for slot in range(4):
                state = (state * 0x9E3779B97F4A7C15 + 1) & mask
                r = (state >> 32) % 100
                code = 0b01 if r <= 5 else (0b00 if r <= 37 else (0b10 if r <= 69 else 0b11))
                byte |= code << (2 * slot)
            raw[j * bpr + b] = byte
    return raw


def lcg_bucket_sign(n, d, seed):
    mask = (1 << 64) - 1
    state = seed
    bucket = np.zeros(n, dtype=np.uint32)
    for i in range(n):
        state = (state * 0x9E3779B97F4A7C15 + 1) & mask
        bucket[i] = ((state >> 32) & 0xFFFFFFFF) % d
    sign = np.zeros(n, dtype=np.float32)
    for i in range(n):
        state = (state * 0x9E3779B97F4A7C15 + 1) & mask
        sign[i] = 1.0 if ((state >> 63) & 1) == 0 else -1.0
    return bucket, sign


def snp_mean_inv(raw, bpr, j, n):
    codes = np.array([(raw[j * bpr + i // 4] >> (2 * (i % 4))) & 3 for i in range(n)])
    g = np.array([2.0, np.nan, 1.0, 0.0])[codes]
    pres = ~np.isnan(g)
    s, cnt, sq = g[pres].sum(), pres.sum(), (g[pres] ** 2).sum()
    mean = s / cnt if cnt else 0.0
    var = (sq - cnt * mean * mean) / n
    return g, np.float32(mean), np.float32(1.0 / np.sqrt(var)) if var > 0 else np.float32(0.0)


def direct_scatter_f32(g, bucket, sign, mean, inv, n_norm, d):
    col = np.zeros(d, dtype=np.float32)
    for i in range(len(g)):
        val = np.float32(0.0) if np.isnan(g[i]) else (np.float32(g[i]) - mean) * inv
        col[bucket[i]] += sign[i] * val
    nrm = float(np.sum(col.astype(np.float64) ** 2))
    if nrm > 0:
        col *= np.float32(np.sqrt(n_norm / nrm))
    return col


def test_scatter_f32_matches_direct_reference_all_iids():
    c, n, d = 8, 503, 50
    raw = lcg_bed_fixture(42, c, n)
    bpr = (n + 3) // 4
    bucket, sign = lcg_bucket_sign(n, d, 7)
    for j in range(c):
        g, mean, inv = snp_mean_inv(raw, bpr, j, n)
        got = scatter_column_f32(raw[j * bpr:(j + 1) * bpr], n, bucket, sign, mean, inv, float(n), d)
        exp = direct_scatter_f32(g, bucket, sign, mean, inv, float(n), d)
        diff = np.abs(got - exp)
        assert np.all((diff < 1e-4) | (diff / np.maximum(np.abs(exp), 1e-6) < 1e-4))


def test_scatter_subsample_matches_all_iids_on_full_keep():
    c, n, d = 3, 47, 16
    raw = lcg_bed_fixture(99, c, n)
    bpr = (n + 3) // 4
    bucket, sign = lcg_bucket_sign(n, d, 5)
    for j in range(c):
        _, mean, inv = snp_mean_inv(raw, bpr, j, n)
        row = raw[j * bpr:(j + 1) * bpr]
        a = scatter_column_f32(row, n, bucket, sign, mean, inv, float(n), d)
        b = scatter_column_f32(row, n, bucket, sign, mean, inv, float(n), d,
                               iid_idx=np.arange(n, dtype=np.int64))
        assert np.array_equal(a, b)


def _numpy_sketch_l2(body, n, chr_, cm, bp, d, maf_aware):
    """Independent restatement of the --sketch d --snp-level-masking path on
    the CPU: per SNP the f32 LUT values (normalize_col_f32_with_stats,
    src/l2/normalize.rs:115-154) scattered into d buckets in individual order
    (src/wasm_simd.rs:1617-1784) and renormalised with an f64 norm; the
    per-pair quadratic bias inversion with the kurtosis shift when MAF-aware
    (quadratic_sketch_correction[_maf_aware], src/l2/compute.rs:947-998;
    per_snp_kappa, :525-538); l2_j = 1 + the corrected r^2 over the SNP's own
    window."""
    from ldsc_b200.plink import decode_genotypes
    from oracle import block_lefts, countsketch_hash
    G = decode_genotypes(body, n)                      # M x N, NaN missing
    m = G.shape[0]
    bucket, sign = countsketch_hash(n, d, 42)
    S = np.zeros((m, d), dtype=np.float32)
    kappa = np.zeros(m)
    for j in range(m):
        g = G[j]
        pres = ~np.isnan(g)
        cnt = pres.sum()
        gv = np.where(pres, g, 0.0)
        mean = gv.sum() / cnt if cnt else 0.0
        css = (gv * gv).sum() - cnt * mean * mean
        sd = np.sqrt(css / n)
        inv = np.float32(1.0 / sd) if sd > 0 else np.float32(0.0)
        m32 = np.float32(mean)
        lut = {2.0: (np.float32(2.0) - m32) * inv, 1.0: (np.float32(1.0) - m32) * inv, 0.0: (-m32) * inv}
        vals = np.array([lut[x] if p else np.float32(0.0) for x, p in zip(gv, pres)], dtype=np.float32)
        out = np.zeros(d, dtype=np.float32)
        np.add.at(out, bucket, (sign * vals).astype(np.float32))
        nrm = float(np.sum(out.astype(np.float64) ** 2))
        if nrm > 0:
            out = out * np.float32(np.sqrt(n / nrm))
        S[j] = out
        if cnt and css > 0:
            dv = gv[pres] - mean
            kappa[j] = float((dv ** 4).sum()) / css ** 2
    bl, _ = block_lefts(chr_, cm, bp, "cm", 1.0)
    denom = n - 2.0
    l2 = np.ones(m)
    for j in range(m):
        for k in range(bl[j], j):
            val = float(np.dot(S[j].astype(np.float64), S[k].astype(np.float64)))
            kap = (kappa[j] + kappa[k]) if maf_aware else 0.0
            tilde = val * val / (n * n)
            dm3 = d - 3.0 - 2.0 * kap
            disc = dm3 * dm3 + 8.0 * (d * tilde - 1.0)
            r2 = (-dm3 + np.sqrt(disc)) / 4.0 if disc >= 0 else 0.0
            r2u = r2 * (1 + 1 / denom) - 1 / denom
            l2[j] += r2u
            l2[k] += r2u
    return l2


@pytest.mark.parametrize("name", ["cm1_sketch50", "cm1_sketch200", "cm1_sketch50_maf", "cm1_sketch200_maf"])
def test_oracle_sketch_matches_numpy_restatement(name):
    """The oracle's sketch path, plain and MAF-aware, against the restatement
    above on the golden panel (the dot products here are f64 over the f32
    sketched values, the oracle's are f32: agreement to f32 rounding)."""
    z = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "small_panel.npz"))
    from golden.make_golden import MODES
    d = MODES[name][6]
    got = _numpy_sketch_l2(z["body"], int(z["n_indiv"]), z["chr"], z["cm"], z["bp"], d, name.endswith("_maf"))
    ref = z[f"l2_{name}"][:, 0]
    # measured ~5e-7 (the f32 dot products' rounding)
    assert np.max(np.abs(got - ref)) < 1e-5
    if name.endswith("_maf"):
        # the kurtosis shift is visible: the plain correction differs by far more
        plain = z[f"l2_{name[:-4]}"][:, 0]
        assert np.max(np.abs(plain - ref)) > 1000 * np.max(np.abs(got - ref))
