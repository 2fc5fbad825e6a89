"""GPU parity of the l2 engine against the CPU oracle (through the C ABI)."""
import os

import numpy as np
import pytest

from ldsc_b200 import synth
from ldsc_b200.plink import BimTable

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
# exact modes: max |l2 - oracle| / max(|oracle|, 1) (FP64 reorders sums; INT8 is exact up to rounding)
EXACT_TOL = 1e-9
# K > 1: r2u tiles contracted with the annotations in f64, relative per l2_jC
ANNOT_TOL = 1e-9
# --sketch: absolute on l2.  Summing each bucket exactly instead of in f32
# individual order moves l2 by ~2.4e-6 at d = 50 on the golden panel (CPU
# restatement of both), the f32 dot products by ~5e-7.
SKETCH_TOL = 3e-5   # measured on a B200: 5.7e-6 (d = 50), 9.3e-6 (d = 200)


def table(chr_, cm, bp):
    m = len(chr_)
    return BimTable(np.asarray(chr_, np.uint8), [f"rs{i}" for i in range(m)], np.asarray(cm, float),
                    np.asarray(bp, np.uint32), np.arange(m, dtype=np.int64))


def relerr(a, b):
    return float(np.max(np.abs(a - b) / np.maximum(np.abs(b), 1.0)))


def entry_relerr(a, b):
    """max over entries of |a - b| / |b|; an entry the oracle has at exactly 0
    must be 0 too."""
    return float(np.max(np.abs(a - b) / np.maximum(np.abs(b), 1e-300)))


@pytest.fixture(scope="module")
def small():
    z = np.load(os.path.join(GOLDEN, "small_panel.npz"))
    return z


@pytest.fixture(scope="module")
def small_panel(ctx, small):
    return ctx.upload(small["body"], int(small["n_indiv"]))


def run_mode(ctx, small, panel, name, precision):
    from golden.make_golden import MAF_AWARE, MODES, annot3
    from ldsc_b200.api import WindowMode, run_l2
    mode, wind, chunk, masking, per_chr, f32, sk, has_annot, pq = MODES[name]
    wm = {"cm": WindowMode.Cm, "kb": WindowMode.Kb, "snp": WindowMode.Snp}[mode](wind)
    snps = table(small["chr"], small["cm"], small["bp"])
    A = annot3(len(snps)) if has_annot else None
    return run_l2(ctx, snps, panel, wm, chunk, annot=A, pq_exp=pq, use_f32=f32, sketch=sk or None,
                  sketch_maf_aware=name in MAF_AWARE, snp_level_masking=masking, global_pass=not per_chr,
                  precision=precision, yes_really=True)


def test_micro_known_answer_from_bytes(ctx):
    """src/l2/mod.rs:1191-1225 through the whole-file entry point."""
    from ldsc_b200.api import L2Config, WindowMode, compute_l2_from_bytes
    bim = "1\trs1\t0\t100\tA\tG\n1\trs2\t0\t200\tA\tG\n"
    fam = "".join(f"F{i}\tI{i}\t0\t0\t1\t-9\n" for i in range(1, 5))
    bed = bytes([0x6C, 0x1B, 0x01, 0xF0, 0xF0])
    for prec in ("fp64", "int8"):
        out = compute_l2_from_bytes(bed, bim, fam, L2Config(mode=WindowMode.Kb(100.0), chunk_size=2,
                                                            precision=prec), ctx=ctx)
        np.testing.assert_allclose(out.l2, [2.0, 2.0], atol=1e-9)
        np.testing.assert_allclose(out.maf, [0.5, 0.5], atol=1e-9)


def test_truncated_bed_is_rejected(ctx):
    from ldsc_b200.api import L2Config, LdscError, compute_l2_from_bytes
    bim = "1\trs1\t0\t100\tA\tG\n1\trs2\t0\t200\tA\tG\n"
    fam = "".join(f"F{i}\tI{i}\t0\t0\t1\t-9\n" for i in range(1, 5))
    with pytest.raises(LdscError, match="invalid length"):
        compute_l2_from_bytes(bytes([0x6C, 0x1B, 0x01, 0xF0]), bim, fam, L2Config(), ctx=ctx)


EXACT_MODES = ["cm1_chunk50", "cm1_masked", "cm1_global", "kb500_chunk40", "snp25_masked",
               "cm1_perallele"]


@pytest.mark.parametrize("precision", ["fp64", "int8"])
@pytest.mark.parametrize("name", EXACT_MODES)
def test_exact_modes_match_oracle(ctx, small, small_panel, name, precision):
    l2, maf, perf = run_mode(ctx, small, small_panel, name, precision)
    assert relerr(l2, small[f"l2_{name}"]) < EXACT_TOL
    np.testing.assert_allclose(maf, small[f"maf_{name}"], atol=1e-15)
    assert perf.n_pairs == int(small[f"pairs_{name}"])


@pytest.mark.parametrize("precision", ["fp64", "int8"])
def test_annotations_match_oracle(ctx, small, small_panel, precision):
    l2, _, _ = run_mode(ctx, small, small_panel, "cm1_annot3", precision)
    ref = small["l2_cm1_annot3"]
    assert entry_relerr(l2, ref) < ANNOT_TOL


def test_fast_f32_flag_within_reference_tolerance(ctx, small, small_panel):
    """--fast-f32 is accepted; the GPU keeps exact arithmetic, which agrees
    with the reference's f32 output within its 2e-2 parity tolerance."""
    l2, _, _ = run_mode(ctx, small, small_panel, "cm1_f32", "int8")
    assert np.max(np.abs(l2 - small["l2_cm1_f32"])) < 2e-2
    assert relerr(l2, small["l2_cm1_chunk50"]) < EXACT_TOL


SKETCH_MODES = ["cm1_sketch50", "cm1_sketch200", "cm1_sketch50_maf", "cm1_sketch200_maf"]


@pytest.mark.parametrize("name", SKETCH_MODES)
def test_sketch_matches_oracle(ctx, small, small_panel, name):
    """CountSketch d = 50 and 200, seed-42 stream, plain and MAF-aware
    correction, against the oracle's f32 --sketch path.  The sketched values
    differ only by rounding (here each bucket is summed exactly and rounded to
    f32 once; the reference accumulates f32 in individual order), and the dot
    products are f32-accurate on both sides."""
    l2, maf, _ = run_mode(ctx, small, small_panel, name, "fp64")
    ref = small[f"l2_{name}"]
    assert np.max(np.abs(l2 - ref)) < SKETCH_TOL
    np.testing.assert_allclose(maf, small[f"maf_{name}"], atol=1e-15)


@pytest.mark.parametrize("d", [50, 200])
def test_sketch_maf_aware_correction_runs(ctx, small, small_panel, d):
    """--sketch-maf-aware is the kurtosis-shifted inversion, not the plain one:
    the two differ by far more than the parity tolerance, as in the oracle."""
    aware = run_mode(ctx, small, small_panel, f"cm1_sketch{d}_maf", "fp64")[0]
    plain = run_mode(ctx, small, small_panel, f"cm1_sketch{d}", "fp64")[0]
    gap = np.max(np.abs(aware - plain))
    want = np.max(np.abs(small[f"l2_cm1_sketch{d}_maf"] - small[f"l2_cm1_sketch{d}"]))
    assert gap > 100 * SKETCH_TOL
    assert abs(gap - want) < 2 * SKETCH_TOL


def test_keep_subset_matches_oracle(ctx, small, small_panel):
    from ldsc_b200.api import WindowMode, run_l2
    from oracle import OracleL2Args, oracle_l2
    n = int(small["n_indiv"])
    keep = np.arange(3, n, 2, dtype=np.int64)
    snps = table(small["chr"], small["cm"], small["bp"])
    ref, ref_maf, _, _ = oracle_l2(OracleL2Args(bed_body=small["body"], n_file_indiv=n, chr=small["chr"],
                                                cm=small["cm"], bp=small["bp"], chunk_c=50, iid_idx=keep))
    for prec in ("fp64", "int8"):
        l2, maf, _ = run_l2(ctx, snps, small_panel, WindowMode.Cm(1.0), 50, iid_indices=keep,
                            precision=prec, yes_really=True)
        assert relerr(l2, ref) < EXACT_TOL
        np.testing.assert_allclose(maf, ref_maf, atol=1e-15)


def test_extract_subset_matches_oracle(ctx, small, small_panel):
    """Non-contiguous SNP records (--extract with gaps)."""
    from ldsc_b200.api import WindowMode, run_l2
    from oracle import OracleL2Args, oracle_l2
    n = int(small["n_indiv"])
    rows = np.sort(np.random.default_rng(3).choice(len(small["chr"]), 900, replace=False))
    snps = table(small["chr"][rows], small["cm"][rows], small["bp"][rows])
    snps.bed_idx = rows.astype(np.int64)
    ref, _, _, _ = oracle_l2(OracleL2Args(bed_body=small["body"], n_file_indiv=n, chr=small["chr"][rows],
                                          cm=small["cm"][rows], bp=small["bp"][rows], bed_idx=rows,
                                          chunk_c=50, masking=True))
    for prec in ("fp64", "int8"):
        l2, _, _ = run_l2(ctx, snps, small_panel, WindowMode.Cm(1.0), 50, snp_level_masking=True,
                          precision=prec, yes_really=True)
        assert relerr(l2, ref) < EXACT_TOL


@pytest.fixture(scope="module")
def fused_ctx():
    """A context that runs the INT8 form as the fused packed-row Gram."""
    from ldsc_b200.api import Context
    c = Context(0, fused_operands=True)
    yield c
    c.close()


@pytest.mark.parametrize("form", ["fused", "staged"])
def test_int8_gram_tile_is_bit_exact(ctx, fused_ctx, form):
    """Raw INT32 accumulators of one tcgen05 tile vs an integer recompute, for
    the fused Gram (packed rows expanded in shared memory; N = 777 leaves a
    partial last stage) and for the Gram over staged operand rows."""
    from ldsc_b200.api import debug_gram_i8_tile
    from ldsc_b200.plink import decode_genotypes
    ctx = fused_ctx if form == "fused" else ctx
    spec = synth.PanelSpec(n_indiv=777, chrom_sizes=[300], chrom_cm=[3.0], founders=9, miss=0.05, seed=5)
    body = synth.bed_body(spec)
    panel = ctx.upload(body, spec.n_indiv)
    G = decode_genotypes(body, spec.n_indiv)
    Gi = np.where(np.isnan(G), 0, G).astype(np.int64)
    Mi = (~np.isnan(G)).astype(np.int64)
    for k0, j0 in [(0, 0), (64, 128), (192, 128), (256, 256)]:
        D = debug_gram_i8_tile(ctx, panel, k0, j0).astype(np.int64)
        A = np.zeros((128, spec.n_indiv), np.int64)
        B = np.zeros((256, spec.n_indiv), np.int64)
        for r in range(64):
            if k0 + r < spec.m:
                A[2 * r], A[2 * r + 1] = Gi[k0 + r], Mi[k0 + r]
        for r in range(128):
            if j0 + r < spec.m:
                B[2 * r], B[2 * r + 1] = Gi[j0 + r], Mi[j0 + r]
        assert np.array_equal(D, A @ B.T), (k0, j0)


@pytest.mark.parametrize("name", EXACT_MODES + ["cm1_annot3"])
def test_fused_and_staged_int8_forms_agree(ctx, fused_ctx, small, small_panel, name):
    """The fused INT8 Gram and the two-pass form give bit-identical l2: the
    same integer sums, and l2 summed in a fixed order in both."""
    a, ma, pa = run_mode(fused_ctx, small, small_panel, name, "int8")
    b, mb, pb = run_mode(ctx, small, small_panel, name, "int8")
    assert np.array_equal(a, b)
    assert np.array_equal(ma, mb)
    assert pa.n_pairs == pb.n_pairs


@pytest.mark.parametrize("masking", [True, False], ids=["masked", "chunk200"])
@pytest.mark.parametrize("subset", ["all", "every_other"])
def test_overlapped_decode_is_bit_identical(ctx, fused_ctx, subset, masking):
    """Resident panels of 16,384 records or more decode in record chunks on a
    side stream while the Gram runs the tiles of chunks already decoded.  The
    result equals, bit for bit, the fused form's (one Gram over packed rows,
    no chunking) on the same records, including a record list (every other
    row) whose chunks are not row ranges."""
    from ldsc_b200.api import WindowMode, run_l2
    spec = synth.PanelSpec(n_indiv=1500, chrom_sizes=[30000, 14000], chrom_cm=[40.0, 20.0], founders=30,
                           miss=0.02, seed=77)
    chr_, cm, bp = synth.positions(spec)
    panel = ctx.synth(spec.n_indiv, spec.m, spec.founders, spec.switch_p, spec.miss, spec.seed)
    try:
        idx = np.arange(spec.m) if subset == "all" else np.arange(0, spec.m, 2)
        if subset == "every_other":
            assert len(idx) >= 16384   # still the overlapped form
        snps = table(chr_[idx], cm[idx], bp[idx])
        snps.bed_idx = idx.astype(np.int64)
        got, maf, perf = run_l2(ctx, snps, panel, WindowMode.Cm(1.0), 200, snp_level_masking=masking,
                                precision="int8", yes_really=True)
        # the same records as consecutive rows of their own panel, through the fused form
        rows = panel.download()[idx]
        sub = fused_ctx.upload(rows.reshape(-1), spec.n_indiv)
        try:
            snps2 = table(chr_[idx], cm[idx], bp[idx])
            ref, ref_maf, rperf = run_l2(fused_ctx, snps2, sub, WindowMode.Cm(1.0), 200,
                                         snp_level_masking=masking, precision="int8", yes_really=True)
        finally:
            sub.close()
        assert perf.n_pairs == rperf.n_pairs
        np.testing.assert_array_equal(maf, ref_maf)
        np.testing.assert_array_equal(got, ref)
        assert perf.kernel_launches > rperf.kernel_launches   # chunked decode + Gram launches
    finally:
        panel.close()


def test_fused_form_at_wide_rows(ctx, fused_ctx):
    """Rows of 32,768 individuals or more run the fused Gram with four
    epilogue and eight converter warps (narrower rows: eight and four); at
    N = 33,001 (a ragged last stage) its l2 and MAF equal the two-pass form's
    bit for bit, in both window modes."""
    from ldsc_b200.api import WindowMode, run_l2
    spec = synth.PanelSpec(n_indiv=33001, chrom_sizes=[700, 300], chrom_cm=[4.0, 2.0], founders=20, miss=0.02,
                           seed=13)
    chr_, cm, bp = synth.positions(spec)
    snps = table(chr_, cm, bp)
    body = synth.bed_body(spec)
    pa, pb = ctx.upload(body, spec.n_indiv), fused_ctx.upload(body, spec.n_indiv)
    try:
        for masking in (True, False):
            a, ma, _ = run_l2(ctx, snps, pa, WindowMode.Cm(1.0), 200, snp_level_masking=masking, precision="int8",
                              yes_really=True)
            b, mb, _ = run_l2(fused_ctx, snps, pb, WindowMode.Cm(1.0), 200, snp_level_masking=masking,
                              precision="int8", yes_really=True)
            np.testing.assert_array_equal(a, b)
            np.testing.assert_array_equal(ma, mb)
    finally:
        pa.close()
        pb.close()


@pytest.mark.parametrize("n_indiv", [40, 128, 129, 1000])
@pytest.mark.parametrize("form", ["fused", "staged"])
def test_int8_form_at_small_and_ragged_n(ctx, fused_ctx, n_indiv, form):
    """Individual counts around the 128-individual stage: a packed row
    narrower than one stage (N = 40, 16-byte rows), exactly one stage, one
    individual into the next, and a ragged tail; against the brute-force
    definition."""
    from conftest import brute_force_l2
    from ldsc_b200.api import WindowMode, left_limits, run_l2
    ctx = fused_ctx if form == "fused" else ctx
    spec = synth.PanelSpec(n_indiv=n_indiv, chrom_sizes=[260, 140], chrom_cm=[2.0, 1.0], founders=7, miss=0.03,
                           seed=n_indiv)
    body = synth.bed_body(spec)
    chr_, cm, bp = synth.positions(spec)
    snps = table(chr_, cm, bp)
    panel = ctx.upload(body, n_indiv)
    for masking in (True, False):
        l2, maf, _ = run_l2(ctx, snps, panel, WindowMode.Cm(1.0), 50, snp_level_masking=masking,
                            precision="int8", yes_really=True)
        left = left_limits(snps, WindowMode.Cm(1.0), 50, snp_level_masking=masking)
        ref, ref_maf = brute_force_l2(body, n_indiv, chr_, cm, bp, left)
        assert relerr(l2, ref) < EXACT_TOL
        np.testing.assert_allclose(maf, ref_maf, atol=1e-15)
    panel.close()


@pytest.mark.parametrize("precision", ["fp64", "int8"])
def test_l2_is_bit_reproducible(ctx, small, small_panel, precision):
    """Repeated calls give bit-identical l2 (no order-dependent atomics)."""
    a = run_mode(ctx, small, small_panel, "cm1_masked", precision)[0]
    for _ in range(3):
        assert np.array_equal(run_mode(ctx, small, small_panel, "cm1_masked", precision)[0], a)


def test_device_synth_matches_numpy(ctx):
    spec = synth.PanelSpec(n_indiv=1001, chrom_sizes=[2500], chrom_cm=[10.0], founders=40, miss=0.01, seed=9)
    panel = ctx.synth(spec.n_indiv, spec.m, spec.founders, spec.switch_p, spec.miss, spec.seed)
    assert np.array_equal(panel.download(), synth.bed_body(spec))


def test_sketch_project_matches_reference_scatter(ctx):
    """Port of scatter_one_column_f32_matches_ref_all_iids (src/wasm_simd.rs:2918-2998)."""
    from ldsc_b200.api import sketch_project
    from test_oracle import direct_scatter_f32, lcg_bed_fixture, lcg_bucket_sign, snp_mean_inv
    c, n, d = 8, 503, 50
    raw = lcg_bed_fixture(42, c, n)
    bpr = (n + 3) // 4
    bucket, sign = lcg_bucket_sign(n, d, 7)
    panel = ctx.upload(raw, n)
    got = sketch_project(ctx, panel, 0, c, bucket, sign, d)
    for j in range(c):
        g, mean, inv = snp_mean_inv(raw, bpr, j, n)
        exp = direct_scatter_f32(g, bucket, sign, mean, inv, float(n), d)
        diff = np.abs(got[j] - exp)
        assert np.all((diff < 1e-4) | (diff / np.maximum(np.abs(exp), 1e-6) < 1e-4))
    # full keep list == all individuals, bit for bit
    sub = sketch_project(ctx, panel, 0, c, bucket, sign, d, keep=np.arange(n))
    assert np.array_equal(sub, got)


def test_argument_errors(ctx, small, small_panel):
    from ldsc_b200.api import LdscError, WindowMode, run_l2
    snps = table(small["chr"], small["cm"], small["bp"])
    with pytest.raises(LdscError, match="chunk_size must be >= 1"):
        run_l2(ctx, snps, small_panel, WindowMode.Cm(1.0), 0)
    with pytest.raises(LdscError, match="out of bounds"):
        run_l2(ctx, snps, small_panel, WindowMode.Cm(1.0), 50, sketch=2)
    with pytest.raises(LdscError, match="Annotation matrix has"):
        run_l2(ctx, snps, small_panel, WindowMode.Cm(1.0), 50, annot=np.ones((5, 2)))
    # the context stays usable after errors
    l2, _, _ = run_mode(ctx, small, small_panel, "cm1_masked", "int8")
    assert relerr(l2, small["l2_cm1_masked"]) < EXACT_TOL


@pytest.fixture(scope="module")
def cfg_small():
    spec = synth.spec_small()
    body = synth.bed_body(spec)
    chr_, cm, bp = synth.positions(spec)
    return spec, body, chr_, cm, bp


@pytest.mark.parametrize("masking", [False, True])
def test_small_config_parity(ctx, cfg_small, masking):
    """N = 2,490 x M = 18,627, 1 cM, chunk 200: both exact forms within
    1e-6 relative of the f64 oracle (the bar), in practice ~1e-12."""
    from ldsc_b200.api import WindowMode, run_l2
    from oracle import OracleL2Args, oracle_l2
    spec, body, chr_, cm, bp = cfg_small
    ref, ref_maf, npairs, _ = oracle_l2(OracleL2Args(bed_body=body, n_file_indiv=spec.n_indiv, chr=chr_,
                                                     cm=cm, bp=bp, chunk_c=200, masking=masking))
    panel = ctx.upload(body, spec.n_indiv)
    snps = table(chr_, cm, bp)
    for prec in ("fp64", "int8"):
        l2, maf, perf = run_l2(ctx, snps, panel, WindowMode.Cm(1.0), 200, snp_level_masking=masking,
                               precision=prec, yes_really=True)
        err = float(np.max(np.abs(l2 - ref) / np.abs(ref)))
        assert err < 1e-6, (prec, err)
        assert relerr(l2, ref) < EXACT_TOL
        assert perf.n_pairs == npairs
        np.testing.assert_allclose(maf, ref_maf, atol=1e-15)


@pytest.mark.parametrize("d", [3, 200, 2559, 2560, 5000])
def test_sketch_project_large_panel(ctx, d):
    """Bucket sums over a 20,000-individual panel with the seed-42 stream
    (runs shorter and longer than a thread's word range; both kernel forms,
    either side of the d = 2,560 switch) vs a direct f64 scatter; the
    tolerance is the reference scatter test's (1e-4)."""
    from ldsc_b200.api import countsketch_hash, sketch_project
    from ldsc_b200.plink import decode_genotypes
    spec = synth.PanelSpec(n_indiv=20011, chrom_sizes=[6], chrom_cm=[1.0], founders=30, miss=0.03, seed=8)
    body = synth.bed_body(spec)
    panel = ctx.upload(body, spec.n_indiv)
    bucket, sign = countsketch_hash(spec.n_indiv, d, 42)
    got = sketch_project(ctx, panel, 0, spec.m, bucket, sign, d)
    G = decode_genotypes(body, spec.n_indiv)
    for j in range(spec.m):
        g = G[j]
        pres = ~np.isnan(g)
        mean = g[pres].mean()
        var = (np.sum(g[pres] ** 2) - pres.sum() * mean * mean) / spec.n_indiv
        inv = np.float32(1.0 / np.sqrt(var)) if var > 0 else np.float32(0.0)
        mean32 = np.float32(mean)
        val = np.where(pres, (np.nan_to_num(g) - float(mean32)) * float(inv), 0.0)
        col = np.zeros(d)
        np.add.at(col, bucket, sign.astype(np.float64) * val)
        nrm = np.sum(col ** 2)
        if nrm > 0:
            col *= np.sqrt(spec.n_indiv / nrm)
        diff = np.abs(got[j] - col)
        assert np.all((diff < 1e-4) | (diff / np.maximum(np.abs(col), 1e-6) < 1e-4)), (j, diff.max())


@pytest.mark.parametrize("precision", ["fp64", "int8"])
def test_many_annotations_match_oracle(ctx, small, small_panel, precision):
    """K = 33 columns: the contraction splits columns unevenly between threads."""
    from ldsc_b200.api import WindowMode, run_l2
    from oracle import OracleL2Args, oracle_l2
    m = len(small["chr"])
    rng = np.random.default_rng(33)
    A = np.asfortranarray(np.concatenate([np.ones((m, 1)), (rng.random((m, 20)) < 0.2).astype(float),
                                          np.clip(rng.standard_normal((m, 12)), -3, 3)], axis=1))
    n = int(small["n_indiv"])
    ref, _, _, _ = oracle_l2(OracleL2Args(bed_body=small["body"], n_file_indiv=n, chr=small["chr"],
                                          cm=small["cm"], bp=small["bp"], chunk_c=50, annot=A))
    snps = table(small["chr"], small["cm"], small["bp"])
    l2, _, _ = run_l2(ctx, snps, small_panel, WindowMode.Cm(1.0), 50, annot=A, precision=precision,
                      yes_really=True)
    scale = np.maximum(np.abs(ref).max(axis=0, keepdims=True), 1.0)
    assert np.max(np.abs(l2 - ref) / scale) < ANNOT_TOL


@pytest.fixture(scope="module")
def streamed():
    """A 150,000-row panel of 4,000 individuals: 150 MB of BED rows, so the
    whole-file entry point streams it in three 64 MB chunks."""
    spec = synth.PanelSpec(n_indiv=4000, chrom_sizes=[150000], chrom_cm=[60.0], founders=40, miss=0.01,
                           seed=21)
    _, cm, bp = synth.positions(spec)
    return spec, cm, bp


@pytest.mark.parametrize("case", ["all_int8", "all_fp64", "every_other_int8", "unordered_int8", "sketch"])
def test_whole_file_entry_matches_resident_panel(ctx, streamed, case):
    """ldsc_l2_from_bed streams the file through the copy stream and decodes
    chunk by chunk; its results equal a run on the same rows uploaded first."""
    from ldsc_b200.api import WindowMode, l2_from_bed_bytes, run_l2
    spec, cm, bp = streamed
    panel = ctx.synth(spec.n_indiv, spec.m, spec.founders, spec.switch_p, spec.miss, spec.seed)
    rows = panel.download()
    bed = np.concatenate([np.array([0x6C, 0x1B, 0x01], np.uint8), rows.reshape(-1)])
    del rows
    idx = np.arange(spec.m)
    pos = idx
    if case == "every_other_int8":
        idx = pos = idx[::2]
    elif case == "unordered_int8":
        # records out of row order (any BIM-to-row map is legal): the entry
        # point then waits for the whole file before decoding
        pos = idx[:60000]
        idx = pos.reshape(-1, 2)[:, ::-1].reshape(-1)
    snps = table(np.ones(len(idx)), cm[pos], bp[pos])
    snps.bed_idx = idx.astype(np.int64)
    prec = "fp64" if case == "all_fp64" else "int8"
    sk = 200 if case == "sketch" else None
    ref, ref_maf, _ = run_l2(ctx, snps, panel, WindowMode.Cm(1.0), 200, precision=prec, sketch=sk,
                             snp_level_masking=True, yes_really=True)
    got, maf, perf = l2_from_bed_bytes(ctx, bed, spec.n_indiv, snps, WindowMode.Cm(1.0), 200, precision=prec,
                                       sketch=sk, snp_level_masking=True)
    np.testing.assert_array_equal(maf, ref_maf)
    assert relerr(got, ref) < 1e-12
    assert perf.bed_read_secs > 0
