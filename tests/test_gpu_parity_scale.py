"""GPU parity against the CPU oracle at the benchmark configurations' own
individual counts (through the C ABI), on SNP samples the oracle finishes in
seconds:

* biobank shape, N = 50,000: the first 1,500 SNPs of the seeded panel, 1 cM,
  per-SNP masking and the default chunk-200 mode, INT8 and FP64 forms,
  max relative error per l2_j <= 1e-6 (the bar for exact mode);
* partitioned shape, N = 10,000: chromosomes 21 and 22 of the 22-chromosome
  panel (5,928 SNPs) with all 97 annotations (all-ones, 80 binary, 16
  continuous), default chunk-200 mode, max relative error per l2_jC <= 1e-6
  in every column;
* CountSketch shape, N = 100,000: the first 600 SNPs of the seeded sketch
  panel, d = 200, 1000 and 5000 (the last on the large-d kernel), plain and
  MAF-aware, per-SNP masking, against the oracle's f32 --sketch path with the
  same seed-42 stream.  The two differ by rounding only (buckets summed
  exactly and rounded to f32 once here, accumulated in f32 in individual
  order by the reference; f32 dot products on both sides); the bar, 6e-5
  absolute per l2_j, is about twice the largest difference measured on 2,000
  SNPs of this panel.
"""
import numpy as np
import pytest

from ldsc_b200 import synth
from ldsc_b200.plink import BimTable

pytestmark = pytest.mark.gpu

PER_L2J_TOL = 1e-6   # exact mode: max_j |l2_j - oracle_j| / |oracle_j|
SKETCH_ABS_TOL = 6e-5  # sketch mode: max_j |l2_j - oracle_j|


def table(chr_, cm, bp, rows=None):
    m = len(chr_)
    return BimTable(np.asarray(chr_, np.uint8), [f"rs{i}" for i in range(m)], np.asarray(cm, float),
                    np.asarray(bp, np.uint32), np.arange(m, dtype=np.int64) if rows is None else rows)


@pytest.fixture(scope="module")
def biobank(ctx):
    """The first 1,500 SNPs of the seeded biobank panel, generated on the
    device (the device generator is byte-identical to synth.bed_body) and
    downloaded for the oracle."""
    spec = synth.spec_biobank()
    m = 1500
    chr_, cm, bp = synth.positions(spec)
    panel = ctx.synth(spec.n_indiv, m, spec.founders, spec.switch_p, spec.miss, spec.seed)
    yield spec, panel, panel.download(), table(chr_[:m], cm[:m], bp[:m]), (chr_[:m], cm[:m], bp[:m])
    panel.close()


@pytest.mark.parametrize("masking", [True, False], ids=["masked", "chunk200"])
def test_biobank_n_matches_oracle_per_l2j(ctx, biobank, masking):
    from ldsc_b200.api import WindowMode, run_l2
    from oracle import OracleL2Args, oracle_l2
    spec, panel, rows, snps, (chr_, cm, bp) = biobank
    ref, ref_maf, pairs, _ = oracle_l2(OracleL2Args(bed_body=rows, n_file_indiv=spec.n_indiv, chr=chr_, cm=cm,
                                                    bp=bp, chunk_c=200, masking=masking))
    assert np.min(np.abs(ref)) > 0.5
    for prec in ("int8", "fp64"):
        l2, maf, perf = run_l2(ctx, snps, panel, WindowMode.Cm(1.0), 200, snp_level_masking=masking,
                               precision=prec, yes_really=True)
        assert perf.n_pairs == pairs
        assert np.max(np.abs(l2[:, 0] - ref[:, 0]) / np.abs(ref[:, 0])) < PER_L2J_TOL, prec
        np.testing.assert_allclose(maf, ref_maf, atol=1e-15)


def test_partitioned_k97_matches_oracle_per_l2jc(ctx):
    from ldsc_b200.api import WindowMode, run_l2
    from oracle import OracleL2Args, oracle_l2
    spec = synth.spec_partitioned()
    chr_, cm, bp = synth.positions(spec)
    annot = synth.partitioned_annot(spec.m)
    start = int(np.searchsorted(chr_, 21))
    panel = ctx.synth(spec.n_indiv, spec.m, spec.founders, spec.switch_p, spec.miss, spec.seed)
    try:
        rows = panel.download(start, spec.m)
        sub = table(chr_[start:], cm[start:], bp[start:], np.arange(start, spec.m, dtype=np.int64))
        ref, ref_maf, pairs, _ = oracle_l2(OracleL2Args(bed_body=rows, n_file_indiv=spec.n_indiv, chr=chr_[start:],
                                                        cm=cm[start:], bp=bp[start:], chunk_c=200,
                                                        annot=annot[start:]))
        for prec in ("int8", "fp64"):
            l2, maf, perf = run_l2(ctx, sub, panel, WindowMode.Cm(1.0), 200, annot=annot[start:], precision=prec,
                                   yes_really=True)
            assert perf.n_pairs == pairs
            # entries the oracle has at exactly 0 (no annotated SNP in the window) must be 0 too
            rel = np.abs(l2 - ref) / np.maximum(np.abs(ref), 1e-300)
            assert rel.max() < PER_L2J_TOL, (prec, float(rel.max()))
            np.testing.assert_allclose(maf, ref_maf, atol=1e-15)
    finally:
        panel.close()


@pytest.fixture(scope="module")
def sketch_sample(ctx):
    spec = synth.spec_sketch()
    m = 600
    chr_, cm, bp = synth.positions(spec)
    panel = ctx.synth(spec.n_indiv, m, spec.founders, spec.switch_p, spec.miss, spec.seed)
    yield spec, panel, panel.download(), table(chr_[:m], cm[:m], bp[:m]), (chr_[:m], cm[:m], bp[:m])
    panel.close()


@pytest.mark.parametrize("d,maf_aware", [(200, False), (1000, False), (5000, False), (1000, True)])
def test_sketch_at_n100000_matches_oracle(ctx, sketch_sample, d, maf_aware):
    from ldsc_b200.api import WindowMode, run_l2
    from oracle import OracleL2Args, oracle_l2
    spec, panel, rows, snps, (chr_, cm, bp) = sketch_sample
    ref, ref_maf, _, _ = oracle_l2(OracleL2Args(bed_body=rows, n_file_indiv=spec.n_indiv, chr=chr_, cm=cm, bp=bp,
                                                chunk_c=200, masking=True, use_f32=True, sketch_d=d,
                                                sketch_maf_aware=maf_aware))
    l2, maf, _ = run_l2(ctx, snps, panel, WindowMode.Cm(1.0), 200, snp_level_masking=True, sketch=d,
                        sketch_maf_aware=maf_aware, yes_really=True)
    assert np.max(np.abs(l2[:, 0] - ref[:, 0])) < SKETCH_ABS_TOL, (d, maf_aware)
    np.testing.assert_allclose(maf, ref_maf, atol=1e-15)
