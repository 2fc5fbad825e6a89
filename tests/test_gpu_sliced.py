"""l2 in SNP slices (ldsc_b200.sliced) against one resident run of the same
panel, and the CLI's sliced path against its resident path.

Tolerance: each slice sums the same pair contributions into l2 in its own
tile order (tile grids start at each call's first record).  The sums are f64
for one annotation column and for K > 1 alike, and agree to 1e-12 of the
column's largest value.  The written files are identical.
"""
import gzip
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _panel():
    from ldsc_b200 import synth
    spec = synth.PanelSpec(n_indiv=1200, chrom_sizes=[2500, 1500, 2000], chrom_cm=[9.0, 5.0, 7.0], founders=40,
                           miss=0.01, seed=71)
    chr_, cm, bp = synth.positions(spec)
    return spec, synth.bed_body(spec), chr_, cm, bp


def _snps(chr_, cm, bp, rows=None):
    from ldsc_b200.plink import BimTable
    m = len(chr_)
    t = BimTable(chr_, [f"rs{i}" for i in range(m)], cm, bp, np.arange(m, dtype=np.int64))
    return t if rows is None else t.subset(rows)


CASES = [  # (precision, masking, global_pass, sketch, K)
    ("int8", False, False, None, 1), ("int8", True, False, None, 1), ("fp64", False, True, None, 1),
    ("int8", True, True, None, 1), ("fp64", False, False, 64, 1), ("int8", False, False, None, 2),
    ("fp64", True, False, None, 2)]


@pytest.mark.parametrize("precision,masking,global_pass,sketch,k", CASES)
def test_sliced_equals_resident(ctx, precision, masking, global_pass, sketch, k):
    from ldsc_b200.api import WindowMode, run_l2
    from ldsc_b200.sliced import run_l2_sliced
    spec, body, chr_, cm, bp = _panel()
    rows = np.array([i for i in range(spec.m) if i % 7 != 3])     # --extract-like gaps in the BED rows
    snps = _snps(chr_, cm, bp, rows)
    rng = np.random.default_rng(3)
    annot = None if k == 1 else np.stack([np.ones(len(snps)), rng.normal(size=len(snps))], axis=1)
    mode = WindowMode.Cm(1.0)
    kw = dict(annot=annot, snp_level_masking=masking, global_pass=global_pass, precision=precision, sketch=sketch)
    panel = ctx.upload(body, spec.n_indiv)
    try:
        want, maf_w, _ = run_l2(ctx, snps, panel, mode, 200, yes_really=True, **kw)
    finally:
        panel.close()
    got, maf_g, slices, perfs = run_l2_sliced(ctx, snps, body, spec.n_indiv, mode, 200, max_call_records=1800, **kw)
    assert len(slices) >= 4 and all(s.call_hi - s.call_lo <= 1800 for s in slices)
    scale = np.abs(want).max(axis=0, keepdims=True)
    np.testing.assert_allclose(got / scale, want / scale, rtol=0, atol=1e-12)
    np.testing.assert_array_equal(maf_g, maf_w)


def test_budget_in_bytes(ctx):
    from ldsc_b200.api import WindowMode, run_l2
    from ldsc_b200.sliced import call_bytes_per_record, run_l2_sliced
    spec, body, chr_, cm, bp = _panel()
    snps = _snps(chr_, cm, bp)
    mode = WindowMode.Cm(1.0)
    per = call_bytes_per_record(snps, spec.n_indiv, mode, 200, precision="int8")
    budget = int(per * spec.m / 3)
    panel = ctx.upload(body, spec.n_indiv)
    try:
        want, _, _ = run_l2(ctx, snps, panel, mode, 200, precision="int8")
    finally:
        panel.close()
    got, _, slices, _ = run_l2_sliced(ctx, snps, body, spec.n_indiv, mode, 200, device_budget_bytes=budget,
                                      precision="int8")
    assert len(slices) >= 3
    np.testing.assert_allclose(got, want, rtol=1e-12, atol=1e-12)


def test_cli_sliced_path_writes_the_same_files(ctx, tmp_path):
    from ldsc_b200.cli import build_parser, run
    from ldsc_b200.plink import write_plink
    spec, body, chr_, cm, bp = _panel()
    prefix = str(tmp_path / "p")
    write_plink(prefix, body.reshape(spec.m, -1), chr_, cm, bp, spec.n_indiv)
    outs = {}
    for tag, extra in (("res", []), ("sl", ["--max-device-gb", "0.004"])):
        out = str(tmp_path / tag)
        args = build_parser().parse_args(["--bfile", prefix, "--out", out, "--ld-wind-cm", "1", "--maf", "0.01",
                                          "--yes-really"] + extra)
        run(args, ctx)
        with gzip.open(out + ".l2.ldscore.gz", "rt") as f:
            outs[tag] = (f.read(), open(out + ".l2.M").read(), open(out + ".l2.M_5_50").read())
    assert outs["res"] == outs["sl"]
