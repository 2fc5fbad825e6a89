"""The `l2` command end to end on a small PLINK fileset (src/l2/mod.rs:46-805):
its .l2.ldscore.gz values against the C oracle (3 decimals, as written),
M / M_5_50 files, per-chromosome files, and the --maf prefilter, --print-snps,
--annot, --per-allele, --extract and --keep paths."""
import gzip
import os

import numpy as np
import pytest

from ldsc_b200 import synth
from ldsc_b200.plink import write_plink

pytestmark = pytest.mark.gpu

N = 600


@pytest.fixture(scope="module")
def bfile(tmp_path_factory):
    d = tmp_path_factory.mktemp("cli")
    spec = synth.PanelSpec(n_indiv=N, chrom_sizes=[1500, 1000], chrom_cm=[10.0, 6.0], founders=30, miss=0.02,
                           seed=51)
    chr_, cm, bp = synth.positions(spec)
    body = synth.bed_body(spec)
    prefix = str(d / "panel")
    write_plink(prefix, body, chr_, cm, bp, N)
    return prefix, body, chr_, cm, bp, d


def read_ldscore(path):
    lines = gzip.open(path, "rt").read().splitlines()
    head = lines[0].split("\t")
    rows = [ln.split("\t") for ln in lines[1:]]
    vals = np.array([[float(x) for x in r[3:]] for r in rows]) if rows else np.zeros((0, len(head) - 3))
    return head, [r[1] for r in rows], vals


def run_cli(*argv):
    from ldsc_b200.cli import main
    assert main(["l2", *argv]) == 0


def test_default_run_matches_oracle(bfile):
    from oracle import OracleL2Args, oracle_l2
    prefix, body, chr_, cm, bp, d = bfile
    out = str(d / "def")
    run_cli("--bfile", prefix, "--out", out, "--ld-wind-cm", "1", "--yes-really")
    head, ids, vals = read_ldscore(out + ".l2.ldscore.gz")
    assert head == ["CHR", "SNP", "BP", "L2"] and len(ids) == 2500
    ref, maf, _, _ = oracle_l2(OracleL2Args(bed_body=body, n_file_indiv=N, chr=chr_, cm=cm, bp=bp, chunk_c=200))
    assert np.max(np.abs(vals[:, 0] - ref[:, 0])) <= 5e-4 + 1e-9
    assert open(out + ".l2.M").read() == "2500\n"
    assert open(out + ".l2.M_5_50").read() == f"{int((maf > 0.05).sum())}\n"
    h1, ids1, v1 = read_ldscore(out + "1.l2.ldscore.gz")
    h2, ids2, v2 = read_ldscore(out + "2.l2.ldscore.gz")
    assert ids1 + ids2 == ids and open(out + "1.l2.M").read() == "1500\n"


def test_maf_prefilter_print_snps_and_masking(bfile):
    from oracle import OracleL2Args, oracle_l2, oracle_snp_stats
    prefix, body, chr_, cm, bp, d = bfile
    ps = d / "print.txt"
    wanted = [f"rs{j + 1}" for j in range(0, 2500, 7)]
    ps.write_text("\n".join(wanted) + "\n")
    out = str(d / "maf")
    run_cli("--bfile", prefix, "--out", out, "--maf", "0.1", "--print-snps", str(ps), "--snp-level-masking")
    maf_all, ok = oracle_snp_stats(body, N, np.arange(2500))
    kept = np.nonzero(ok & (maf_all > 0.1))[0]
    ref, maf, _, _ = oracle_l2(OracleL2Args(bed_body=body, n_file_indiv=N, chr=chr_[kept], cm=cm[kept],
                                            bp=bp[kept], bed_idx=kept, chunk_c=200, masking=True))
    pos = {f"rs{j + 1}": i for i, j in enumerate(kept)}
    head, ids, vals = read_ldscore(out + ".l2.ldscore.gz")
    want_ids = [f"rs{j + 1}" for j in kept if f"rs{j + 1}" in set(wanted) and maf[pos[f'rs{j + 1}']] > 0.1]
    assert ids == want_ids
    assert np.max(np.abs(vals[:, 0] - ref[[pos[i] for i in ids], 0])) <= 5e-4 + 1e-9
    assert open(out + ".l2.M").read() == f"{len(kept)}\n"


def test_annot_per_allele(bfile):
    from oracle import OracleL2Args, oracle_l2, oracle_snp_stats
    prefix, body, chr_, cm, bp, d = bfile
    rng = np.random.default_rng(3)
    A = np.stack([np.ones(2500), (rng.random(2500) < 0.3).astype(float)], axis=1)
    ap = d / "an.annot"
    with open(ap, "w") as f:
        f.write("CHR\tBP\tSNP\tCM\tbase\tcod\n")
        for j in range(2500):
            f.write(f"{chr_[j]}\t{bp[j]}\trs{j + 1}\t{cm[j]}\t{A[j, 0]:g}\t{A[j, 1]:g}\n")
    out = str(d / "ann")
    run_cli("--bfile", prefix, "--out", out, "--annot", str(ap), "--per-allele")
    maf_all, ok = oracle_snp_stats(body, N, np.arange(2500))
    kept = np.nonzero(ok & (maf_all > 0.0))[0]
    pq = maf_all[kept] * (1 - maf_all[kept])
    As = A[kept] * pq[:, None]
    ref, _, _, _ = oracle_l2(OracleL2Args(bed_body=body, n_file_indiv=N, chr=chr_[kept], cm=cm[kept], bp=bp[kept],
                                          bed_idx=kept, chunk_c=200, annot=As))
    head, ids, vals = read_ldscore(out + ".l2.ldscore.gz")
    assert head == ["CHR", "SNP", "BP", "baseL2_S1", "codL2_S1"]
    assert np.max(np.abs(vals - ref)) <= 5e-4 + 1e-9
    mvals = [float(x) for x in open(out + ".l2.M").read().split("\t")]
    np.testing.assert_allclose(mvals, As.sum(axis=0), rtol=1e-12)


def test_extract_and_keep(bfile):
    from oracle import OracleL2Args, oracle_l2
    prefix, body, chr_, cm, bp, d = bfile
    ex = d / "extract.txt"
    rows = np.arange(0, 2500, 2)
    ex.write_text("".join(f"rs{j + 1}\n" for j in rows))
    kp = d / "keep.txt"
    keep = np.arange(0, N, 3)
    kp.write_text("".join(f"F{i + 1} I{i + 1}\n" for i in keep))
    out = str(d / "ek")
    run_cli("--bfile", prefix, "--out", out, "--extract", str(ex), "--keep", str(kp), "--ld-wind-kb", "500")
    ref, _, _, _ = oracle_l2(OracleL2Args(bed_body=body, n_file_indiv=N, chr=chr_[rows], cm=cm[rows], bp=bp[rows],
                                          bed_idx=rows, iid_idx=keep, mode="kb", wind=500.0, chunk_c=200))
    head, ids, vals = read_ldscore(out + ".l2.ldscore.gz")
    assert ids == [f"rs{j + 1}" for j in rows]
    assert np.max(np.abs(vals[:, 0] - ref[:, 0])) <= 5e-4 + 1e-9


def test_snp_stats_matches_oracle(ctx, bfile):
    from ldsc_b200.api import snp_stats
    from ldsc_b200.plink import BimTable
    from oracle import oracle_snp_stats
    prefix, body, chr_, cm, bp, d = bfile
    panel = ctx.upload(body, N)
    rows = np.arange(3, 2500, 5)
    keep = np.arange(1, N, 2)
    snps = BimTable(chr_[rows], [f"rs{j}" for j in rows], cm[rows], bp[rows], rows.astype(np.int64))
    maf, ok = snp_stats(ctx, snps, panel, keep)
    rmaf, rok = oracle_snp_stats(body, N, rows, keep)
    np.testing.assert_allclose(maf, rmaf, rtol=0, atol=1e-15)
    assert (ok == rok).all()
