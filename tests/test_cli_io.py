"""Output formats and flag checks of the `l2` command (CPU only):
src/l2/io.rs:93-165 and src/l2/mod.rs:55-97, 807-933."""
import gzip
import math

import numpy as np
import pytest

from ldsc_b200 import io as lio
from ldsc_b200.plink import BimTable


@pytest.mark.parametrize("v,want", [(1000.0, "1000"), (0.5, "0.5"), (1e20, "100000000000000000000"),
                                    (1.5e-7, "0.00000015"), (123.456, "123.456"), (-2.0, "-2"),
                                    (0.1 + 0.2, "0.30000000000000004"), (float("nan"), "NaN"),
                                    (float("inf"), "inf")])
def test_rust_f64_display(v, want):
    assert lio.rust_f64(v) == want


def test_m_file_format():
    assert lio.format_m_vals([18627.0]) == "18627\n"
    assert lio.format_m_vals([3.0, 0.25]) == "3\t0.25\n"


def test_ldscore_writer(tmp_path):
    snps = BimTable(np.array([1, 1, 2], np.uint8), ["a", "b", "c"], np.zeros(3), np.array([10, 20, 5], np.uint32),
                    np.arange(3, dtype=np.int64))
    l2 = np.array([[1.23456, 2.0], [0.0004, -0.0006], [7.0, 8.5]])
    p = tmp_path / "x.l2.ldscore.gz"
    lio.write_ldscore(str(p), snps, np.array([0, 2]), l2[[0, 2]], ["AL2", "BL2"])
    lines = gzip.open(p, "rt").read().splitlines()
    assert lines == ["CHR\tSNP\tBP\tAL2\tBL2", "1\ta\t10\t1.235\t2.000", "2\tc\t5\t7.000\t8.500"]


def test_descriptive_stats_follow_the_reference():
    v = np.array([4.0, 1.0, 3.0, 2.0])
    assert lio._stat(v, "mean") == 2.5
    assert lio._stat(v, "std") == pytest.approx(math.sqrt(5.0 / 3.0))
    assert lio._stat(v, "25%") == pytest.approx(1.75)   # linear interpolation, as pandas
    assert lio._stat(v, "50%") == pytest.approx(2.5)
    assert math.isnan(lio._corr(v, np.ones(4)))


def test_summary_block(capsys):
    lio.print_ld_score_summary("o.l2.ldscore.gz", np.array([0.1, 0.2, 0.3]), np.array([[1.0], [2.0], [4.0]]), ["L2"])
    out = capsys.readouterr().out.splitlines()
    assert out[1] == "Summary of LD Scores in o.l2.ldscore.gz"
    assert out[2] == " " * 8 + "     MAF      L2"
    assert out[3] == "    mean  0.2000  2.3333"
    assert out[-2] == "     MAF  1.0000  0.9820"


@pytest.mark.parametrize("extra,msg", [(["--per-allele", "--pq-exp", "1"], "Cannot set both"),
                                       (["--ld-wind-cm", "1", "--ld-wind-kb", "100"], "exactly one"),
                                       (["--python-compat", "--snp-level-masking"], "incompatible"),
                                       (["--sketch-maf-aware"], "requires --sketch")])
def test_flag_conflicts(tmp_path, extra, msg):
    from ldsc_b200.cli import build_parser, run
    args = build_parser().parse_args(["--bfile", str(tmp_path / "none"), "--out", str(tmp_path / "o")] + extra)
    with pytest.raises(ValueError, match=msg):
        run(args)
