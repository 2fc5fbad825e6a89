"""Input readers and output writers of the `l2` command (src/l2/io.rs,
src/l2/mod.rs:584-955, src/parse.rs:159-230).

Outputs are the reference's formats: `{out}.l2.ldscore.gz` (gzip TSV,
`CHR SNP BP {name}L2...`, values with 3 decimals), `{out}.l2.M` and
`{out}.l2.M_5_50` (tab-joined values, Rust `f64` Display), the per-chromosome
files, and the "Summary of LD Scores" block on stdout.
"""
from __future__ import annotations

import bz2
import decimal
import gzip
import math
import os
from typing import List, Optional, Sequence, Set, Tuple

import numpy as np

from .plink import BimTable


def rust_f64(v: float) -> str:
    """Rust's `{}` Display of an f64: the shortest round-trip digits, never in
    exponent form, no trailing `.0` for integral values."""
    if math.isnan(v):
        return "NaN"
    if math.isinf(v):
        return "inf" if v > 0 else "-inf"
    if v == 0.0:
        return "-0" if math.copysign(1.0, v) < 0 else "0"
    s = repr(float(v))
    if "e" in s or "E" in s:
        s = format(decimal.Decimal(s), "f")
    if s.endswith(".0"):
        s = s[:-2]
    return s


def _open_text(path: str):
    if path.endswith(".gz"):
        return gzip.open(path, "rt")
    if path.endswith(".bz2"):
        return bz2.open(path, "rt")
    return open(path, "r")


def load_snp_set(path: str) -> Set[str]:
    """load_snp_set (src/l2/io.rs:167-187): first token per line, `#` lines skipped."""
    out = set()
    with _open_text(path) as f:
        for line in f:
            if line.lstrip().startswith("#"):
                continue
            tok = line.split()
            if tok:
                out.add(tok[0])
    print(f"  Loaded {len(out)} SNP IDs from '{path}'")
    return out


def load_print_snps(path: str) -> Set[str]:
    """load_print_snps (src/l2/io.rs:190-209): exactly one column of SNP IDs."""
    out = set()
    with _open_text(path) as f:
        for line in f:
            if line.lstrip().startswith("#"):
                continue
            tok = line.split()
            if not tok:
                continue
            if len(tok) != 1:
                raise ValueError("--print-snps must refer to a file with a one column of SNP IDs.")
            out.add(tok[0])
    print(f"  Loaded {len(out)} SNP IDs from '{path}'")
    return out


def load_individual_indices(keep_path: str, fam_ids: Sequence[Tuple[str, str]]) -> np.ndarray:
    """load_individual_indices (src/l2/io.rs:55-91): FAM rows whose (FID, IID)
    appear in the keep file, in FAM order."""
    keep = set()
    with _open_text(keep_path) as f:
        for line in f:
            if line.lstrip().startswith("#"):
                continue
            tok = line.split()
            if len(tok) >= 2:
                keep.add((tok[0], tok[1]))
    idx = np.array([i for i, fi in enumerate(fam_ids) if tuple(fi) in keep], dtype=np.int64)
    if idx.size == 0:
        raise ValueError(f"--keep '{keep_path}': none of {len(keep)} individuals matched the FAM "
                         f"({len(fam_ids)} individuals)")
    print(f"  --keep: retaining {idx.size}/{len(fam_ids)} individuals")
    return idx


def resolve_annot_path(prefix: str) -> str:
    """resolve_annot_path (src/parse.rs:166-189)."""
    if prefix.endswith((".annot", ".annot.gz", ".annot.bz2")):
        if os.path.exists(prefix):
            return prefix
        raise FileNotFoundError(f"Annotation file not found: '{prefix}'")
    for suf in (".annot.gz", ".annot.bz2", ".annot"):
        if os.path.exists(prefix + suf):
            return prefix + suf
    raise FileNotFoundError(f"Annotation file not found: '{prefix}.annot[.gz|.bz2]'")


def read_annot_path(path: str, thin: bool) -> Tuple[np.ndarray, List[str]]:
    """read_annot_path (src/parse.rs:191-230): whitespace-separated table with
    a header; annotation columns start at index 4 (CHR SNP BP CM ...) or 0
    (--thin-annot); missing values read as 0."""
    import pandas as pd
    df = pd.read_csv(path, sep=r"\s+", compression="infer")
    skip = 0 if thin else 4
    cols = list(df.columns)
    if len(cols) <= skip:
        raise ValueError(f"Annot file '{path}' has {len(cols)} columns; expected > {skip} "
                         f"({'thin format' if thin else 'full format: CHR SNP BP CM + annotations'})")
    names = [str(c) for c in cols[skip:]]
    mat = np.array(df[cols[skip:]].apply(pd.to_numeric, errors="coerce").to_numpy(dtype=np.float64), order="F")
    mat[np.isnan(mat)] = 0.0
    return mat, names


def write_ldscore(path: str, snps: BimTable, rows: np.ndarray, l2: np.ndarray, col_names: Sequence[str]):
    """write_ldscore_refs (src/l2/io.rs:93-125): gzip TSV, `{:.3}` values."""
    with gzip.open(path, "wt", compresslevel=1) as f:
        f.write("CHR\tSNP\tBP" + "".join("\t" + n for n in col_names) + "\n")
        for t, i in enumerate(rows):
            vals = "".join("\t%.3f" % l2[t, k] for k in range(len(col_names)))
            f.write(f"{int(snps.chr[i])}\t{snps.snp[i]}\t{int(snps.bp[i])}{vals}\n")


def format_m_vals(vals: Sequence[float]) -> str:
    """format_m_vals (src/l2/io.rs:158-165)."""
    return "\t".join(rust_f64(float(v)) for v in vals) + "\n"


def _stat(vals: np.ndarray, label: str) -> float:
    """compute_descriptive_stat (src/l2/mod.rs:868-891); percentiles with linear
    interpolation (src/l2/mod.rs:893-911)."""
    n = len(vals)
    if n == 0:
        return float("nan")
    if label == "mean":
        return float(vals.sum() / n)
    if label == "std":
        mean = vals.sum() / n
        return float(math.sqrt(((vals - mean) ** 2).sum() / max(n - 1, 1)))
    if label == "min":
        return float(vals.min())
    if label == "max":
        return float(vals.max())
    q = {"25%": 0.25, "50%": 0.50, "75%": 0.75}[label]
    s = np.sort(vals)
    if n == 1:
        return float(s[0])
    pos = q * (n - 1)
    lo = int(math.floor(pos))
    hi = lo + 1
    frac = pos - lo
    return float(s[lo]) if hi >= n else float(s[lo] * (1.0 - frac) + s[hi] * frac)


def _corr(x: np.ndarray, y: np.ndarray) -> float:
    """pearson_corr (src/l2/mod.rs:913-933)."""
    dx, dy = x - x.mean(), y - y.mean()
    vx, vy = float((dx * dx).sum()), float((dy * dy).sum())
    if vx == 0.0 or vy == 0.0:
        return float("nan")
    return float((dx * dy).sum()) / math.sqrt(vx * vy)


def _cell(v: float, w: int = 8) -> str:
    if math.isnan(v):
        return "NaN".rjust(w)
    return f"{v:>{w}.4f}"


def print_ld_score_summary(out_path: str, maf: np.ndarray, l2: np.ndarray, col_names: Sequence[str]):
    """print_ld_score_summary (src/l2/mod.rs:807-866)."""
    if len(maf) == 0:
        return
    cols = [("MAF", np.asarray(maf, dtype=np.float64))] + \
           [(n, np.asarray(l2[:, k], dtype=np.float64)) for k, n in enumerate(col_names)]
    print(f"\nSummary of LD Scores in {out_path}")
    print(" " * 8 + "".join(f"{n:>8}" for n, _ in cols))
    for label in ("mean", "std", "min", "25%", "50%", "75%", "max"):
        print(f"{label:>8}" + "".join(_cell(_stat(v, label)) for _, v in cols))
    print()
    print("MAF/LD Score Correlation Matrix")
    print(" " * 8 + "".join(f"{n:>8}" for n, _ in cols))
    for i, (ni, vi) in enumerate(cols):
        print(f"{ni:>8}" + "".join(_cell(1.0 if i == j else _corr(vi, vj)) for j, (_, vj) in enumerate(cols)))
