"""PLINK .bed/.bim/.fam host I/O for the l2 path.

Mirrors the reference's input layer:
  * ``BimRecord`` and the BIM parser  -- src/parse.rs:500-598
  * FAM counting / parsing            -- src/l2/io.rs:9-50
  * BED header + length validation    -- src/bed.rs:53-128 (``Bed::from_bytes``)
Errors are raised as ``ValueError`` with the reference's wording, so callers
see "invalid magic bytes" / "invalid length" exactly where the reference's
``anyhow::ensure!`` fires.
"""
from __future__ import annotations

import dataclasses
import os
from typing import List, Optional, Sequence, Tuple

import numpy as np

BED_MAGIC = bytes([0x6C, 0x1B, 0x01])


@dataclasses.dataclass
class BimTable:
    """Columnar ``Vec<BimRecord>``: chr, snp id, cM, bp, BED row index."""

    chr: np.ndarray       # uint8
    snp: List[str]
    cm: np.ndarray        # float64
    bp: np.ndarray        # uint32
    bed_idx: np.ndarray   # int64
    a1: Optional[List[str]] = None
    a2: Optional[List[str]] = None

    def __len__(self) -> int:
        return len(self.snp)

    def subset(self, rows: Sequence[int]) -> "BimTable":
        rows = np.asarray(rows, dtype=np.int64)
        pick = lambda xs: None if xs is None else [xs[i] for i in rows]  # noqa: E731
        return BimTable(self.chr[rows], pick(self.snp), self.cm[rows], self.bp[rows],
                        self.bed_idx[rows], pick(self.a1), pick(self.a2))


def _parse_chr(tok: str) -> int:
    t = tok.lower()
    if t.startswith("chr"):
        t = t[3:]
    if t == "x":
        return 23
    if t == "y":
        return 24
    return int(t)


def parse_bim_text(text: str) -> BimTable:
    """Parse BIM text (CHR SNP CM BP A1 A2, whitespace separated)."""
    chrs, snps, cms, bps, a1, a2 = [], [], [], [], [], []
    for lineno, line in enumerate(text.splitlines(), 1):
        if not line.strip():
            continue
        cols = line.split()
        if len(cols) < 4:
            raise ValueError(f"BIM line {lineno}: expected >= 4 columns, got {len(cols)}")
        chrs.append(_parse_chr(cols[0]))
        snps.append(cols[1])
        cms.append(float(cols[2]))
        bps.append(int(cols[3]))
        a1.append(cols[4] if len(cols) > 4 else "")
        a2.append(cols[5] if len(cols) > 5 else "")
    m = len(snps)
    return BimTable(np.array(chrs, dtype=np.uint8), snps, np.array(cms, dtype=np.float64),
                    np.array(bps, dtype=np.uint32), np.arange(m, dtype=np.int64), a1, a2)


def parse_bim(path: str) -> BimTable:
    with open(path) as f:
        return parse_bim_text(f.read())


def count_fam_str(text: str) -> int:
    return len(text.splitlines())


def parse_fam_text(text: str) -> List[Tuple[str, str]]:
    ids = []
    for i, line in enumerate(text.splitlines(), 1):
        cols = line.split()
        if len(cols) < 2:
            raise ValueError(f"FAM line {i}: expected >= 2 columns (FID IID ...), got {len(cols)}")
        ids.append((cols[0], cols[1]))
    return ids


def count_fam(path: str) -> int:
    with open(path) as f:
        return count_fam_str(f.read())


def bed_bytes_per_snp(n_indiv: int) -> int:
    return (n_indiv + 3) // 4


def validate_bed(data: bytes | np.ndarray, n_indiv: int, n_snp: int) -> np.ndarray:
    """``Bed::from_bytes`` validation (src/bed.rs:73-110).  Returns the body
    (without the 3 magic bytes) as a uint8 array view."""
    buf = np.frombuffer(data, dtype=np.uint8) if not isinstance(data, np.ndarray) else data
    if buf.size < 3:
        raise ValueError(f"BED too short ({buf.size}B)")
    if buf[0] != 0x6C or buf[1] != 0x1B:
        raise ValueError("BED has invalid magic bytes")
    if buf[2] != 0x01:
        raise ValueError("BED is not SNP-major (mode=1 required)")
    expected = bed_bytes_per_snp(n_indiv) * n_snp + 3
    if buf.size != expected:
        raise ValueError(f"BED has invalid length (expected {expected}, got {buf.size})")
    return buf[3:]


def read_bed(path: str, n_indiv: int, n_snp: int, mmap: bool = False) -> np.ndarray:
    """The validated BED body; with mmap, a read-only memory map of the file
    (rows are read when a slice of them is uploaded)."""
    data = np.memmap(path, dtype=np.uint8, mode="r") if mmap else np.fromfile(path, dtype=np.uint8)
    return validate_bed(data, n_indiv, n_snp)


def write_plink(prefix: str, body: np.ndarray, chr_: np.ndarray, cm: np.ndarray,
                bp: np.ndarray, n_indiv: int, snp_ids: Optional[List[str]] = None) -> None:
    """Write prefix.bed/.bim/.fam for a BED body (M x bpr uint8)."""
    m = len(chr_)
    body = np.ascontiguousarray(body, dtype=np.uint8)
    assert body.size == m * bed_bytes_per_snp(n_indiv)
    with open(prefix + ".bed", "wb") as f:
        f.write(BED_MAGIC)
        f.write(body.tobytes())
    ids = snp_ids or [f"rs{j + 1}" for j in range(m)]
    with open(prefix + ".bim", "w") as f:
        for j in range(m):
            f.write(f"{int(chr_[j])}\t{ids[j]}\t{float(cm[j])!r}\t{int(bp[j])}\tA\tG\n")
    with open(prefix + ".fam", "w") as f:
        for i in range(n_indiv):
            f.write(f"F{i + 1}\tI{i + 1}\t0\t0\t1\t-9\n")


def decode_genotypes(body: np.ndarray, n_indiv: int) -> np.ndarray:
    """Reference decode (count-A1 LUT [2, missing, 1, 0], src/bed.rs:470-521)
    to float64 with NaN at missing; M x N.  Test helper for small panels."""
    body = np.asarray(body, dtype=np.uint8)
    m = body.size // bed_bytes_per_snp(n_indiv)
    b = body.reshape(m, -1)
    codes = np.stack([(b >> (2 * k)) & 3 for k in range(4)], axis=-1).reshape(m, -1)[:, :n_indiv]
    lut = np.array([2.0, np.nan, 1.0, 0.0])
    return lut[codes]


def exists_plink(prefix: str) -> bool:
    return all(os.path.exists(prefix + ext) for ext in (".bed", ".bim", ".fam"))
