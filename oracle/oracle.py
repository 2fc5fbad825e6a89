"""ctypes binding of the C oracle (``ldsc_oracle.c``) -- TEST INFRASTRUCTURE ONLY.

Every function here follows the reference function named in its docstring; the
C file's header lists the reference lines each piece restates.
"""
from __future__ import annotations

import ctypes as C
import dataclasses
from typing import Optional

import numpy as np

from .build import build

_lib = None


def _load():
    global _lib
    if _lib is None:
        _lib = C.CDLL(build())
        _lib.oracle_l2.restype = C.c_int
        _lib.oracle_block_lefts.restype = C.c_int
        _lib.oracle_max_threads.restype = C.c_int
    return _lib


class _Args(C.Structure):
    _fields_ = [
        ("bed", C.c_void_p),
        ("bpr", C.c_int64),
        ("n_file_indiv", C.c_int64),
        ("iid_idx", C.c_void_p),
        ("n_indiv", C.c_int64),
        ("m", C.c_int64),
        ("bed_idx", C.c_void_p),
        ("chr", C.c_void_p),
        ("cm", C.c_void_p),
        ("bp", C.c_void_p),
        ("mode", C.c_int),
        ("wind", C.c_double),
        ("wind_snp", C.c_int64),
        ("chunk_c", C.c_int64),
        ("annot", C.c_void_p),
        ("K", C.c_int64),
        ("has_pq", C.c_int),
        ("pq_exp", C.c_double),
        ("use_f32", C.c_int),
        ("sketch_d", C.c_int64),
        ("sketch_maf_aware", C.c_int),
        ("masking", C.c_int),
        ("per_chr", C.c_int),
        ("n_threads", C.c_int),
    ]


class _Info(C.Structure):
    _fields_ = [("n_pairs", C.c_int64), ("any_full_chr_window", C.c_int), ("n_dots", C.c_int64),
                ("gemm_secs", C.c_double)]


MODE = {"cm": 0, "kb": 1, "snp": 2}


@dataclasses.dataclass
class OracleL2Args:
    """Arguments of ``compute_ldscore_global`` (src/l2/compute.rs:1009-1028)
    plus the per-chromosome / global-pass choice made by ``l2::run``
    (src/l2/mod.rs:439-575)."""

    bed_body: np.ndarray            # uint8, M_file * bpr bytes (no magic header)
    n_file_indiv: int
    chr: np.ndarray                 # uint8 per SNP record
    cm: np.ndarray                  # float64 per SNP record
    bp: np.ndarray                  # uint32 per SNP record
    bed_idx: Optional[np.ndarray] = None   # int64 BED row per record (None = 0..m-1)
    iid_idx: Optional[np.ndarray] = None   # int64 kept individuals (None = all)
    mode: str = "cm"
    wind: float = 1.0
    wind_snp: int = 0
    chunk_c: int = 200
    annot: Optional[np.ndarray] = None     # float64 m x K
    pq_exp: Optional[float] = None
    use_f32: bool = False
    sketch_d: int = 0
    sketch_maf_aware: bool = False
    masking: bool = False
    per_chr: bool = True
    n_threads: int = 0


def oracle_l2(a: OracleL2Args, work: Optional[dict] = None):
    """Returns (l2 [m x K], maf [m], n_pairs, any_full_chr_window).  With a
    ``work`` dict, also fills in the f64 chunk Grams' dot products computed
    (``n_dots``) and their wall time (``gemm_secs``)."""
    lib = _load()
    m = len(a.chr)
    bpr = (a.n_file_indiv + 3) // 4
    bed = np.ascontiguousarray(a.bed_body, dtype=np.uint8)
    chr_ = np.ascontiguousarray(a.chr, dtype=np.uint8)
    cm = np.ascontiguousarray(a.cm, dtype=np.float64)
    bp = np.ascontiguousarray(a.bp, dtype=np.uint32)
    bed_idx = (np.arange(m, dtype=np.int64) if a.bed_idx is None
               else np.ascontiguousarray(a.bed_idx, dtype=np.int64))
    if bed_idx.size and (bed_idx.max() + 1) * bpr > bed.size:
        raise ValueError("bed_idx points past the end of the BED body")
    iid = None if a.iid_idx is None else np.ascontiguousarray(a.iid_idx, dtype=np.int64)
    n_indiv = a.n_file_indiv if iid is None else len(iid)
    annot = None
    K = 1
    if a.annot is not None:
        annot = np.asfortranarray(a.annot, dtype=np.float64)
        if annot.ndim == 1:
            annot = annot.reshape(-1, 1, order="F")
        if annot.shape[0] != m:
            raise ValueError(f"Annotation matrix has {annot.shape[0]} rows but BIM has {m} SNPs")
        K = annot.shape[1]
    args = _Args(
        bed=bed.ctypes.data, bpr=bpr, n_file_indiv=a.n_file_indiv,
        iid_idx=None if iid is None else iid.ctypes.data, n_indiv=n_indiv, m=m,
        bed_idx=bed_idx.ctypes.data, chr=chr_.ctypes.data, cm=cm.ctypes.data, bp=bp.ctypes.data,
        mode=MODE[a.mode], wind=float(a.wind), wind_snp=int(a.wind_snp), chunk_c=int(a.chunk_c),
        annot=None if annot is None else annot.ctypes.data, K=K,
        has_pq=int(a.pq_exp is not None), pq_exp=float(a.pq_exp or 0.0),
        use_f32=int(a.use_f32), sketch_d=int(a.sketch_d), sketch_maf_aware=int(a.sketch_maf_aware),
        masking=int(a.masking), per_chr=int(a.per_chr), n_threads=int(a.n_threads),
    )
    l2 = np.zeros((m, K), dtype=np.float64, order="F")
    maf = np.zeros(m, dtype=np.float64)
    info = _Info()
    err = C.create_string_buffer(512)
    rc = lib.oracle_l2(C.byref(args), l2.ctypes.data_as(C.c_void_p), maf.ctypes.data_as(C.c_void_p),
                       C.byref(info), err, 512)
    if rc != 0:
        raise ValueError(err.value.decode())
    if work is not None:
        work["n_dots"] = int(info.n_dots)
        work["gemm_secs"] = float(info.gemm_secs)
    return l2, maf, int(info.n_pairs), bool(info.any_full_chr_window)


def block_lefts(chr_, cm, bp, mode="cm", wind=1.0, half=0):
    """get_block_lefts_by_chr (src/l2/window.rs:32-90)."""
    lib = _load()
    m = len(chr_)
    chr_ = np.ascontiguousarray(chr_, dtype=np.uint8)
    cm = np.ascontiguousarray(cm, dtype=np.float64)
    bp = np.ascontiguousarray(bp, dtype=np.uint32)
    bl = np.zeros(m, dtype=np.int64)
    full = lib.oracle_block_lefts(C.c_int64(m), chr_.ctypes.data_as(C.c_void_p),
                                  cm.ctypes.data_as(C.c_void_p), bp.ctypes.data_as(C.c_void_p),
                                  C.c_int(MODE[mode]), C.c_double(wind), C.c_int64(half),
                                  bl.ctypes.data_as(C.c_void_p))
    return bl, bool(full)


def countsketch_hash(n_indiv: int, d: int, seed: int = 42):
    """CountSketchProj::new (src/l2/compute.rs:179-192): buckets then signs."""
    lib = _load()
    bucket = np.zeros(n_indiv, dtype=np.uint32)
    sign = np.zeros(n_indiv, dtype=np.float32)
    lib.oracle_countsketch_hash(C.c_int64(n_indiv), C.c_uint32(d), C.c_uint64(seed),
                                bucket.ctypes.data_as(C.c_void_p), sign.ctypes.data_as(C.c_void_p))
    return bucket, sign


def wyrand_stream(seed: int, count: int):
    lib = _load()
    out = np.zeros(count, dtype=np.uint64)
    lib.oracle_wyrand_stream(C.c_uint64(seed), C.c_int64(count), out.ctypes.data_as(C.c_void_p))
    return out


def scatter_column_f32(row: np.ndarray, n_indiv: int, bucket, sign, mean: float, inv_std: float,
                       n_norm: float, d: int, iid_idx=None):
    """scatter_one_column_f32_scalar (src/wasm_simd.rs:1691-1784) on one SNP row."""
    lib = _load()
    row = np.ascontiguousarray(row, dtype=np.uint8)
    bucket = np.ascontiguousarray(bucket, dtype=np.uint32)
    sign = np.ascontiguousarray(sign, dtype=np.float32)
    iid = None if iid_idx is None else np.ascontiguousarray(iid_idx, dtype=np.int64)
    out = np.zeros(d, dtype=np.float32)
    lib.oracle_scatter_column_f32(
        row.ctypes.data_as(C.c_void_p), None if iid is None else iid.ctypes.data_as(C.c_void_p),
        C.c_int64(n_indiv), bucket.ctypes.data_as(C.c_void_p), sign.ctypes.data_as(C.c_void_p),
        C.c_float(mean), C.c_float(inv_std), C.c_double(n_norm), C.c_int64(d),
        out.ctypes.data_as(C.c_void_p))
    return out


def max_threads() -> int:
    return int(_load().oracle_max_threads())


def oracle_snp_stats(bed_body: np.ndarray, n_file_indiv: int, bed_idx: np.ndarray,
                     iid_idx: Optional[np.ndarray] = None):
    """compute_snp_stats (src/l2/snp_stats.rs:5-195): per record, MAF from
    sum / (2 count) over the kept individuals, and het + missing < n.
    Codes: 00 -> 2, 01 -> missing, 10 -> 1 (het), 11 -> 0."""
    bpr = (n_file_indiv + 3) // 4
    rows = np.asarray(bed_body, dtype=np.uint8).reshape(-1, bpr)[np.asarray(bed_idx, dtype=np.int64)]
    codes = np.stack([(rows >> (2 * k)) & 3 for k in range(4)], axis=-1).reshape(len(rows), -1)[:, :n_file_indiv]
    if iid_idx is not None:
        codes = codes[:, np.asarray(iid_idx, dtype=np.int64)]
    n = codes.shape[1]
    count = (codes != 1).sum(axis=1)
    s = 2 * (codes == 0).sum(axis=1) + (codes == 2).sum(axis=1)
    het = (codes == 2).sum(axis=1)
    freq = np.where(count > 0, s / np.maximum(2.0 * count, 1), 0.0)
    maf = np.minimum(freq, 1.0 - freq)
    ok = het + (n - count) < n
    return maf, ok
