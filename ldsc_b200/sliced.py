"""l2 over a panel larger than device memory: the run in consecutive SNP
slices on one device.

The reference streams the BED file through a ring of chunk windows
(src/l2/compute.rs:1164-1299) and never holds more than one window.  The
engine holds a whole call's panel rows and decoded operands in HBM, so a
panel beyond that budget runs as slices: each slice uploads only the BED rows
of its call range (core plus halos, `parallel.call_range`), computes them and
keeps the core rows.  The result equals the unsliced run up to the order in
which pair contributions are summed.
"""
from __future__ import annotations

import ctypes as C
from typing import List, Optional, Tuple

import numpy as np

from . import _lib as L
from .api import Context, L2Perf, LdscError, WindowMode, _ArgPack, run_l2
from .parallel import Shard, plan_slices
from .plink import BimTable


def call_bytes_per_record(snps: BimTable, n_indiv: int, mode: WindowMode, chunk_c: int = 200,
                          annot=None, iid_indices=None, precision: str = "fp64", sketch=None,
                          snp_level_masking: bool = False, global_pass: bool = False) -> float:
    """Device bytes per record of an l2 call: the engine's workspace estimate
    for the whole record list (ldsc_l2_workspace_bytes) per record, plus the
    record's panel row (twice with a sketch: the bucket-major copy)."""
    m = len(snps)
    if m == 0:
        return 0.0
    pack = _ArgPack(snps, mode, chunk_c, annot, iid_indices, None, True, False, sketch, False,
                    snp_level_masking, precision, global_pass, None)
    out = C.c_uint64()
    rc = L.load().ldsc_l2_workspace_bytes(C.byref(pack.args), n_indiv, C.byref(out))
    if rc != L.LDSC_OK:
        raise LdscError(rc, "workspace estimate failed")
    bpr = (n_indiv + 3) // 4
    # the panel row, and with a sketch its bucket-major copy
    return out.value / m + bpr * (2 if sketch else 1)


def max_records_for_budget(snps: BimTable, n_indiv: int, budget_bytes: int, **kw) -> int:
    """Largest call (in records) whose panel rows and workspace fit the budget."""
    per = call_bytes_per_record(snps, n_indiv, **kw)
    return max(1, int(budget_bytes // max(per, 1.0)))


def run_l2_sliced(ctx: Context, snps: BimTable, bed_body: np.ndarray, n_indiv: int, mode: WindowMode,
                  chunk_c: int = 200, max_call_records: Optional[int] = None,
                  device_budget_bytes: Optional[int] = None, annot=None, iid_indices=None, pq_exp=None,
                  sketch=None, sketch_maf_aware: bool = False, snp_level_masking: bool = False,
                  global_pass: bool = False, precision: str = "fp64", use_f32: bool = False,
                  on_slice=None) -> Tuple[np.ndarray, np.ndarray, List[Shard], List[L2Perf]]:
    """l2 (M x K) and MAF of `snps` computed slice by slice.  bed_body: the
    BED rows (file order, ceil(n_indiv / 4) bytes each; a memory map works),
    indexed by snps.bed_idx.  The slice size is max_call_records, or what
    device_budget_bytes allows.  Returns (l2, maf, slices, per-slice perf)."""
    m = len(snps)
    bpr = (n_indiv + 3) // 4
    body = np.asarray(bed_body, dtype=np.uint8).reshape(-1, bpr) if bpr else np.zeros((0, 0), np.uint8)
    bed_idx = np.asarray(snps.bed_idx, dtype=np.int64)
    if m and np.any(np.diff(bed_idx) <= 0):
        raise LdscError(L.LDSC_E_INVALID, "records must be in BED row order")
    if m and (bed_idx[0] < 0 or bed_idx[-1] >= body.shape[0]):
        raise LdscError(L.LDSC_E_INVALID, "SNP index out of range of the BED rows")
    kw = dict(mode=mode, chunk_c=chunk_c, precision=precision, sketch=sketch,
              snp_level_masking=snp_level_masking, global_pass=global_pass)
    if max_call_records is None:
        if device_budget_bytes is None:
            raise ValueError("give max_call_records or device_budget_bytes")
        max_call_records = max_records_for_budget(snps, n_indiv, device_budget_bytes, annot=annot,
                                                  iid_indices=iid_indices, **kw)
    slices = plan_slices(snps, mode, max_call_records, chunk_c, snp_level_masking, global_pass)
    ann = None
    if annot is not None:
        ann = np.asarray(annot, dtype=np.float64)
        ann = ann.reshape(-1, 1) if ann.ndim == 1 else ann
    K = 1 if ann is None else ann.shape[1]
    l2 = np.zeros((m, K), dtype=np.float64, order="F")
    maf = np.zeros(m, dtype=np.float64)
    perfs: List[L2Perf] = []
    for sl in slices:
        a, b = sl.call_lo, sl.call_hi
        r0, r1 = int(bed_idx[a]), int(bed_idx[b - 1]) + 1
        sub = snps.subset(np.arange(a, b))
        sub = BimTable(sub.chr, sub.snp, sub.cm, sub.bp, np.asarray(sub.bed_idx, dtype=np.int64) - r0)
        panel = ctx.upload(body[r0:r1], n_indiv)
        try:
            out, mf, pf = run_l2(ctx, sub, panel, mode, chunk_c, annot=None if ann is None else ann[a:b],
                                 iid_indices=iid_indices, pq_exp=pq_exp, yes_really=True, use_f32=use_f32,
                                 sketch=sketch, sketch_maf_aware=sketch_maf_aware,
                                 snp_level_masking=snp_level_masking, global_pass=global_pass,
                                 precision=precision)
        finally:
            panel.close()
        l2[sl.core_lo:sl.core_hi] = out[sl.core_lo - a: sl.core_hi - a]
        maf[sl.core_lo:sl.core_hi] = mf[sl.core_lo - a: sl.core_hi - a]
        perfs.append(pf)
        if on_slice is not None:
            on_slice(sl, pf)
    return l2, maf, slices, perfs
