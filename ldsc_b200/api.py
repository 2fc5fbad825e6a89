"""Python binding of the l2 engine, shaped like the reference's Rust API.

  * ``compute_ldscore_global`` -- src/l2/compute.rs:1009-1028 (one pass over
    the given SNP list, chunked from its first record);
  * ``run_l2`` -- the per-chromosome fan-out of ``l2::run``
    (src/l2/mod.rs:439-575), default mode of the CLI;
  * ``L2Config`` / ``compute_l2_from_bytes`` / ``L2Output`` -- the library API
    (src/l2/mod.rs:950-1169);
  * ``WindowMode`` -- src/l2/window.rs:5-12.
Errors raise ``LdscError`` carrying the engine's message (the reference
returns ``anyhow::Error``; malformed input never panics).
"""
from __future__ import annotations

import ctypes as C
import dataclasses
import time
from typing import Callable, Optional

import numpy as np

from . import _lib as L
from .plink import BimTable, count_fam_str, parse_bim_text


class LdscError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{L.STATUS_NAMES.get(code, code)}: {msg}")
        self.code = code
        self.msg = msg


@dataclasses.dataclass(frozen=True)
class WindowMode:
    kind: str     # "cm" | "kb" | "snp"
    value: float

    @staticmethod
    def Cm(x: float) -> "WindowMode":
        return WindowMode("cm", float(x))

    @staticmethod
    def Kb(x: float) -> "WindowMode":
        return WindowMode("kb", float(x))

    @staticmethod
    def Snp(n: int) -> "WindowMode":
        return WindowMode("snp", int(n))


@dataclasses.dataclass
class L2Perf:
    """L2Perf (src/l2/mod.rs:1016-1034) plus device detail."""
    m: int
    n_indiv: int
    bed_read_secs: float
    norm_secs: float
    sketch_secs: Optional[float]
    bb_dot_secs: float
    ab_dot_secs: float
    ring_store_secs: float
    n_pairs: int
    n_tiles: int
    kernel_launches: int
    gram_kind: str
    device_ms: float
    contract_secs: float = 0.0
    layout_secs: float = 0.0


def _perf(p: L.Perf) -> L2Perf:
    return L2Perf(int(p.m), int(p.n_indiv), p.bed_read_secs, p.norm_secs,
                  None if p.sketch_secs < 0 else p.sketch_secs, p.bb_dot_secs, p.ab_dot_secs,
                  p.ring_store_secs, int(p.n_pairs), int(p.n_tiles), int(p.kernel_launches),
                  {0: "fp64", 1: "int8", 2: "fp32-sketch"}.get(int(p.gram_kind), "?"),
                  p.device_ms, p.contract_secs, p.layout_secs)


class Context:
    """One engine context on a CUDA device (GpuContext, src/gpu.rs:92-130)."""

    def __init__(self, device: int = 0, fused_operands: bool = False):
        """fused_operands: run the INT8 form as the fused packed-row Gram
        (LDSC_CTX_FUSED_OPERANDS, no operand buffer) instead of decoding the
        operand rows into device memory first."""
        self.lib = L.load()
        h = C.c_void_p()
        flags = L.CTX_FUSED_OPERANDS if fused_operands else 0
        rc = self.lib.ldsc_ctx_create(int(device), flags, C.byref(h))
        if rc != L.LDSC_OK:
            raise LdscError(rc, f"could not create a context on CUDA device {device}")
        self.h = h

    def close(self):
        if self.h:
            self.lib.ldsc_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def error(self) -> str:
        buf = C.create_string_buffer(1024)
        self.lib.ldsc_last_error(self.h, buf, 1024)
        return buf.value.decode(errors="replace")

    def check(self, rc: int):
        if rc != L.LDSC_OK:
            raise LdscError(rc, self.error())

    def set_stream(self, stream_ptr: int | None):
        self.check(self.lib.ldsc_ctx_set_stream(self.h, C.c_void_p(stream_ptr or 0)))

    @property
    def kernel_count(self) -> int:
        return int(self.lib.ldsc_ctx_kernel_count(self.h))

    # ---- panels ----
    def upload(self, body: np.ndarray, n_indiv: int) -> "Panel":
        body = np.ascontiguousarray(body, dtype=np.uint8).reshape(-1)
        bpr = (n_indiv + 3) // 4
        n_snp = body.size // bpr if bpr else 0
        h = C.c_void_p()
        self.check(self.lib.ldsc_panel_upload(self.h, body.ctypes.data, body.size, n_indiv, n_snp,
                                              C.byref(h)))
        return Panel(self, h, n_indiv, n_snp)

    def upload_ptr(self, ptr: int, nbytes: int, n_indiv: int) -> "Panel":
        bpr = (n_indiv + 3) // 4
        n_snp = nbytes // bpr
        h = C.c_void_p()
        self.check(self.lib.ldsc_panel_upload(self.h, C.c_void_p(ptr), nbytes, n_indiv, n_snp,
                                              C.byref(h)))
        return Panel(self, h, n_indiv, n_snp)

    def synth(self, n_indiv: int, n_snp: int, founders: int, switch_p: float, miss: float,
              seed: int) -> "Panel":
        spec = L.SynthSpec(n_indiv, n_snp, founders, switch_p, miss, seed)
        h = C.c_void_p()
        self.check(self.lib.ldsc_panel_synth(self.h, C.byref(spec), C.byref(h)))
        return Panel(self, h, n_indiv, n_snp)


class Panel:
    """A BED panel resident in device memory."""

    def __init__(self, ctx: Context, h: C.c_void_p, n_indiv: int, n_snp: int):
        self.ctx, self.h, self.n_indiv, self.n_snp = ctx, h, n_indiv, n_snp

    @property
    def bpr(self) -> int:
        return (self.n_indiv + 3) // 4

    def download(self, begin: int = 0, end: Optional[int] = None) -> np.ndarray:
        end = self.n_snp if end is None else end
        out = np.zeros((end - begin, self.bpr), dtype=np.uint8)
        self.ctx.check(self.ctx.lib.ldsc_panel_download(self.ctx.h, self.h, begin, end,
                                                        out.ctypes.data))
        return out

    def close(self):
        if self.h:
            self.ctx.lib.ldsc_panel_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


_MODE = {"cm": L.WINDOW_CM, "kb": L.WINDOW_KB, "snp": L.WINDOW_SNP}


class _ArgPack:
    """Keeps the numpy buffers behind an L2Args alive."""

    def __init__(self, snps: BimTable, mode: WindowMode, chunk_c: int, annot, iid_indices, pq_exp,
                 yes_really, use_f32, sketch, sketch_maf_aware, snp_level_masking, precision,
                 global_pass, on_progress, records_are_rows: bool = False, row_begin: int = 0,
                 annot_device=None):
        m = len(snps)
        self.chr = np.ascontiguousarray(snps.chr, dtype=np.uint8)
        self.cm = np.ascontiguousarray(snps.cm, dtype=np.float64)
        self.bp = np.ascontiguousarray(snps.bp, dtype=np.uint32)
        self.bed_idx = None if records_are_rows else np.ascontiguousarray(snps.bed_idx, dtype=np.uint64)
        self.keep = None if iid_indices is None else np.ascontiguousarray(iid_indices, dtype=np.int64)
        self.annot = None
        K = 1
        if annot is not None:
            a = np.asarray(annot, dtype=np.float64)
            if a.ndim == 1:
                a = a.reshape(-1, 1)
            if a.shape[0] != m:
                raise LdscError(L.LDSC_E_INVALID,
                                f"Annotation matrix has {a.shape[0]} rows but BIM has {m} SNPs")
            self.annot = np.asfortranarray(a)
            K = a.shape[1]
        annot_ptr, annot_ld = (None if self.annot is None else self.annot.ctypes.data), 0
        if annot_device is not None:
            # (device pointer, leading dimension in rows, K) of a resident annotation matrix
            annot_ptr, annot_ld, K = int(annot_device[0]), int(annot_device[1]), int(annot_device[2])
        self.K = K
        self.cb = PROGRESS_NONE
        if on_progress is not None:
            def _cb(p, _u):
                c = p.contents
                on_progress(dict(chunks_done=c.chunks_done, chunks_total=c.chunks_total,
                                 snps_done=c.snps_done, snps_total=c.snps_total,
                                 chunk_wall_ms=c.chunk_wall_ms))
            self.cb = L.PROGRESS_FN(_cb)
        prec = {"fp64": L.PRECISION_FP64, "int8": L.PRECISION_INT8}[precision]
        self.args = L.L2Args(
            n_snp=m, bed_idx=None if self.bed_idx is None else self.bed_idx.ctypes.data,
            chr=self.chr.ctypes.data, cm=self.cm.ctypes.data, bp=self.bp.ctypes.data,
            window_mode=_MODE[mode.kind], window_size=float(mode.value) if mode.kind != "snp" else 0.0,
            window_snps=int(mode.value) if mode.kind == "snp" else 0, chunk_size=int(chunk_c),
            global_pass=int(bool(global_pass)), snp_level_masking=int(bool(snp_level_masking)),
            precision=prec, use_f32=int(bool(use_f32)), sketch_d=int(sketch or 0),
            sketch_maf_aware=int(bool(sketch_maf_aware)),
            keep_iids=None if self.keep is None else self.keep.ctypes.data,
            n_keep=0 if self.keep is None else len(self.keep),
            annot=annot_ptr, n_annot=K,
            has_pq_exp=int(pq_exp is not None), pq_exp=float(pq_exp or 0.0),
            yes_really=int(bool(yes_really)), on_progress=self.cb, progress_user=None,
            row_begin=int(row_begin), annot_on_device=int(annot_device is not None), annot_ld=annot_ld)


PROGRESS_NONE = L.PROGRESS_FN()


def _run(ctx: Context, panel: Panel, pack: _ArgPack, m: int, out_device=None):
    if out_device is not None:
        # (l2, maf) CUDA tensors: l2 of shape (K, m) row-major = m x K column-major; maf (m,)
        l2, maf = out_device
        if tuple(l2.shape) != (pack.K, m) or tuple(maf.shape) != (m,) or not l2.is_contiguous():
            raise LdscError(L.LDSC_E_INVALID, "out_device wants contiguous (K, m) and (m,) float64 tensors")
        pack.args.out_on_device = 1
        perf = L.Perf()
        ctx.check(ctx.lib.ldsc_l2_run(ctx.h, panel.h, C.byref(pack.args), l2.data_ptr(), maf.data_ptr(),
                                      C.byref(perf)))
        return l2, maf, _perf(perf)
    l2 = np.zeros((m, pack.K), dtype=np.float64, order="F")
    maf = np.zeros(m, dtype=np.float64)
    perf = L.Perf()
    ctx.check(ctx.lib.ldsc_l2_run(ctx.h, panel.h, C.byref(pack.args), l2.ctypes.data,
                                  maf.ctypes.data, C.byref(perf)))
    return l2, maf, _perf(perf)


def compute_ldscore_global(ctx: Context, all_snps: BimTable, panel: Panel, n_indiv: int,
                           mode: WindowMode, chunk_c: int, annot=None, iid_indices=None,
                           pq_exp: Optional[float] = None, yes_really: bool = False,
                           use_f32: bool = False, verbose_timing: bool = False,
                           sketch: Optional[int] = None, sketch_maf_aware: bool = False,
                           snp_level_masking: bool = False,
                           on_progress: Optional[Callable] = None, precision: str = "fp64"):
    """compute_ldscore_global (src/l2/compute.rs:1009-1028): one chunked pass
    over ``all_snps``; returns (l2 M x K, maf, L2Perf)."""
    if panel.n_indiv != n_indiv:
        raise LdscError(L.LDSC_E_INVALID, "n_indiv does not match the panel")
    pack = _ArgPack(all_snps, mode, chunk_c, annot, iid_indices, pq_exp, yes_really, use_f32,
                    sketch, sketch_maf_aware, snp_level_masking, precision, True, on_progress)
    l2, maf, perf = _run(ctx, panel, pack, len(all_snps))
    if verbose_timing:
        _print_perf(perf)
    return l2, maf, perf


def run_l2(ctx: Context, all_snps: BimTable, panel: Panel, mode: WindowMode, chunk_c: int = 200,
           annot=None, iid_indices=None, pq_exp=None, yes_really=False, use_f32=False,
           sketch=None, sketch_maf_aware=False, snp_level_masking=False, global_pass=False,
           precision="fp64", on_progress=None, annot_device=None, out_device=None):
    """The compute part of ``l2::run``: per-chromosome chunking (default) or
    one global pass (src/l2/mod.rs:439-575).  ``annot_device`` = (device
    pointer, leading dimension, K) of resident annotations; ``out_device`` =
    (l2, maf) CUDA tensors that receive the results in place of host arrays."""
    pack = _ArgPack(all_snps, mode, chunk_c, annot, iid_indices, pq_exp, yes_really, use_f32,
                    sketch, sketch_maf_aware, snp_level_masking, precision, global_pass,
                    on_progress, annot_device=annot_device)
    return _run(ctx, panel, pack, len(all_snps), out_device)


def l2_from_bed_bytes(ctx: Context, bed_file: np.ndarray, n_indiv: int, snps: BimTable,
                      mode: WindowMode, chunk_c: int = 200, precision: str = "fp64",
                      snp_level_masking: bool = False, global_pass: bool = False, sketch=None,
                      annot=None, iid_indices=None, pq_exp=None, yes_really=True):
    """Whole-file entry (validate + upload + compute + download) through
    ``ldsc_l2_from_bed``.  ``bed_file`` includes the 3 magic bytes and may be
    a pinned host buffer."""
    bed_file = np.ascontiguousarray(bed_file, dtype=np.uint8).reshape(-1)
    pack = _ArgPack(snps, mode, chunk_c, annot, iid_indices, pq_exp, yes_really, False, sketch,
                    False, snp_level_masking, precision, global_pass, None)
    m = len(snps)
    l2 = np.zeros((m, pack.K), dtype=np.float64, order="F")
    maf = np.zeros(m, dtype=np.float64)
    perf = L.Perf()
    ctx.check(ctx.lib.ldsc_l2_from_bed(ctx.h, bed_file.ctypes.data, bed_file.size, n_indiv,
                                       C.byref(pack.args), l2.ctypes.data, maf.ctypes.data,
                                       C.byref(perf)))
    return l2, maf, _perf(perf)


def pair_count(snps: BimTable, mode: WindowMode, chunk_c: int = 200, snp_level_masking=False,
               global_pass=False) -> int:
    """Off-diagonal pairs a run accumulates (the r^2-pairs/sec numerator)."""
    lib = L.load()
    pack = _ArgPack(snps, mode, chunk_c, None, None, None, True, False, None, False,
                    snp_level_masking, "fp64", global_pass, None)
    out = C.c_uint64()
    rc = lib.ldsc_l2_pair_count(C.byref(pack.args), C.byref(out))
    if rc != L.LDSC_OK:
        raise LdscError(rc, "pair count failed")
    return int(out.value)


def left_limits(snps: BimTable, mode: WindowMode, chunk_c: int = 200, snp_level_masking=False,
                global_pass=False) -> np.ndarray:
    lib = L.load()
    pack = _ArgPack(snps, mode, chunk_c, None, None, None, True, False, None, False,
                    snp_level_masking, "fp64", global_pass, None)
    out = np.zeros(len(snps), dtype=np.int64)
    rc = lib.ldsc_l2_left_limits(C.byref(pack.args), out.ctypes.data)
    if rc != L.LDSC_OK:
        raise LdscError(rc, "invalid window arguments")
    return out


def bed_validate(bed_file: bytes | np.ndarray, n_indiv: int, n_snp: int) -> None:
    """Bed::from_bytes validation (src/bed.rs:73-110); raises LdscError."""
    lib = L.load()
    buf = np.frombuffer(bytes(bed_file), dtype=np.uint8) if not isinstance(bed_file, np.ndarray) \
        else np.ascontiguousarray(bed_file, dtype=np.uint8)
    err = C.create_string_buffer(256)
    rc = lib.ldsc_bed_validate(buf.ctypes.data if buf.size else None, buf.size, n_indiv, n_snp,
                               err, 256)
    if rc != L.LDSC_OK:
        raise LdscError(rc, err.value.decode())


def countsketch_hash(n_indiv: int, d: int, seed: int = 42):
    lib = L.load()
    bucket = np.zeros(n_indiv, dtype=np.uint32)
    sign = np.zeros(n_indiv, dtype=np.float32)
    rc = lib.ldsc_countsketch_hash(n_indiv, d, seed, bucket.ctypes.data, sign.ctypes.data)
    if rc != L.LDSC_OK:
        raise LdscError(rc, "countsketch_hash")
    return bucket, sign


def sketch_project(ctx: Context, panel: Panel, begin: int, end: int, bucket, sign, d: int,
                   keep=None) -> np.ndarray:
    bucket = np.ascontiguousarray(bucket, dtype=np.uint32)
    sign = np.ascontiguousarray(sign, dtype=np.float32)
    keep_arr = None if keep is None else np.ascontiguousarray(keep, dtype=np.int64)
    out = np.zeros((end - begin, d), dtype=np.float32)
    ctx.check(ctx.lib.ldsc_sketch_project(
        ctx.h, panel.h, begin, end, None if keep_arr is None else keep_arr.ctypes.data,
        0 if keep_arr is None else len(keep_arr), bucket.ctypes.data, sign.ctypes.data, d,
        out.ctypes.data))
    return out


def debug_gram_i8_tile(ctx: Context, panel: Panel, k0: int, j0: int) -> np.ndarray:
    out = np.zeros((128, 256), dtype=np.int32)
    ctx.check(ctx.lib.ldsc_debug_gram_i8_tile(ctx.h, panel.h, k0, j0, out.ctypes.data))
    return out


def _print_perf(p: L2Perf):
    if p.sketch_secs is not None:
        print(f"[perf] compute_ldscore: bed_read(stall)={p.bed_read_secs:.3f}s norm={p.norm_secs:.3f}s "
              f"sketch={p.sketch_secs:.3f}s bb_dot={p.bb_dot_secs:.3f}s ab_dot={p.ab_dot_secs:.3f}s "
              f"ring_store={p.ring_store_secs:.3f}s")
    else:
        print(f"[perf] compute_ldscore: bed_read(stall)={p.bed_read_secs:.3f}s norm={p.norm_secs:.3f}s "
              f"bb_dot={p.bb_dot_secs:.3f}s ab_dot={p.ab_dot_secs:.3f}s "
              f"ring_store={p.ring_store_secs:.3f}s")


# ---- library API (src/l2/mod.rs:950-1169) ----

@dataclasses.dataclass
class L2Config:
    mode: WindowMode = dataclasses.field(default_factory=lambda: WindowMode.Kb(1000.0))
    chunk_size: int = 200
    use_f32: bool = False
    sketch: Optional[int] = None
    sketch_maf_aware: bool = False
    snp_level_masking: bool = False
    yes_really: bool = True
    pq_exp: Optional[float] = None
    verbose_timing: bool = False
    precision: str = "fp64"


@dataclasses.dataclass
class L2Output:
    snps: BimTable
    l2: np.ndarray
    maf: np.ndarray
    wall_seconds: float
    perf: L2Perf


def compute_l2_from_bytes(bed_bytes: bytes, bim_text: str, fam_text: str, config: L2Config,
                          ctx: Optional[Context] = None, on_progress=None) -> L2Output:
    """compute_l2_from_bytes (src/l2/mod.rs:1049-1092): K = 1, no keep/annot."""
    snps = parse_bim_text(bim_text)
    if len(snps) == 0:
        raise LdscError(L.LDSC_E_INVALID, "compute_l2_from_bytes: BIM has zero SNPs")
    n_indiv = count_fam_str(fam_text)
    if n_indiv == 0:
        raise LdscError(L.LDSC_E_INVALID, "compute_l2_from_bytes: FAM has zero individuals")
    bed_validate(bed_bytes, n_indiv, len(snps))
    own = ctx is None
    ctx = ctx or Context(0)
    try:
        t0 = time.time()
        buf = np.frombuffer(bytes(bed_bytes), dtype=np.uint8)
        pack = _ArgPack(snps, config.mode, config.chunk_size, None, None, config.pq_exp,
                        config.yes_really, config.use_f32, config.sketch, config.sketch_maf_aware,
                        config.snp_level_masking, config.precision, True, on_progress)
        m = len(snps)
        l2 = np.zeros((m, 1), dtype=np.float64, order="F")
        maf = np.zeros(m, dtype=np.float64)
        perf = L.Perf()
        ctx.check(ctx.lib.ldsc_l2_from_bed(ctx.h, buf.ctypes.data, buf.size, n_indiv,
                                           C.byref(pack.args), l2.ctypes.data, maf.ctypes.data,
                                           C.byref(perf)))
        p = _perf(perf)
        if config.verbose_timing:
            _print_perf(p)
        return L2Output(snps, l2[:, 0].copy(), maf, time.time() - t0, p)
    finally:
        if own:
            ctx.close()


# ---- regressions (src/h2.rs, src/regressions.rs) ----

def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def h2_batch(ctx: Context, chi2, n, ref_l2, w_l2, m_snps: float, n_blocks: int = 200,
             intercept: Optional[float] = None, lambda_gc: bool = True,
             two_step: Optional[float] = None) -> np.ndarray:
    """run_h2_ldsc for many traits (K = 1, no --two-step).  chi2: T x n_snp;
    n: T scalars or T x n_snp.  Returns a structured array with the fields of
    ldsc_h2_result."""
    chi2 = _f64(np.atleast_2d(chi2))
    T, m = chi2.shape
    n = _f64(n)
    per_snp = n.ndim == 2
    ref_l2, w_l2 = _f64(ref_l2), _f64(w_l2)
    args = L.H2Args(n_snp=m, n_traits=T, n_blocks=n_blocks, chi2=chi2.ctypes.data,
                    n_per_snp=n.ctypes.data if per_snp else None,
                    n_scalar=None if per_snp else n.ctypes.data,
                    ref_l2=ref_l2.ctypes.data, w_l2=w_l2.ctypes.data, m_snps=float(m_snps),
                    fixed_intercept=int(intercept is not None), intercept=float(intercept or 0.0),
                    want_lambda_gc=int(lambda_gc), device_pointers=0, two_step=int(two_step is not None),
                    two_step_cutoff=float(two_step or 0.0))
    out = (L.H2Result * T)()
    ctx.check(ctx.lib.ldsc_h2_batch(ctx.h, C.byref(args), C.cast(out, C.c_void_p)))
    names = [f for f, _ in L.H2Result._fields_]
    return np.array([tuple(getattr(r, f) for f in names) for r in out],
                    dtype=[(f, np.float64) for f in names])


def rg_batch(ctx: Context, z1, z2, n1, n2, ref_l2, w_l2, m_snps: float,
             n_blocks: int = 200) -> np.ndarray:
    """run_rg for many trait pairs (free intercepts, no --two-step)."""
    z1, z2 = _f64(np.atleast_2d(z1)), _f64(np.atleast_2d(z2))
    P, m = z1.shape
    n1, n2 = _f64(np.broadcast_to(n1, (P,))), _f64(np.broadcast_to(n2, (P,)))
    ref_l2, w_l2 = _f64(ref_l2), _f64(w_l2)
    args = L.RgArgs(n_snp=m, n_pairs=P, n_blocks=n_blocks, z1=z1.ctypes.data, z2=z2.ctypes.data,
                    n1=n1.ctypes.data, n2=n2.ctypes.data, ref_l2=ref_l2.ctypes.data,
                    w_l2=w_l2.ctypes.data, m_snps=float(m_snps), device_pointers=0)
    out = (L.RgResult * P)()
    ctx.check(ctx.lib.ldsc_rg_batch(ctx.h, C.byref(args), C.cast(out, C.c_void_p)))
    names = [f for f, _ in L.RgResult._fields_]
    return np.array([tuple(getattr(r, f) for f in names) for r in out],
                    dtype=[(f, np.float64) for f in names])


def snp_stats(ctx: Context, snps: BimTable, panel: Panel, iid_indices=None):
    """compute_snp_stats (src/l2/snp_stats.rs:5-195): (MAF, het_miss_ok) per
    record, the --maf / --pq-exp prefilter."""
    pack = _ArgPack(snps, WindowMode.Cm(1.0), 200, None, iid_indices, None, True, False, None, False,
                    False, "fp64", False, None)
    m = len(snps)
    maf = np.zeros(m, dtype=np.float64)
    ok = np.zeros(m, dtype=np.uint8)
    ctx.check(ctx.lib.ldsc_snp_stats(ctx.h, panel.h, C.byref(pack.args), maf.ctypes.data, ok.ctypes.data))
    return maf, ok.astype(bool)
