"""Continuous-batching server over resident panels (``ldsc_server_*``).

The reference runs one computation per process; the server keeps panels,
LD scores and summary statistics resident on the device and runs l2, h2 and
rg jobs of uneven size concurrently, one per slot, admitting queued jobs as
slots and device memory free up.  Submission returns a ticket at once;
``wait`` blocks (without the GIL) until that job ends.
"""
from __future__ import annotations

import ctypes as C
import dataclasses
import threading
from typing import Optional

import numpy as np

from . import _lib as L
from .api import LdscError, Panel, WindowMode, _ArgPack, _f64, _perf
from .plink import BimTable


def _is_device(x) -> bool:
    return hasattr(x, "is_cuda") and bool(x.is_cuda)


def _ptr(x):
    """(pointer, keep-alive) of a float64 host array or a CUDA tensor."""
    if _is_device(x):
        return x.data_ptr(), x
    a = _f64(x)
    return a.ctypes.data, a


@dataclasses.dataclass
class JobTiming:
    slot: int
    queue_ms: float
    run_ms: float
    latency_ms: float


class Server:
    def __init__(self, device: int = 0, n_slots: int = 4, budget_bytes: int = 0):
        self.lib = L.load()
        h = C.c_void_p()
        rc = self.lib.ldsc_server_create(int(device), int(n_slots), int(budget_bytes), C.byref(h))
        if rc != L.LDSC_OK:
            raise LdscError(rc, "could not create the server")
        self.h = h
        self._live = {}
        self._mu = threading.Lock()

    def close(self):
        if self.h:
            self.lib.ldsc_server_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def prewarm(self, submit_fn, *args, **kw) -> None:
        """Run one job on every slot, one after another (ldsc_server_prewarm):
        ``srv.prewarm(srv.submit_l2, panel, snps, mode, ...)``.  Each slot's
        workspace is then sized for that job, so later jobs no larger than it
        allocate no device memory while others run."""
        self._warm = True
        try:
            submit_fn(*args, **kw)
        finally:
            self._warm = False

    def _submit(self, job: L.Job, keep: dict) -> int:
        if getattr(self, "_warm", False):
            rc = self.lib.ldsc_server_prewarm(self.h, C.byref(job))
            if rc != L.LDSC_OK:
                raise LdscError(rc, "prewarm job failed")
            return 0
        t = C.c_uint64()
        rc = self.lib.ldsc_server_submit(self.h, C.byref(job), C.byref(t))
        if rc != L.LDSC_OK:
            raise LdscError(rc, "job rejected (workspace above the device budget)" if rc == L.LDSC_E_NOMEM
                            else "job rejected")
        with self._mu:
            self._live[t.value] = (job, keep)
        return t.value

    # ---- job kinds ----
    def submit_l2(self, panel: Panel, snps: BimTable, mode: WindowMode, chunk_c: int = 200, *,
                  row_begin: Optional[int] = None, annot=None, annot_device=None, sketch=None,
                  precision: str = "int8", snp_level_masking: bool = False, global_pass: bool = False,
                  iid_indices=None, pq_exp=None) -> int:
        """l2 over ``snps``.  With ``row_begin`` the records are panel rows
        row_begin .. row_begin+len(snps)-1 (no per-record row array).
        ``annot_device`` = (device pointer, leading dimension, K) of a
        resident annotation matrix whose row 0 is the first record."""
        pack = _ArgPack(snps, mode, chunk_c, annot, iid_indices, pq_exp, True, False, sketch, False,
                        snp_level_masking, precision, global_pass, None, records_are_rows=row_begin is not None,
                        row_begin=row_begin or 0, annot_device=annot_device)
        m = len(snps)
        l2 = np.zeros((m, pack.K), dtype=np.float64, order="F")
        maf = np.zeros(m, dtype=np.float64)
        job = L.Job(kind=L.JOB_L2, panel=panel.h, l2=pack.args, l2_out=l2.ctypes.data, maf_out=maf.ctypes.data)
        return self._submit(job, dict(pack=pack, l2=l2, maf=maf, panel=panel, kind="l2"))

    def submit_h2(self, chi2, n, ref_l2, w_l2, m_snps: float, n_blocks: int = 200,
                  intercept: Optional[float] = None, lambda_gc: bool = True) -> int:
        """h2 for T traits.  All arrays on the host (numpy), or all CUDA
        tensors (chi2 T x n row-major, n: T scalars, ref_l2 / w_l2: n)."""
        dev = _is_device(chi2)
        T, m = (chi2.shape if chi2.ndim == 2 else (1, chi2.shape[0]))
        pc, kc = _ptr(chi2)
        pn, kn = _ptr(n if dev else np.broadcast_to(np.asarray(n, float), (T,)))
        pl, kl = _ptr(ref_l2)
        pw, kw = _ptr(w_l2)
        args = L.H2Args(n_snp=m, n_traits=T, n_blocks=n_blocks, chi2=pc, n_per_snp=None, n_scalar=pn,
                        ref_l2=pl, w_l2=pw, m_snps=float(m_snps), fixed_intercept=int(intercept is not None),
                        intercept=float(intercept or 0.0), want_lambda_gc=int(lambda_gc), device_pointers=int(dev))
        out = (L.H2Result * T)()
        job = L.Job(kind=L.JOB_H2, h2=args, h2_out=C.cast(out, C.c_void_p))
        return self._submit(job, dict(keep=(kc, kn, kl, kw), out=out, kind="h2"))

    def submit_rg(self, z1, z2, n1, n2, ref_l2, w_l2, m_snps: float, n_blocks: int = 200) -> int:
        """rg for P trait pairs (z1, z2: P x n; n1, n2: P scalars); host
        arrays or all CUDA tensors."""
        dev = _is_device(z1)
        P, m = (z1.shape if z1.ndim == 2 else (1, z1.shape[0]))
        p1, k1 = _ptr(z1)
        p2, k2 = _ptr(z2)
        pn1, kn1 = _ptr(n1 if dev else np.broadcast_to(np.asarray(n1, float), (P,)))
        pn2, kn2 = _ptr(n2 if dev else np.broadcast_to(np.asarray(n2, float), (P,)))
        pl, kl = _ptr(ref_l2)
        pw, kw = _ptr(w_l2)
        args = L.RgArgs(n_snp=m, n_pairs=P, n_blocks=n_blocks, z1=p1, z2=p2, n1=pn1, n2=pn2, ref_l2=pl,
                        w_l2=pw, m_snps=float(m_snps), device_pointers=int(dev))
        out = (L.RgResult * P)()
        job = L.Job(kind=L.JOB_RG, rg=args, rg_out=C.cast(out, C.c_void_p))
        return self._submit(job, dict(keep=(k1, k2, kn1, kn2, kl, kw), out=out, kind="rg"))

    def submit_h2_partitioned(self, chi2, n, ref_l2, w_l2, m_vec, chisq_max, n_blocks: int = 200,
                              intercept: Optional[float] = None) -> int:
        """Partitioned h2 for T traits on CUDA tensors: chi2 (T, n_snp), n
        (T,) sample sizes, ref_l2 (K, n_snp) (the l2 run's device layout),
        w_l2 (n_snp,); m_vec K values, chisq_max T cut-offs (host).  wait()
        returns a list of PartitionedFit."""
        T, m = int(chi2.shape[0]), int(chi2.shape[1])
        K = int(ref_l2.shape[0])
        fixed = intercept is not None
        P = K + (0 if fixed else 1)
        mv = np.ascontiguousarray(m_vec, dtype=np.float64)
        cm = np.ascontiguousarray(np.broadcast_to(np.asarray(chisq_max, float), (T,)))
        est, cov = np.zeros((T, P)), np.zeros((T, P, P))
        dv, h2a = np.zeros((T, n_blocks, P)), np.zeros((T, K))
        args = L.H2PArgs(n_snp=m, n_traits=T, n_annot=K, n_blocks=n_blocks, chi2=chi2.data_ptr(), n_per_snp=None,
                         n_scalar=n.data_ptr(), ref_l2=ref_l2.data_ptr(), ref_ld=m, w_l2=w_l2.data_ptr(),
                         m_vec=mv.ctypes.data, fixed_intercept=int(fixed), intercept=float(intercept or 0.0),
                         chisq_max=cm.ctypes.data, device_pointers=1, est=est.ctypes.data, cov=cov.ctypes.data,
                         delete_values=dv.ctypes.data, h2_annot=h2a.ctypes.data)
        out = (L.H2PResult * T)()
        job = L.Job(kind=L.JOB_H2P, h2p=args, h2p_out=C.cast(out, C.c_void_p))
        return self._submit(job, dict(keep=(chi2, n, ref_l2, w_l2, mv, cm), out=out, kind="h2p",
                                      arrays=(est, cov, dv, h2a, mv)))

    def wait(self, ticket: int):
        """Block until the job ends.  Returns (result, JobTiming) where
        result is (l2, maf, L2Perf) for l2 jobs and a structured array for
        h2 / rg jobs; raises LdscError if the job failed."""
        res = L.JobResult()
        rc = self.lib.ldsc_server_wait(self.h, int(ticket), C.byref(res))
        with self._mu:
            job, keep = self._live.pop(int(ticket), (None, None))
        if rc != L.LDSC_OK:
            raise LdscError(rc, res.error.decode(errors="replace"))
        timing = JobTiming(int(res.slot), res.queue_ms, res.run_ms, res.latency_ms)
        kind = keep["kind"]
        if kind == "l2":
            return (keep["l2"], keep["maf"], _perf(res.perf)), timing
        if kind == "h2p":
            from .partitioned import PartitionedFit
            est, cov, dv, h2a, mv = keep["arrays"]
            fits = []
            for t, r in enumerate(keep["out"]):
                nb = int(r.n_blocks)
                fits.append(PartitionedFit(est=est[t], cov=cov[t], delete_values=dv[t, :nb], m_vec=mv.copy(),
                                           n_mean=r.n_mean, h2_annot=h2a[t], h2_total=r.h2_total,
                                           h2_total_se=r.h2_total_se, intercept=r.intercept,
                                           intercept_se=r.intercept_se, mean_chi2=r.mean_chi2,
                                           n_obs=int(r.n_obs), n_blocks=nb))
            return fits, timing
        struct = L.H2Result if kind == "h2" else L.RgResult
        names = [f for f, _ in struct._fields_]
        out = np.array([tuple(getattr(r, f) for f in names) for r in keep["out"]],
                       dtype=[(f, np.float64) for f in names])
        return out, timing

    def stats(self) -> dict:
        st = L.ServerStats()
        self.lib.ldsc_server_stats_get(self.h, C.byref(st))
        return {f: int(getattr(st, f)) for f, _ in L.ServerStats._fields_}
