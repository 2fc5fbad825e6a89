"""ctypes declarations of the C ABI in include/ldsc_b200.h.

The shared library is built in-tree (``python -m ldsc_b200.build``).  There is
no fallback: if ``libldsc_b200.so`` is missing, importing the compute API
raises, and every compute call fails on a machine without a B200.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libldsc_b200.so")

LDSC_OK = 0
LDSC_E_INVALID = -1
LDSC_E_NOMEM = -2
LDSC_E_CUDA = -3
LDSC_E_TIMEOUT = -4
LDSC_E_UNSUPPORTED = -5
LDSC_E_BED = -6

STATUS_NAMES = {
    LDSC_E_INVALID: "invalid argument",
    LDSC_E_NOMEM: "out of device memory",
    LDSC_E_CUDA: "CUDA error",
    LDSC_E_TIMEOUT: "device wait timed out",
    LDSC_E_UNSUPPORTED: "unsupported",
    LDSC_E_BED: "invalid BED",
}

WINDOW_CM, WINDOW_KB, WINDOW_SNP = 0, 1, 2
PRECISION_FP64, PRECISION_INT8 = 0, 1
CTX_FUSED_OPERANDS = 1   # context flag: fused INT8 Gram over the packed rows (no operand buffer)


class Progress(C.Structure):
    _fields_ = [("chunks_done", C.c_uint64), ("chunks_total", C.c_uint64),
                ("snps_done", C.c_uint64), ("snps_total", C.c_uint64),
                ("chunk_wall_ms", C.c_double)]


PROGRESS_FN = C.CFUNCTYPE(None, C.POINTER(Progress), C.c_void_p)


class Perf(C.Structure):
    _fields_ = [("m", C.c_uint64), ("n_indiv", C.c_uint64), ("bed_read_secs", C.c_double),
                ("norm_secs", C.c_double), ("sketch_secs", C.c_double),
                ("bb_dot_secs", C.c_double), ("ab_dot_secs", C.c_double),
                ("ring_store_secs", C.c_double), ("n_pairs", C.c_uint64),
                ("n_tiles", C.c_uint64), ("kernel_launches", C.c_uint32),
                ("gram_kind", C.c_uint32), ("device_ms", C.c_double), ("contract_secs", C.c_double),
                ("layout_secs", C.c_double)]


class L2Args(C.Structure):
    _fields_ = [
        ("n_snp", C.c_uint64), ("bed_idx", C.c_void_p), ("chr", C.c_void_p), ("cm", C.c_void_p),
        ("bp", C.c_void_p), ("window_mode", C.c_int32), ("window_size", C.c_double),
        ("window_snps", C.c_uint64), ("chunk_size", C.c_uint32), ("global_pass", C.c_int32),
        ("snp_level_masking", C.c_int32), ("precision", C.c_int32), ("use_f32", C.c_int32),
        ("sketch_d", C.c_uint32), ("sketch_maf_aware", C.c_int32), ("keep_iids", C.c_void_p),
        ("n_keep", C.c_uint64), ("annot", C.c_void_p), ("n_annot", C.c_uint32),
        ("has_pq_exp", C.c_int32), ("pq_exp", C.c_double), ("yes_really", C.c_int32),
        ("on_progress", PROGRESS_FN), ("progress_user", C.c_void_p),
        ("row_begin", C.c_uint64), ("annot_on_device", C.c_int32), ("annot_ld", C.c_uint64),
        ("out_on_device", C.c_int32),
    ]


class SynthSpec(C.Structure):
    _fields_ = [("n_indiv", C.c_uint64), ("n_snp", C.c_uint64), ("founders", C.c_uint32),
                ("switch_p", C.c_double), ("miss", C.c_double), ("seed", C.c_uint64)]


class H2Args(C.Structure):
    _fields_ = [("n_snp", C.c_uint64), ("n_traits", C.c_uint32), ("n_blocks", C.c_uint32),
                ("chi2", C.c_void_p), ("n_per_snp", C.c_void_p), ("n_scalar", C.c_void_p),
                ("ref_l2", C.c_void_p), ("w_l2", C.c_void_p), ("m_snps", C.c_double),
                ("fixed_intercept", C.c_int32), ("intercept", C.c_double),
                ("want_lambda_gc", C.c_int32), ("device_pointers", C.c_int32), ("two_step", C.c_int32),
                ("two_step_cutoff", C.c_double)]


class H2Result(C.Structure):
    _fields_ = [(f, C.c_double) for f in ("h2", "h2_se", "intercept", "intercept_se", "mean_chi2",
                                          "lambda_gc", "ratio", "ratio_se", "coef", "coef_se")]


class H2PArgs(C.Structure):
    _fields_ = [("n_snp", C.c_uint64), ("n_traits", C.c_uint32), ("n_annot", C.c_uint32),
                ("n_blocks", C.c_uint32), ("chi2", C.c_void_p), ("n_per_snp", C.c_void_p),
                ("n_scalar", C.c_void_p), ("ref_l2", C.c_void_p), ("ref_ld", C.c_uint64),
                ("w_l2", C.c_void_p), ("m_vec", C.c_void_p), ("fixed_intercept", C.c_int32),
                ("intercept", C.c_double), ("chisq_max", C.c_void_p), ("device_pointers", C.c_int32),
                ("est", C.c_void_p), ("cov", C.c_void_p), ("delete_values", C.c_void_p),
                ("h2_annot", C.c_void_p)]


class H2PResult(C.Structure):
    _fields_ = [(f, C.c_double) for f in ("h2_total", "h2_total_se", "intercept", "intercept_se",
                                          "n_mean", "mean_chi2")] + \
               [("n_obs", C.c_uint64), ("n_blocks", C.c_uint32)]


class RgArgs(C.Structure):
    _fields_ = [("n_snp", C.c_uint64), ("n_pairs", C.c_uint32), ("n_blocks", C.c_uint32),
                ("z1", C.c_void_p), ("z2", C.c_void_p), ("n1", C.c_void_p), ("n2", C.c_void_p),
                ("ref_l2", C.c_void_p), ("w_l2", C.c_void_p), ("m_snps", C.c_double),
                ("device_pointers", C.c_int32)]


class RgResult(C.Structure):
    _fields_ = [(f, C.c_double) for f in ("rg", "rg_se", "z", "p", "gencov", "gencov_se",
                                          "gencov_intercept", "gencov_intercept_se", "h2_1",
                                          "h2_1_se", "h2_2", "h2_2_se", "mean_z1z2")]


JOB_L2, JOB_H2, JOB_RG, JOB_H2P = 0, 1, 2, 3


class Job(C.Structure):
    _fields_ = [("kind", C.c_int32), ("panel", C.c_void_p), ("l2", L2Args), ("l2_out", C.c_void_p),
                ("maf_out", C.c_void_p), ("h2", H2Args), ("h2_out", C.c_void_p), ("rg", RgArgs),
                ("rg_out", C.c_void_p), ("device_bytes", C.c_uint64), ("h2p", H2PArgs),
                ("h2p_out", C.c_void_p)]


class JobResult(C.Structure):
    _fields_ = [("status", C.c_int32), ("slot", C.c_uint32), ("queue_ms", C.c_double),
                ("run_ms", C.c_double), ("latency_ms", C.c_double), ("perf", Perf),
                ("error", C.c_char * 256)]


class ServerStats(C.Structure):
    _fields_ = [(f, C.c_uint64) for f in ("submitted", "completed", "running", "queued", "budget_bytes",
                                          "reserved_bytes", "graph_launches", "kernels")]


# name -> (restype, argtypes)
SIGNATURES = {
    "ldsc_abi_version": (C.c_int, []),
    "ldsc_ctx_create": (C.c_int, [C.c_int, C.c_uint32, C.POINTER(C.c_void_p)]),
    "ldsc_ctx_destroy": (C.c_int, [C.c_void_p]),
    "ldsc_ctx_set_stream": (C.c_int, [C.c_void_p, C.c_void_p]),
    "ldsc_last_error": (C.c_int, [C.c_void_p, C.c_char_p, C.c_size_t]),
    "ldsc_ctx_kernel_count": (C.c_uint64, [C.c_void_p]),
    "ldsc_bed_validate": (C.c_int, [C.c_void_p, C.c_uint64, C.c_uint64, C.c_uint64, C.c_char_p,
                                    C.c_size_t]),
    "ldsc_panel_upload": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint64, C.c_uint64, C.c_uint64,
                                    C.POINTER(C.c_void_p)]),
    "ldsc_panel_synth": (C.c_int, [C.c_void_p, C.POINTER(SynthSpec), C.POINTER(C.c_void_p)]),
    "ldsc_panel_download": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint64, C.c_uint64, C.c_void_p]),
    "ldsc_panel_destroy": (C.c_int, [C.c_void_p]),
    "ldsc_l2_run": (C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(L2Args), C.c_void_p, C.c_void_p,
                              C.POINTER(Perf)]),
    "ldsc_l2_from_bed": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint64, C.c_uint64,
                                   C.POINTER(L2Args), C.c_void_p, C.c_void_p, C.POINTER(Perf)]),
    "ldsc_l2_pair_count": (C.c_int, [C.POINTER(L2Args), C.POINTER(C.c_uint64)]),
    "ldsc_snp_stats": (C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(L2Args), C.c_void_p, C.c_void_p]),
    "ldsc_l2_left_limits": (C.c_int, [C.POINTER(L2Args), C.c_void_p]),
    "ldsc_countsketch_hash": (C.c_int, [C.c_uint64, C.c_uint32, C.c_uint64, C.c_void_p,
                                        C.c_void_p]),
    "ldsc_sketch_project": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint64, C.c_uint64, C.c_void_p,
                                      C.c_uint64, C.c_void_p, C.c_void_p, C.c_uint32,
                                      C.c_void_p]),
    "ldsc_debug_gram_i8_tile": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint64, C.c_uint64,
                                          C.c_void_p]),
    "ldsc_l2_int8_noalloc": (C.c_int, [C.c_void_p, C.c_uint64, C.c_uint64, C.c_uint64, C.c_void_p,
                                       C.c_void_p, C.c_void_p, C.c_void_p]),
    "ldsc_noalloc_last_error": (C.c_int, [C.c_char_p, C.c_size_t]),
    "ldsc_ctx_graph_launches": (C.c_uint64, [C.c_void_p]),
    "ldsc_ctx_trim": (C.c_int, [C.c_void_p]),
    "ldsc_panel_shape": (C.c_int, [C.c_void_p, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]),
    "ldsc_l2_workspace_bytes": (C.c_int, [C.POINTER(L2Args), C.c_uint64, C.POINTER(C.c_uint64)]),
    "ldsc_server_create": (C.c_int, [C.c_int, C.c_uint32, C.c_uint64, C.POINTER(C.c_void_p)]),
    "ldsc_server_submit": (C.c_int, [C.c_void_p, C.POINTER(Job), C.POINTER(C.c_uint64)]),
    "ldsc_server_wait": (C.c_int, [C.c_void_p, C.c_uint64, C.POINTER(JobResult)]),
    "ldsc_server_stats_get": (C.c_int, [C.c_void_p, C.POINTER(ServerStats)]),
    "ldsc_server_prewarm": (C.c_int, [C.c_void_p, C.POINTER(Job)]),
    "ldsc_server_destroy": (C.c_int, [C.c_void_p]),
    "ldsc_h2_batch": (C.c_int, [C.c_void_p, C.POINTER(H2Args), C.c_void_p]),
    "ldsc_rg_batch": (C.c_int, [C.c_void_p, C.POINTER(RgArgs), C.c_void_p]),
    "ldsc_h2_partitioned": (C.c_int, [C.c_void_p, C.POINTER(H2PArgs), C.c_void_p]),
}

NOALLOC_SCRATCH_BYTES = 64 * 1024 * 1024

_lib = None


def load() -> C.CDLL:
    """Load libldsc_b200.so; raise if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"{LIB_PATH} is missing: build it with `python -m ldsc_b200.build` "
                "(there is no CPU fallback)")
        lib = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
    return _lib
