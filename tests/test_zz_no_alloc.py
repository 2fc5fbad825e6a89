"""The allocation-free INT8 l2 entry point (ldsc_l2_int8_noalloc).

It serves callers that cannot allocate device memory (hosts that own all device
memory through their own arena, latency-critical request loops in which an
allocation would synchronise the device).  Its scratch is a static device
array inside the library; inputs and outputs are the caller's device buffers.

This file is collected last on purpose: if it fails, a run that stops at the
first failure has already run every other test.  The test allocates its own
input/output buffers with torch -- only the entry point itself must not
allocate.
"""
import ctypes as C
import os

import numpy as np
import pytest

from ldsc_b200.plink import BimTable

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
TOL = 1e-9   # same bar as the other exact-mode parity tests


def _relerr(a, b):
    return float(np.max(np.abs(a - b) / np.maximum(np.abs(b), 1.0)))


def _device_rows(body, n_indiv):
    import torch
    bpr = (n_indiv + 3) // 4
    pitch = (bpr + 15) // 16 * 16
    padded = np.zeros((body.shape[0], pitch), dtype=np.uint8)
    padded[:, :bpr] = body.reshape(body.shape[0], bpr)
    return torch.from_numpy(padded).cuda(), pitch


def _noalloc(lib, rows, pitch, n_indiv, left):
    import torch
    m = len(left)
    l2 = torch.full((m,), np.nan, dtype=torch.float64, device="cuda")
    maf = torch.full((m,), np.nan, dtype=torch.float64, device="cuda")
    left = np.ascontiguousarray(left, dtype=np.int64)
    rc = lib.ldsc_l2_int8_noalloc(C.c_void_p(rows.data_ptr()), pitch, n_indiv, m, left.ctypes.data,
                                  C.c_void_p(l2.data_ptr()), C.c_void_p(maf.data_ptr()),
                                  C.c_void_p(torch.cuda.current_stream().cuda_stream))
    if rc != 0:
        buf = C.create_string_buffer(512)
        lib.ldsc_noalloc_last_error(buf, 512)
        raise RuntimeError(f"ldsc_l2_int8_noalloc failed ({rc}): {buf.value.decode()}")
    torch.cuda.synchronize()
    return l2.cpu().numpy(), maf.cpu().numpy()


def _case(ctx, body, n_indiv, chr_, cm, bp, masking, chunk):
    from ldsc_b200.api import WindowMode, left_limits, run_l2
    m = len(chr_)
    snps = BimTable(chr_, [f"rs{i}" for i in range(m)], cm, bp, np.arange(m, dtype=np.int64))
    panel = ctx.upload(body, n_indiv)
    ref, ref_maf, _ = run_l2(ctx, snps, panel, WindowMode.Cm(1.0), chunk, snp_level_masking=masking,
                             precision="int8", yes_really=True)
    left = left_limits(snps, WindowMode.Cm(1.0), chunk, snp_level_masking=masking)
    panel.close()
    return ref[:, 0], ref_maf, left


def test_noalloc_matches_existing_entry_point_twice(ctx):
    import torch
    torch.cuda.init()
    lib = ctx.lib
    z = np.load(os.path.join(GOLDEN, "small_panel.npz"))
    n = int(z["n_indiv"])
    rows, pitch = _device_rows(z["body"], n)
    for masking, chunk in [(True, 50), (False, 50)]:
        ref, ref_maf, left = _case(ctx, z["body"], n, z["chr"], z["cm"], z["bp"], masking, chunk)
        for _ in range(2):   # two calls in a row on the same static scratch
            l2, maf = _noalloc(lib, rows, pitch, n, left)
            assert _relerr(l2, ref) < TOL
            np.testing.assert_allclose(maf, ref_maf, atol=1e-15)


def test_noalloc_reuses_scratch_across_shapes(ctx):
    """A call of a different shape in between leaves no trace in the next one."""
    from ldsc_b200 import synth
    lib = ctx.lib
    spec = synth.PanelSpec(n_indiv=1337, chrom_sizes=[900], chrom_cm=[4.0], founders=15, miss=0.02, seed=21)
    body = synth.bed_body(spec)
    chr_, cm, bp = synth.positions(spec)
    ref_b, _, left_b = _case(ctx, body, spec.n_indiv, chr_, cm, bp, True, 200)
    rows_b, pitch_b = _device_rows(body, spec.n_indiv)
    z = np.load(os.path.join(GOLDEN, "small_panel.npz"))
    n = int(z["n_indiv"])
    ref_a, _, left_a = _case(ctx, z["body"], n, z["chr"], z["cm"], z["bp"], True, 50)
    rows_a, pitch_a = _device_rows(z["body"], n)
    l2a1, _ = _noalloc(lib, rows_a, pitch_a, n, left_a)
    l2b, _ = _noalloc(lib, rows_b, pitch_b, spec.n_indiv, left_b)
    l2a2, _ = _noalloc(lib, rows_a, pitch_a, n, left_a)
    assert _relerr(l2b, ref_b) < TOL
    assert _relerr(l2a1, ref_a) < TOL
    assert _relerr(l2a2, ref_a) < TOL


def test_noalloc_call_leaves_device_memory_unchanged(ctx):
    """After a first call on the device, a call changes neither the device's
    free memory nor torch's allocations: the entry point allocates nothing."""
    import torch
    lib = ctx.lib
    z = np.load(os.path.join(GOLDEN, "small_panel.npz"))
    n = int(z["n_indiv"])
    rows, pitch = _device_rows(z["body"], n)
    _, _, left = _case(ctx, z["body"], n, z["chr"], z["cm"], z["bp"], True, 50)
    left = np.ascontiguousarray(left, dtype=np.int64)
    m = len(left)
    l2 = torch.zeros(m, dtype=torch.float64, device="cuda")
    maf = torch.zeros(m, dtype=torch.float64, device="cuda")
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)

    def call():
        rc = lib.ldsc_l2_int8_noalloc(C.c_void_p(rows.data_ptr()), pitch, n, m, left.ctypes.data,
                                      C.c_void_p(l2.data_ptr()), C.c_void_p(maf.data_ptr()), stream)
        assert rc == 0
        torch.cuda.synchronize()

    call()   # first call on the device: symbol lookup, kernels loaded
    free0, _ = torch.cuda.mem_get_info()
    alloc0 = torch.cuda.memory_allocated()
    call()
    free1, _ = torch.cuda.mem_get_info()
    assert torch.cuda.memory_allocated() == alloc0
    assert free1 >= free0


def test_noalloc_rejects_requests_beyond_the_scratch(ctx):
    import torch
    from ldsc_b200._lib import NOALLOC_SCRATCH_BYTES
    lib = ctx.lib
    n = 50000
    m = NOALLOC_SCRATCH_BYTES // (2 * 50048) + 16      # operands alone overflow the array
    rows = torch.zeros(16, dtype=torch.uint8, device="cuda")   # never read: rejected before launch
    left = np.zeros(m, dtype=np.int64)
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    rc = lib.ldsc_l2_int8_noalloc(C.c_void_p(rows.data_ptr()), 12512, n, m, left.ctypes.data,
                                  C.c_void_p(out.data_ptr()), C.c_void_p(out.data_ptr()), None)
    assert rc == -1
    buf = C.create_string_buffer(512)
    lib.ldsc_noalloc_last_error(buf, 512)
    assert b"bytes of scratch" in buf.value
