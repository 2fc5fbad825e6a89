"""Benchmark of the l2 LD-score hot path: r^2-pairs/sec on one B200.

Workload (N = 1): the exact biobank-scale configuration -- synthetic panel
N = 50,000 individuals x M = 100,000 SNPs (200 founders, 1% missing, 100 cM),
--ld-wind-cm 1 --snp-level-masking.  One step = one full l2 pass over the
panel (decode + band Gram + r^2 epilogue + l2 back to the host) in the
INT8-exact form.  The plain FP64 form is timed on the same panel for the
INT8-vs-FP64 ratio.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

With --gpus N (launched by torchrun) the ranks split the one panel into
record cores balanced by pair count; each rank computes its core plus the
halo records its windows need on its own GPU, and one all-gather of the core
rows assembles the l2 (strong scaling; the time is the max over ranks).
With --weak each rank computes its own panel (seed + rank) instead.  The reference arm
(--impl reference) times the C restatement of the reference's CPU l2 path
(the reference is Rust and cannot be compiled in this image) on all host
cores, on a bounded SNP sample of the same workload.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "r2 pairs/sec (INT8 exact vs FP64 plain, same GPU); p50/p99 request latency"
CPU_SAMPLE_SNPS = 3000
SKETCH_ORACLE_SNPS = 2000


def workload_spec(seed_offset=0, workload="biobank"):
    """biobank: N=50,000 x M=100,000 (the measured configuration);
    profile: the same panel truncated to its first 8,000 SNPs (INT8 operands
    0.8 GB, larger than L2) for ncu captures."""
    from ldsc_b200 import synth
    s = synth.spec_biobank()
    if workload == "profile":
        s.chrom_sizes = [8000]
        s.chrom_cm = [8.0]
    s.seed += seed_offset
    return s


def config_dict(spec, workload="biobank exact l2, 1 cM, per-SNP masking"):
    return {"workload": workload, "n_indiv": spec.n_indiv, "n_snp": spec.m, "founders": spec.founders,
            "missing": spec.miss, "window": "1 cM", "snp_level_masking": True, "chunk_size": 200,
            "l2_flush": "inputs larger than L2 (1.25 GB packed panel, 10 GB INT8 operands)"}


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if not self.proc:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx.append(float(f[2]))
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        os.unlink(self.path)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return d.get("hbm_gbs", 6650.0), d.get("bf16_tflops", 1590.0), "measured"
    return 6650.0, 1590.0, "fallback"


def committed_traffic(kernel: str):
    """DRAM bytes per launch of the kernel from the committed ncu summary."""
    p = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return d.get(kernel)
    return None


def cpu_baseline(body_rows, spec, chr_, cm, bp, n_threads=0, masking=True, want_l2=False):
    """The C restatement of the reference's l2 (OpenMP, all host threads) on
    the first CPU_SAMPLE_SNPS SNPs of the panel, same flags."""
    sys.path.insert(0, ROOT)
    from oracle import OracleL2Args, max_threads, oracle_l2
    m = body_rows.shape[0]
    a = OracleL2Args(bed_body=body_rows, n_file_indiv=spec.n_indiv, chr=chr_[:m], cm=cm[:m], bp=bp[:m],
                     mode="cm", wind=1.0, chunk_c=200, masking=masking, per_chr=True, n_threads=n_threads)
    work = {}
    t0 = time.perf_counter()
    l2, _, pairs, _ = oracle_l2(a, work)
    dt = time.perf_counter() - t0
    cores = n_threads or max_threads()
    # the restatement's chunk Grams: dot products actually computed (w x c + c x c
    # per chunk, 2 N flops each) over their wall time, per host thread
    work["gemm_gflops_per_core"] = 2.0 * spec.n_indiv * work["n_dots"] / work["gemm_secs"] / 1e9 / cores
    work["gemm_share_of_time"] = work["gemm_secs"] / dt
    work["useful_gflops_per_core"] = 2.0 * spec.n_indiv * pairs / dt / 1e9 / cores
    if want_l2:
        return pairs / dt, pairs, dt, cores, l2[:, 0], work
    return pairs / dt, pairs, dt, cores, work


def cpu_gemm_fields(work):
    return {"gemm_gflops_per_core": work["gemm_gflops_per_core"],
            "gemm_share_of_time": work["gemm_share_of_time"],
            "useful_gflops_per_core": work["useful_gflops_per_core"],
            "gemm_note": "cache-blocked Gram of the C restatement (64 x 64 column macro tiles, 256-individual "
                         "slices; where the host has AVX-512 the slice's A columns are packed and a 16 x 8 "
                         "outer-product micro kernel runs over them, else 3 x 4 AVX2 dot-product blocks); "
                         "gemm = dot products the chunk Grams computed, useful = 2 N per counted pair"}


def max_rel_per_l2j(got, ref):
    """max_j |got_j - ref_j| / |ref_j| (every l2_j of these panels is well away from 0)."""
    return float(np.max(np.abs(got - ref) / np.abs(ref)))


def oracle_parity(ctx, panel, spec, snps, chr_, cm, bp, l2_full_masked, masked_sample_l2):
    """Per-l2_j parity of the GPU forms against the oracle at the benchmark's
    own N, on the SNP sample the CPU baseline times (records
    [0, CPU_SAMPLE_SNPS) of the panel, both window modes):
      * sample: the INT8 and FP64 forms run on exactly the oracle's inputs;
      * full panel: l2 of the full-size INT8 run for every SNP whose pairs all
        lie inside the sample (j < left[CPU_SAMPLE_SNPS] of the full run, as
        left is non-decreasing), against the same oracle values."""
    from ldsc_b200.api import WindowMode, left_limits, run_l2
    from ldsc_b200.plink import BimTable
    m = CPU_SAMPLE_SNPS
    wm = WindowMode.Cm(1.0)
    sample = BimTable(chr_[:m], [f"rs{i}" for i in range(m)], cm[:m], bp[:m], np.arange(m, dtype=np.int64))
    rows = panel.download(0, m)
    out = {"sample": f"records [0, {m}) of the panel, N={spec.n_indiv}, 1 cM, chunk 200",
           "metric": "max_j |l2_j - oracle_j| / |oracle_j|"}
    per_mode = {}
    for name, masking in (("masked", True), ("chunk200", False)):
        if masking:
            ref = masked_sample_l2
        else:
            ref = cpu_baseline(rows, spec, chr_, cm, bp, masking=False, want_l2=True)[4]
        got8 = run_l2(ctx, sample, panel, wm, 200, snp_level_masking=masking, precision="int8", yes_really=True)[0]
        got64 = run_l2(ctx, sample, panel, wm, 200, snp_level_masking=masking, precision="fp64", yes_really=True)[0]
        full = l2_full_masked if masking else run_l2(ctx, snps, panel, wm, 200, snp_level_masking=False,
                                                     precision="int8", yes_really=True)[0][:, 0]
        inside = int(left_limits(snps, wm, 200, snp_level_masking=masking)[m])
        per_mode[name] = {"int8": max_rel_per_l2j(got8[:, 0], ref), "fp64": max_rel_per_l2j(got64[:, 0], ref),
                          "full_panel_int8": max_rel_per_l2j(full[:inside], ref[:inside]),
                          "full_panel_snps_compared": inside, "min_abs_oracle_l2": float(np.min(np.abs(ref)))}
    out["int8_vs_oracle_max_rel_per_l2j"] = {k: v["int8"] for k, v in per_mode.items()}
    out["fp64_vs_oracle_max_rel_per_l2j"] = {k: v["fp64"] for k, v in per_mode.items()}
    out["full_panel_int8_vs_oracle_max_rel_per_l2j"] = {k: v["full_panel_int8"] for k, v in per_mode.items()}
    out["detail"] = per_mode
    out["bar"] = 1e-6
    return out


def run_reference(args):
    """--impl reference: the reference's CPU path (C restatement) on host cores."""
    from ldsc_b200 import synth
    spec = workload_spec()
    chr_, cm, bp = synth.positions(spec)
    rows = synth.bed_body(spec, 0, CPU_SAMPLE_SNPS)
    for _ in range(args.warmup):
        cpu_baseline(rows[:200], spec, chr_, cm, bp)
    vals, tot_pairs, tot_t = [], 0, 0.0
    cores, work = None, None
    for _ in range(args.steps):
        v, pairs, dt, cores, work = cpu_baseline(rows, spec, chr_, cm, bp)
        vals.append(v)
        tot_pairs += pairs
        tot_t += dt
    value = tot_pairs / tot_t
    sample = (f"first {CPU_SAMPLE_SNPS} SNPs of the N=50,000 x M=100,000 panel per step "
              "(1 cM, per-SNP masking, chunk 200, f64)")
    out = {"metric": METRIC, "impl": "reference", "value": value, "unit": "r2 pairs/s", "n_gpus": args.gpus,
           "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * tot_t / args.steps,
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
           "data": "synthetic (seeded founder-mosaic panel)", "config": config_dict(spec),
           "cpu_baseline": {"value": value, "unit": "r2 pairs/s", "cores": cores, "kind": "port",
                            "sample": sample, **cpu_gemm_fields(work)},
           "e2e": {"value": value, "unit": "r2 pairs/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
           "note": "reference is Rust (no cargo/rustc in this image); timed arm is the C restatement "
                   "oracle/ldsc_oracle.c of its CPU l2 path"}
    print(json.dumps(out))


def _timed_passes(ctx, stream, fn, warmup, steps):
    """Run fn() warmup times, then time `steps` calls on the stream (CUDA events)."""
    import torch
    outs = []
    for _ in range(warmup):
        fn()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        outs.append(fn())
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / 1e3, outs


def run_sketch_workload(args, ctx, stream):
    """Fused CountSketch l2: N=100,000 x M=200,000 (1% missing, 150 cM),
    --sketch d --snp-level-masking, 1 cM.  Prints one JSON line per d with
    the sketch pass rate, the scatter kernel's HBM roofline, the error of the
    sketched l2 against exact l2 (INT8 form) on the same panel, and -- on the
    first SKETCH_ORACLE_SNPS records -- the GPU sketch against the oracle's
    f32 --sketch path (seed-42 stream) and both sketches' Pearson r against
    the oracle's exact l2 on that sample."""
    from ldsc_b200 import synth
    from ldsc_b200.api import WindowMode, pair_count, run_l2
    from ldsc_b200.plink import BimTable
    spec = synth.spec_sketch()
    if args.sketch_snps:
        spec.chrom_sizes = [args.sketch_snps]
        spec.chrom_cm = [150.0 * args.sketch_snps / 200000]
    chr_, cm, bp = synth.positions(spec)
    m = spec.m
    snps = BimTable(chr_, [f"rs{i}" for i in range(m)], cm, bp, np.arange(m, dtype=np.int64))
    panel = ctx.synth(spec.n_indiv, m, spec.founders, spec.switch_p, spec.miss, spec.seed)
    wm = WindowMode.Cm(1.0)
    npairs = pair_count(snps, wm, 200, snp_level_masking=True)
    t_ex, outs = _timed_passes(ctx, stream, lambda: run_l2(ctx, snps, panel, wm, 200, snp_level_masking=True,
                                                           precision="int8", yes_really=True), 1, 1)
    exact = outs[0][0][:, 0]
    hbm, bf16, src = measured_peaks()
    tf32_peak = bf16 / 2.0
    # oracle sample: records [0, ms) of the same panel
    from oracle import OracleL2Args, oracle_l2
    ms = min(SKETCH_ORACLE_SNPS, m)
    sample = BimTable(chr_[:ms], [f"rs{i}" for i in range(ms)], cm[:ms], bp[:ms], np.arange(ms, dtype=np.int64))
    srows = panel.download(0, ms)
    sarg = dict(bed_body=srows, n_file_indiv=spec.n_indiv, chr=chr_[:ms], cm=cm[:ms], bp=bp[:ms], chunk_c=200,
                masking=True)
    exact_o = oracle_l2(OracleL2Args(**sarg))[0][:, 0]
    for d in [int(x) for x in args.sketch_d.split(",")]:
        # the first call with this d builds the CountSketch layout (hash, bucket-major
        # order, panel rewritten in it): its one-time cost, then the timed passes
        layout_s = run_l2(ctx, snps, panel, wm, 200, snp_level_masking=True, sketch=d,
                          yes_really=True)[2].layout_secs
        t, outs = _timed_passes(ctx, stream, lambda: run_l2(ctx, snps, panel, wm, 200, snp_level_masking=True,
                                                            sketch=d, yes_really=True), args.warmup, args.steps)
        sk = outs[-1][0][:, 0]
        sk_o = oracle_l2(OracleL2Args(**sarg, use_f32=True, sketch_d=d))[0][:, 0]
        sk_g = run_l2(ctx, sample, panel, wm, 200, snp_level_masking=True, sketch=d, yes_really=True)[0][:, 0]
        vs_oracle = {"snps": ms, "max_abs_diff": float(np.max(np.abs(sk_g - sk_o))),
                     "max_rel_per_l2j": float(np.max(np.abs(sk_g - sk_o) / np.abs(sk_o))),
                     "pearson_gpu_sketch_vs_exact": float(np.corrcoef(sk_g, exact_o)[0, 1]),
                     "pearson_oracle_sketch_vs_exact": float(np.corrcoef(sk_o, exact_o)[0, 1]),
                     "mean_exact_l2": float(np.mean(exact_o))}
        perf = outs[-1][2]
        sk_s = float(np.mean([o[2].sketch_secs for o in outs]))
        gram_s = float(np.mean([o[2].ab_dot_secs for o in outs]))
        bpr = (spec.n_indiv + 3) // 4
        alg_bytes = m * bpr + m * d * 4 + spec.n_indiv * 4
        achieved = alg_bytes / sk_s / 1e9
        out = {"workload": "sketch", "config": {"n_indiv": spec.n_indiv, "n_snp": m, "sketch_d": d,
                                                "window": "1 cM", "snp_level_masking": True},
               "metric": "r2 pairs/sec (sketch form)", "value": npairs * args.steps / t, "unit": "r2 pairs/s",
               "ms_per_step": 1e3 * t / args.steps, "n_pairs": npairs,
               "exact_int8_pairs_per_s": npairs / t_ex,
               "layout_build_ms": 1e3 * layout_s,
               "sketch_kernel_ms": 1e3 * sk_s, "sketch_gram_ms": 1e3 * gram_s, "decode_ms": 1e3 * perf.norm_secs,
               "device_ms_per_call": float(np.mean([o[2].device_ms for o in outs])),
               "sketch_roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                                   "frac": achieved / hbm, "algorithmic_bytes": alg_bytes, "peak_source": src},
               # the TF32 band Gram: every tile computes 64 x 128 record pairs over hi/lo rows
               # (4 products of round_up(d, 32) terms per pair, 8 flops per term); useful
               # work is 2 d flops per in-band pair
               "sketch_gram_roofline": {"bound": "tensor (TF32)", "unit": "TFLOP/s",
                                        "achieved": 8.0 * ((d + 31) // 32 * 32) * 64 * 128 * perf.n_tiles
                                        / gram_s / 1e12,
                                        "peak": tf32_peak, "frac": 8.0 * ((d + 31) // 32 * 32) * 64 * 128
                                        * perf.n_tiles / gram_s / 1e12 / tf32_peak,
                                        "useful_tflops": 2.0 * d * npairs / gram_s / 1e12,
                                        "tiles": int(perf.n_tiles), "peak_source": src,
                                        "note": "peak = half the bf16 dense burst (dense TF32 is half rate)"},
               "vs_exact": {"pearson_r": float(np.corrcoef(sk, exact)[0, 1]),
                            "max_abs_err": float(np.max(np.abs(sk - exact))),
                            "mean_abs_err": float(np.mean(np.abs(sk - exact))),
                            "mean_exact_l2": float(np.mean(exact))},
               "vs_oracle_sketch": vs_oracle}
        print(json.dumps(out), flush=True)
    panel.close()


def run_partitioned_workload(args, ctx, stream):
    """Partitioned LD scores: N=10,000, M=500,000 over 22 chromosomes, 97
    annotations, 1 cM windows, chunk 200 (default mode), all chromosomes in
    one call.  INT8 and FP64 forms; the last three chromosomes are checked
    against the C oracle."""
    from ldsc_b200 import synth
    from ldsc_b200.api import WindowMode, pair_count, run_l2
    from ldsc_b200.plink import BimTable
    from oracle import OracleL2Args, oracle_l2
    spec = synth.spec_partitioned()
    if args.part_snps:
        # profiling case: chromosome 1 alone, cut to part_snps records at the same SNP density
        spec.chrom_cm = [spec.chrom_cm[0] * args.part_snps / spec.chrom_sizes[0]]
        spec.chrom_sizes = [args.part_snps]
    chr_, cm, bp = synth.positions(spec)
    m = spec.m
    snps = BimTable(chr_, [f"rs{i}" for i in range(m)], cm, bp, np.arange(m, dtype=np.int64))
    annot = synth.partitioned_annot(m)
    panel = ctx.synth(spec.n_indiv, m, spec.founders, spec.switch_p, spec.miss, spec.seed)
    wm = WindowMode.Cm(1.0)
    npairs = pair_count(snps, wm, 200)
    import torch
    res = {}
    for prec in ("int8", "fp64"):
        t, outs = _timed_passes(ctx, stream, lambda: run_l2(ctx, snps, panel, wm, 200, annot=annot,
                                                            precision=prec, yes_really=True),
                                args.warmup if prec == "int8" else 1, args.steps if prec == "int8" else 2)
        res[prec] = (t / (args.steps if prec == "int8" else 2), outs[-1])
    # inputs and outputs resident in HBM: annotations read in place, l2 / MAF left on the device
    K = annot.shape[1]
    d_annot = torch.from_numpy(np.ascontiguousarray(annot.T)).cuda()   # column c of SNP r at c * m + r
    d_l2 = torch.empty((K, m), dtype=torch.float64, device="cuda")
    d_maf = torch.empty(m, dtype=torch.float64, device="cuda")
    t_res, outs_res = _timed_passes(ctx, stream, lambda: run_l2(ctx, snps, panel, wm, 200, precision="int8",
                                                                yes_really=True,
                                                                annot_device=(d_annot.data_ptr(), m, K),
                                                                out_device=(d_l2, d_maf)),
                                    args.warmup, args.steps)
    pr = outs_res[-1][2]
    resident = {"pairs_per_s": npairs * args.steps / t_res, "ms_per_step": 1e3 * t_res / args.steps,
                "decode_ms": 1e3 * pr.norm_secs, "gram_and_contraction_ms": 1e3 * pr.ab_dot_secs,
                "contraction_ms": 1e3 * pr.contract_secs,
                "device_ms": pr.device_ms,
                "matches_host_call": float(np.max(np.abs(d_l2.T.cpu().numpy() - res["int8"][1][0])))}
    h2p = None if args.part_snps else _partitioned_h2(ctx, stream, d_l2, annot, args)
    l2i = res["int8"][1][0]
    l2f = res["fp64"][1][0]
    # oracle on the three smallest chromosomes (independent in per-chromosome mode);
    # not on the one-chromosome profiling case
    start = int(np.searchsorted(chr_, 20)) if not args.part_snps else m
    ref = np.zeros((0, annot.shape[1]))
    if start < m:
        rows = panel.download(start, m)
        ref, _, _, _ = oracle_l2(OracleL2Args(bed_body=rows, n_file_indiv=spec.n_indiv, chr=chr_[start:],
                                              cm=cm[start:], bp=bp[start:], chunk_c=200, annot=annot[start:]))
    scale = np.maximum(np.abs(ref).max(axis=0, keepdims=True), 1.0) if start < m else 1.0
    out = {"workload": "partitioned", "config": {"n_indiv": spec.n_indiv, "n_snp": m, "chromosomes": len(spec.chrom_sizes),
                                                 "annotations": annot.shape[1], "window": "1 cM", "chunk_size": 200},
           "metric": "r2 pairs/sec", "n_pairs": npairs,
           "int8_resident": resident,
           "int8": {"pairs_per_s": npairs / res["int8"][0], "ms_per_step": 1e3 * res["int8"][0],
                    "gram_ms": 1e3 * res["int8"][1][2].ab_dot_secs},
           "fp64": {"pairs_per_s": npairs / res["fp64"][0], "ms_per_step": 1e3 * res["fp64"][0],
                    "gram_ms": 1e3 * res["fp64"][1][2].ab_dot_secs},
           "int8_vs_oracle_chr20_22": float(np.max(np.abs(l2i[start:] - ref) / scale)) if start < m else None,
           "fp64_vs_oracle_chr20_22": float(np.max(np.abs(l2f[start:] - ref) / scale)) if start < m else None,
           "int8_vs_fp64_all": float(np.max(np.abs(l2i - l2f) / np.maximum(np.abs(l2f).max(axis=0, keepdims=True), 1.0))),
           "error_metric": "max |l2_jC - ref_jC| / max(max_j |ref_jC|, 1) per annotation column",
           "h2_partitioned": h2p}
    print(json.dumps(out), flush=True)
    panel.close()


def run_partitioned_h2_workload(args, ctx, stream):
    """Partitioned h2 alone: seeded synthetic K-column LD scores resident in
    HBM (l2_k = base * Dirichlet fractions, base = 1 + Gamma(2, 15)), traits
    chi2 = chi2_1 * (1 + base / 60), N = 1e5, 200 blocks; times the whole
    ldsc_h2_partitioned call on device pointers.  Sizes: --h2p-snps,
    --h2p-annot, --h2p-traits."""
    import torch
    from ldsc_b200.partitioned import default_chisq_max, h2_partitioned_device
    m, K, T = args.h2p_snps, args.h2p_annot, args.h2p_traits
    rng = np.random.default_rng(1)
    base = 1.0 + rng.gamma(2.0, 15.0, m)
    l2 = np.ascontiguousarray((base[:, None] * rng.dirichlet(np.ones(K), size=m)).T)   # (K, m)
    chi2 = rng.chisquare(1, (T, m)) * (1.0 + base / 60.0)
    nn = np.full(T, 1e5)
    d = dict(chi2=torch.from_numpy(chi2).cuda(), n=torch.from_numpy(nn).cuda(), l2=torch.from_numpy(l2).cuda(),
             w=torch.from_numpy(base).cuda())
    cmax = [default_chisq_max(chi2[t], nn[t]) for t in range(T)]
    m_vec = np.full(K, 1e4)
    call = lambda: h2_partitioned_device(ctx, d["chi2"], d["n"], d["l2"], d["w"], m_vec, cmax, 200)  # noqa: E731
    t, outs = _timed_passes(ctx, stream, call, max(args.warmup, 1), max(args.steps, 1))
    ms = 1e3 * t / max(args.steps, 1)
    q = K + 2
    print(json.dumps({"workload": "partitioned-h2", "config": {"n_snp": m, "annotations": K, "traits": T,
                                                              "n_blocks": 200},
                      "ms_per_call": ms, "traits_per_s": T / (ms / 1e3),
                      "gram_flops_per_call": sum(f.n_obs for f in outs[-1]) * q * (q + 1)}), flush=True)


def _partitioned_h2(ctx, stream, d_l2, annot, args, n_traits=8, n_blocks=200):
    """Partitioned h2 (fit_h2_partitioned) of n_traits synthetic traits on the
    device-resident K-column LD scores just computed: chi2 = (sqrt(N s) b +
    e)^2 with s = max(h2 (l2_all + sum_c tau_c l2_c) / M, 0) over the binary
    annotations (generating total h2 = h2 sum_k tau_k M_k / M), w_l2 = the
    all-ones column's l2, M_k = annotation column sums.  Times the whole call (device pointers in, estimates out) and checks
    the first trait against the oracle."""
    import torch
    from ldsc_b200.partitioned import default_chisq_max, h2_partitioned_device
    from oracle import regress_oracle as R
    K, m = int(d_l2.shape[0]), int(d_l2.shape[1])
    l2h = d_l2.T.cpu().numpy()
    rng = np.random.default_rng(17)
    h2 = rng.uniform(0.1, 0.5, n_traits)
    nn = np.exp(rng.uniform(np.log(5e4), np.log(3e5), n_traits))
    tau = np.zeros((n_traits, K))
    tau[:, 0] = 1.0
    tau[:, 1:81] = rng.uniform(0.0, 0.5, (n_traits, 80))
    s = np.maximum((h2[:, None] / m) * (tau @ l2h.T), 0.0)
    z = np.sqrt(nn[:, None] * s) * rng.standard_normal((n_traits, m)) + rng.standard_normal((n_traits, m))
    chi2 = z * z
    m_vec = annot.sum(axis=0)
    cmax = np.array([default_chisq_max(chi2[t], nn[t]) for t in range(n_traits)])
    d_chi2 = torch.from_numpy(chi2).cuda()
    d_n = torch.from_numpy(nn).cuda()
    w = d_l2[0].contiguous()
    call = lambda: h2_partitioned_device(ctx, d_chi2, d_n, d_l2, w, m_vec, cmax, n_blocks)  # noqa: E731
    t, outs = _timed_passes(ctx, stream, call, max(args.warmup, 1), max(args.steps, 3))
    fits = outs[-1]
    want = R.fit_h2_partitioned(chi2[0], l2h, l2h[:, 0], nn[0], m_vec, n_blocks)
    got = fits[0]
    n_obs = sum(f.n_obs for f in fits)
    q = K + 2                       # augmented columns: K LD scores, intercept, chi2
    gram_flops = n_obs * q * (q + 1)  # upper triangle, one multiply-add per entry and kept SNP
    ms = 1e3 * t / max(args.steps, 3)
    return {"traits": n_traits, "annotations": K, "n_snp": m, "n_blocks": n_blocks, "ms_per_call": ms,
            "traits_per_s": n_traits / (ms / 1e3), "gram_flops_per_call": gram_flops,
            "gram_tflops_lower_bound": gram_flops / (ms / 1e3) / 1e12,
            "h2_total": [f.h2_total for f in fits],
            "h2_generating": [float(h2[t] / m * np.dot(tau[t], m_vec)) for t in range(n_traits)],
            "vs_oracle_trait0": {"h2_total_rel": abs(got.h2_total - want["h2_total"]) / abs(want["h2_total"]),
                                 "est_max_rel": float(np.max(np.abs(got.est - want["est"])) /
                                                      np.max(np.abs(want["est"])))},
            "note": "whole ldsc_h2_partitioned call on device pointers (8 traits x 500,000 SNPs x 97 "
                    "annotations); the Gram rate is a lower bound (call time includes the solves)"}


def run_regressions_workload(args, seed: int = 7):
    """Batched regressions on device-resident inputs, as the serving mix runs
    them: h2 over 1,000 synthetic traits x 200,000 regression SNPs (200-block
    jackknife; with and without lambda GC) and rg over 200 trait pairs, each
    through one server slot.  Prints one JSON line with the median run time
    of each (the first call of each kind, which captures its graph, is left
    out)."""
    import torch
    from ldsc_b200.serve import Server
    T, P, n_reg, M = 1000, 200, 200_000, 1_200_000
    dev = torch.device("cuda")
    g = torch.Generator(device=dev)
    g.manual_seed(seed)
    f64 = torch.float64
    ld = 1 + 30 * torch.rand(n_reg, generator=g, device=dev, dtype=f64)
    h2 = 0.05 + 0.45 * torch.rand(T, generator=g, device=dev, dtype=f64)
    n_t = torch.exp(np.log(1e4) + (np.log(5e5) - np.log(1e4)) * torch.rand(T, generator=g, device=dev, dtype=f64))
    z = torch.sqrt(n_t[:, None] * h2[:, None] * ld[None, :] / M) * torch.randn(T, n_reg, generator=g, device=dev,
                                                                               dtype=f64)
    z += torch.randn(T, n_reg, generator=g, device=dev, dtype=f64)
    chi2 = (z * z).contiguous()
    del z
    z1 = torch.randn(P, n_reg, generator=g, device=dev, dtype=f64)
    z2 = 0.5 * z1 + torch.randn(P, n_reg, generator=g, device=dev, dtype=f64)
    n1 = torch.full((P,), 1e5, device=dev, dtype=f64)
    torch.cuda.synchronize()
    srv = Server(torch.cuda.current_device(), n_slots=1)
    out = {"workload": "regressions", "metric": "run time per batched call (ms, median)",
           "config": {"h2": f"{T} traits x {n_reg} SNPs, 200 blocks", "rg": f"{P} pairs x {n_reg} SNPs, 200 blocks",
                      "inputs": "device-resident (chi2 / z, LD scores, N)"}}
    try:
        for name, fn in [("h2_lambda_gc", lambda: srv.submit_h2(chi2, n_t, ld, ld, float(M), 200)),
                         ("h2", lambda: srv.submit_h2(chi2, n_t, ld, ld, float(M), 200, lambda_gc=False)),
                         ("rg", lambda: srv.submit_rg(z1, z2, n1, n1, ld, ld, float(M), 200))]:
            runs = [srv.wait(fn())[1].run_ms for _ in range(args.warmup + args.steps)]
            out[name + "_ms"] = float(np.median(runs[args.warmup:]))
    finally:
        srv.close()
    out["h2_bytes_per_weighted_pass"] = T * n_reg * 8
    return out


def run_serving_workload(args, ctx, duration_s: float, rates, seed: int = 7):
    """Serving mix on a resident N=20,000 x M=1,200,000 panel (22
    chromosomes, 3,500 cM).  Poisson arrivals at each rate (requests/s) for
    `duration_s` seconds: 70% LD-score requests (region M log-uniform in
    [2,000, 200,000], K in {1, 10, 97} from resident annotations, exact INT8
    or sketch d=1000, 1 cM, per-SNP masking), 20% h2 over 1,000 traits and 10%
    rg over 200 trait pairs, both against the resident LD scores of every 6th
    SNP (200,000 regression SNPs, 200-block jackknife).  Returns the latency
    and throughput summary, one per rate of `rates` (the same server and
    resident data serve the rates one after another)."""
    import threading
    import queue as pyqueue
    import torch
    from ldsc_b200 import synth
    from ldsc_b200.api import WindowMode, run_l2
    from ldsc_b200.plink import BimTable
    from ldsc_b200.serve import Server
    t_setup = time.perf_counter()
    spec = synth.spec_resident()
    chr_, cm, bp = synth.positions(spec)
    M = spec.m
    names = [f"rs{i}" for i in range(M)]
    snps = BimTable(chr_, names, cm, bp, np.arange(M, dtype=np.int64))
    panel = ctx.synth(spec.n_indiv, M, spec.founders, spec.switch_p, spec.miss, spec.seed)
    wm = WindowMode.Cm(1.0)
    # resident LD-score store (K = 1, INT8, masked) and regression inputs
    l2_all, _, _ = run_l2(ctx, snps, panel, wm, 200, snp_level_masking=True, precision="int8", yes_really=True)
    reg_idx = np.arange(0, M, 6)
    n_reg = len(reg_idx)
    dev = torch.device("cuda")
    d_ld = torch.from_numpy(np.ascontiguousarray(l2_all[reg_idx, 0])).to(dev)
    g = torch.Generator(device=dev)
    g.manual_seed(seed)
    T = 1000

    def uni(lo, hi, n):
        return lo + (hi - lo) * torch.rand(n, generator=g, device=dev, dtype=torch.float64)

    def randn(r, c):
        return torch.randn(r, c, generator=g, device=dev, dtype=torch.float64)

    h2 = uni(0.05, 0.5, T)
    n_t = torch.exp(uni(np.log(1e4), np.log(5e5), T))
    lm = d_ld.clamp_min(0)[None, :]
    z = torch.sqrt(n_t[:, None] * h2[:, None] * lm / M) * randn(T, n_reg) + randn(T, n_reg)
    d_chi2 = z * z
    del z
    # trait pairs with genetic correlation rg ~ U(-0.8, 0.8)
    Pn = 1000
    rgv = uni(-0.8, 0.8, Pn)
    h1p, h2p = uni(0.05, 0.5, Pn), uni(0.05, 0.5, Pn)
    n1p = torch.exp(uni(np.log(1e4), np.log(5e5), Pn))
    n2p = torch.exp(uni(np.log(1e4), np.log(5e5), Pn))
    b1 = randn(Pn, n_reg)
    b2 = rgv[:, None] * b1 + torch.sqrt(1 - rgv[:, None] ** 2) * randn(Pn, n_reg)
    d_z1 = torch.sqrt(n1p[:, None] * h1p[:, None] * lm / M) * b1 + randn(Pn, n_reg)
    d_z2 = torch.sqrt(n2p[:, None] * h2p[:, None] * lm / M) * b2 + randn(Pn, n_reg)
    del b1, b2
    annot = synth.partitioned_annot(M, seed=seed)
    d_annot = torch.from_numpy(np.ascontiguousarray(annot.T)).to(dev)   # column c of SNP r at c * M + r
    del annot
    torch.cuda.synchronize()

    def make_requests(rate):
        rng = np.random.default_rng(seed)
        n_req = max(1, int(rate * duration_s))
        arrivals = np.cumsum(rng.exponential(1.0 / rate, n_req))
        reqs = []
        for _ in range(n_req):
            u = rng.random()
            if u < 0.7:
                mreg = int(np.exp(rng.uniform(np.log(2000), np.log(200000))))
                b = int(rng.integers(0, M - mreg))
                reqs.append(("l2", dict(b=b, e=b + mreg, K=int(rng.choice([1, 10, 97])),
                                        sketch=None if rng.random() < 0.5 else 1000)))
            elif u < 0.9:
                reqs.append(("h2", {}))
            else:
                reqs.append(("rg", dict(p0=int(rng.integers(0, Pn - 200)))))
        return reqs, arrivals

    def region(b, e):
        return BimTable(chr_[b:e], names[b:e], cm[b:e], bp[b:e], np.arange(b, e, dtype=np.int64))

    def submit(srv, kind, p):
        if kind == "l2":
            ad = None if p["K"] == 1 else (d_annot.data_ptr() + 8 * p["b"], M, p["K"])
            return srv.submit_l2(panel, region(p["b"], p["e"]), wm, 200, row_begin=p["b"], annot_device=ad,
                                 sketch=p["sketch"], precision="int8", snp_level_masking=True)
        if kind == "h2":
            return srv.submit_h2(d_chi2, n_t, d_ld, d_ld, float(M), 200)
        p0 = p["p0"]
        return srv.submit_rg(d_z1[p0:p0 + 200], d_z2[p0:p0 + 200], n1p[p0:p0 + 200], n2p[p0:p0 + 200], d_ld, d_ld,
                             float(M), 200)

    n_slots = args.serve_slots
    srv = Server(torch.cuda.current_device(), n_slots=n_slots)
    # warm-up: the shared sketch layout, then every slot's workspace sized for
    # the largest request of each kind (ldsc_server_prewarm runs a job on each
    # slot in turn), so no request allocates device memory while others run
    srv.wait(submit(srv, "l2", dict(b=0, e=5000, K=1, sketch=1000)))
    for k, p in [("l2", dict(b=500000, e=700000, K=97, sketch=None)), ("l2", dict(b=500000, e=700000, K=97, sketch=1000)),
                 ("l2", dict(b=500000, e=700000, K=1, sketch=None)), ("l2", dict(b=500000, e=700000, K=1, sketch=1000)),
                 ("h2", {}), ("rg", dict(p0=0))]:
        srv.prewarm(lambda *a: submit(srv, k, p))
    setup_s = time.perf_counter() - t_setup

    def one_rate(rate):
        reqs, arrivals = make_requests(rate)
        n_req = len(reqs)
        done = []
        q = pyqueue.Queue()

        def waiter():
            while True:
                item = q.get()
                if item is None:
                    return
                kind, p, t = item
                try:
                    res, timing = srv.wait(t)
                    pairs = res[2].n_pairs if kind == "l2" else 0
                    done.append((kind, p, timing, pairs, None))
                except Exception as e:  # noqa: BLE001
                    done.append((kind, p, None, 0, str(e)))

        waiters = [threading.Thread(target=waiter) for _ in range(n_slots + 2)]
        for w in waiters:
            w.start()
        st0 = srv.stats()
        t0 = time.perf_counter()
        late = []
        for (kind, p), ta in zip(reqs, arrivals):
            now = time.perf_counter() - t0
            if ta > now:
                time.sleep(ta - now)
            else:
                late.append(now - ta)
            q.put((kind, p, submit(srv, kind, p)))
        for _ in waiters:
            q.put(None)
        for w in waiters:
            w.join()
        wall = time.perf_counter() - t0
        st1 = srv.stats()

        ok = [d for d in done if d[4] is None]
        lat = np.array([d[2].latency_ms for d in ok])
        que = np.array([d[2].queue_ms for d in ok])
        run = np.array([d[2].run_ms for d in ok])

        def pct(a):
            return {"p50": float(np.percentile(a, 50)), "p99": float(np.percentile(a, 99)),
                    "mean": float(np.mean(a)), "max": float(np.max(a)), "n": int(len(a))} if len(a) else None

        def label(kind, p):
            if kind != "l2":
                return kind
            return f"l2_{'sketch1000' if p['sketch'] else 'int8'}_K{p['K']}"

        by = {}
        for d in ok:
            by.setdefault(label(d[0], d[1]), []).append(d[2].latency_ms)
        pairs = float(sum(d[3] for d in ok))
        return {"workload": "serving", "metric": "request latency (ms) and throughput at a stated Poisson rate",
                "rate_req_s": rate, "duration_s": duration_s, "requests": n_req, "completed": len(ok),
                "failed": len(done) - len(ok), "errors": sorted({d[4] for d in done if d[4]})[:3],
                "wall_s": wall, "throughput_req_s": len(ok) / wall, "l2_pairs_per_s": pairs / wall,
                "latency_ms": pct(lat), "queue_ms": pct(que), "run_ms": pct(run),
                "by_kind_latency_ms": {k: pct(np.array(v)) for k, v in sorted(by.items())},
                "arrival_lag_ms_p99": float(np.percentile(late, 99) * 1e3) if late else 0.0,
                "slots": n_slots, "graph_launches": st1["graph_launches"] - st0["graph_launches"],
                "gpu_launches": st1["kernels"] - st0["kernels"], "setup_s": setup_s,
                "config": {"panel": "N=20,000 x M=1,200,000, 22 chromosomes, 3,500 cM, 1% missing",
                           "l2": "70%: region M log-uniform [2k, 200k], K in {1,10,97} (resident annotations), "
                                 "INT8 exact or sketch d=1000, 1 cM, per-SNP masking",
                           "h2": "20%: 1,000 traits x 200,000 regression SNPs, 200 blocks",
                           "rg": "10%: 200 trait pairs x 200,000 regression SNPs, 200 blocks",
                           "traits": "z = sqrt(N h2 l2 / M) b + e, h2 ~ U(0.05, 0.5), N log-uniform [1e4, 5e5], "
                                     "chi2 = z^2; rg ~ U(-0.8, 0.8)"}}

    try:
        return [one_rate(r) for r in rates]
    finally:
        srv.close()
        panel.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=30)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--fp64-steps", type=int, default=2)
    ap.add_argument("--fused-steps", type=int, default=5,
                    help="passes of the fused INT8 form (no operand buffer) timed for comparison")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--weak", action="store_true",
                    help="N > 1: every rank runs its own panel (seed + rank) instead of a shard of one panel")
    ap.add_argument("--workload", default="biobank",
                    choices=["biobank", "profile", "sketch", "partitioned", "partitioned-h2", "serving",
                             "regressions"])
    ap.add_argument("--h2p-snps", type=int, default=500_000, help="partitioned-h2: regression SNPs")
    ap.add_argument("--h2p-annot", type=int, default=97, help="partitioned-h2: LD-score columns K")
    ap.add_argument("--h2p-traits", type=int, default=8, help="partitioned-h2: traits per call")
    ap.add_argument("--serve-rate", type=float, default=40.0, help="serving: Poisson arrivals per second")
    ap.add_argument("--serve-rates", default="", help="serving workload: comma-separated rates, one line each")
    ap.add_argument("--serve-seconds", type=float, default=30.0, help="serving: length of the arrival window")
    ap.add_argument("--serve-slots", type=int, default=6, help="serving: concurrent job slots")
    ap.add_argument("--no-serving", action="store_true",
                    help="skip the serving and regression summaries of the default run")
    ap.add_argument("--sketch-d", default="200,1000,5000")
    ap.add_argument("--sketch-snps", type=int, default=0, help="truncate the sketch panel (profiling)")
    ap.add_argument("--part-snps", type=int, default=0,
                    help="partitioned workload on chromosome 1 cut to this many records (profiling)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        if rank != 0:
            return
        run_reference(args)
        return

    import torch
    import torch.distributed as dist
    from ldsc_b200.build import build
    build()
    from ldsc_b200 import synth
    from ldsc_b200.api import Context, WindowMode, l2_from_bed_bytes, pair_count, run_l2
    from ldsc_b200.plink import BimTable

    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600))

    def barrier():
        if world > 1:
            dist.barrier()

    ctx = Context(local)
    stream = torch.cuda.current_stream()
    ctx.set_stream(stream.cuda_stream)

    if args.workload == "sketch":
        run_sketch_workload(args, ctx, stream)
        return
    if args.workload == "partitioned":
        run_partitioned_workload(args, ctx, stream)
        return
    if args.workload == "partitioned-h2":
        run_partitioned_h2_workload(args, ctx, stream)
        return
    if args.workload == "regressions":
        print(json.dumps(run_regressions_workload(args)), flush=True)
        return
    if args.workload == "serving":
        rates = [float(x) for x in args.serve_rates.split(",")] if args.serve_rates else [args.serve_rate]
        for line in run_serving_workload(args, ctx, args.serve_seconds, rates):
            print(json.dumps(line), flush=True)
        return

    # N > 1: the ranks split one panel into cores balanced by pair count, each
    # computing its core plus halos, then one all-gather of the core rows
    # (strong scaling); with --weak every rank runs its own panel (seed + rank)
    sharded = world > 1 and not args.weak
    spec = workload_spec(seed_offset=0 if sharded else rank, workload=args.workload)
    chr_, cm, bp = synth.positions(spec)
    m = spec.m
    snps = BimTable(chr_, [f"rs{i}" for i in range(m)], cm, bp, np.arange(m, dtype=np.int64))
    panel = ctx.synth(spec.n_indiv, m, spec.founders, spec.switch_p, spec.miss, spec.seed)
    wm = WindowMode.Cm(1.0)
    npairs = pair_count(snps, wm, 200, snp_level_masking=True)
    if sharded:
        from ldsc_b200.parallel import gather_l2, plan_shards, shard_records
        plan = plan_shards(snps, wm, world, 200, snp_level_masking=True)
        sh = plan[rank]
        rec = shard_records(snps, sh)
        n_call = sh.call_hi - sh.call_lo
        d_l2 = torch.empty((1, n_call), dtype=torch.float64, device="cuda")
        d_maf = torch.empty(n_call, dtype=torch.float64, device="cuda")
        core = slice(sh.core_lo - sh.call_lo, sh.core_hi - sh.call_lo)

    def step(precision):
        if not sharded:
            return run_l2(ctx, snps, panel, wm, 200, snp_level_masking=True, precision=precision, yes_really=True)
        # this rank's call on the resident panel, l2 left on the device, then
        # the gather of every rank's core rows (the full l2 on rank 0's host)
        _, _, perf = run_l2(ctx, rec, panel, wm, 200, snp_level_masking=True, precision=precision,
                            yes_really=True, out_device=(d_l2, d_maf))
        return gather_l2(d_l2[0, core].reshape(-1, 1), plan, rank, dst=0), None, perf

    # ---- INT8 form, inputs resident in HBM ----
    for _ in range(args.warmup):
        step("int8")
    sampler = ClockSampler(local)
    sampler.start()
    barrier()
    torch.cuda.synchronize()
    k0 = ctx.kernel_count
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    gram_s, dec_s, dev_ms = [], [], []
    for _ in range(args.steps):
        l2_last, _, perf = step("int8")
        gram_s.append(perf.ab_dot_secs)
        dec_s.append(perf.norm_secs)
        dev_ms.append(perf.device_ms)
    ev1.record(stream)
    torch.cuda.synchronize()
    barrier()
    clocks = sampler.stop()
    launches = ctx.kernel_count - k0
    t_local = ev0.elapsed_time(ev1) / 1e3
    t_max, pairs_all = t_local, npairs
    rank_pairs = perf.n_pairs   # pairs this rank's call computed (core plus halos when sharded)
    if world > 1:
        tt = torch.tensor([t_local], device="cuda", dtype=torch.float64)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        pp = torch.tensor([npairs], device="cuda", dtype=torch.float64)
        dist.all_reduce(pp, op=dist.ReduceOp.SUM)
        # sharded: the panel's own pairs once; weak: every rank's panel
        t_max, pairs_all = float(tt.item()), (npairs if sharded else float(pp.item()))
    value = pairs_all * args.steps / t_max
    gram_avg = float(np.mean(gram_s))

    # ---- FP64 plain form, same panel ----
    fp64_value, fp64_gram, int8_err = None, [float("nan")], None
    if args.fp64_steps > 0:
        l2_64 = step("fp64")[0]
        l2_i8 = step("int8")[0]
        # l2 of the INT8 form against the FP64 form on the same panel: max |a - b| / max(|b|, 1)
        if l2_64 is not None:
            int8_err = float(np.max(np.abs(l2_i8 - l2_64) / np.maximum(np.abs(l2_64), 1.0)))
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        fp64_gram = []
        for _ in range(args.fp64_steps):
            _, _, p64 = step("fp64")
            fp64_gram.append(p64.ab_dot_secs)
        e1.record(stream)
        torch.cuda.synchronize()
        t64 = e0.elapsed_time(e1) / 1e3
        if world > 1:
            tt = torch.tensor([t64], device="cuda", dtype=torch.float64)
            dist.all_reduce(tt, op=dist.ReduceOp.MAX)
            t64 = float(tt.item())
        fp64_value = pairs_all * args.fp64_steps / t64 / (1 if sharded else world)

    # ---- the fused INT8 form (packed rows expanded in shared memory, no operand buffer) ----
    fused = None
    if not sharded and args.fused_steps > 0:
        ctx2 = Context(local, fused_operands=True)
        ctx2.set_stream(stream.cuda_stream)
        for _ in range(2):
            l2_fused = run_l2(ctx2, snps, panel, wm, 200, snp_level_masking=True, precision="int8",
                              yes_really=True)[0]
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        tp = []
        for _ in range(args.fused_steps):
            tp.append(run_l2(ctx2, snps, panel, wm, 200, snp_level_masking=True, precision="int8",
                             yes_really=True)[2])
        e1.record(stream)
        torch.cuda.synchronize()
        t2 = e0.elapsed_time(e1) / 1e3
        fused = {"pairs_per_s": npairs * args.fused_steps / t2, "ms_per_pass": 1e3 * t2 / args.fused_steps,
                 "gram_ms": 1e3 * float(np.mean([q.ab_dot_secs for q in tp])),
                 "decode_ms": 1e3 * float(np.mean([q.norm_secs for q in tp])),
                 "operand_bytes_saved": 2 * m * ((spec.n_indiv + 127) // 128 * 128),
                 "l2_bit_identical_to_two_pass": bool(np.array_equal(l2_fused, l2_last))}
        ctx2.close()

    # ---- end to end through the whole-file C ABI entry point, host buffers ----
    e2e = None
    if not args.no_e2e:
        # the BED image this rank reads: the whole panel, or its call's rows when sharded
        r0, r1 = (sh.call_lo, sh.call_hi) if sharded else (0, m)
        e2e_snps = snps
        if sharded:
            e2e_snps = rec.subset(np.arange(n_call))
            e2e_snps.bed_idx = np.arange(n_call, dtype=np.int64)
        rows = panel.download(r0, r1)
        bed = torch.empty(3 + rows.size, dtype=torch.uint8, pin_memory=True)
        bnp = bed.numpy()
        bnp[:3] = [0x6C, 0x1B, 0x01]
        bnp[3:] = rows.reshape(-1)
        del rows

        def e2e_step():
            l2h, _, p = l2_from_bed_bytes(ctx, bnp, spec.n_indiv, e2e_snps, wm, 200, precision="int8",
                                          snp_level_masking=True)
            if sharded:
                gather_l2(l2h[core], plan, rank, dst=0)
            return p

        e2e_step()
        barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        e2e_perf = []
        for _ in range(args.steps):
            e2e_perf.append(e2e_step())
        torch.cuda.synchronize()
        te = time.perf_counter() - t0
        if world > 1:
            tt = torch.tensor([te], device="cuda", dtype=torch.float64)
            dist.all_reduce(tt, op=dist.ReduceOp.MAX)
            te = float(tt.item())
        e2e = {"value": pairs_all * args.steps / te, "unit": "r2 pairs/s", "h2d_bytes_per_step": int(bnp.size),
               "d2h_bytes_per_step": int(16 * m), "ms_per_step": 1e3 * te / args.steps,
               "api": "ldsc_l2_from_bed (validate + upload + compute + download)",
               "h2d_ms_median": 1e3 * float(np.median([p.bed_read_secs for p in e2e_perf])),
               "h2d_gbs": bnp.size / 1e9 / float(np.median([p.bed_read_secs for p in e2e_perf])),
               "device_ms_median": float(np.median([p.device_ms for p in e2e_perf]))}

    # ---- roofline of the dominant kernel (INT8 band Gram) ----
    hbm, bf16, src = measured_peaks()
    int8_peak = 2.0 * bf16   # dense int8 tensor rate is 2x bf16 on sm_100
    ops = 8.0 * spec.n_indiv * rank_pairs   # 4 integer products x 2 ops x N per in-band pair
    achieved = ops / gram_avg / 1e12
    roofline = {"bound": "tensor", "achieved": achieved, "peak": int8_peak, "unit": "TFLOP/s",
                "frac": achieved / int8_peak, "traffic": committed_traffic("k_gram_tc"),
                "kernel": "k_gram_tc<4,0,4,0> (tcgen05.mma kind::i8, TMA-staged operand rows)",
                "note": "int8 ops counted like flops (2 per MAC, 4 products per pair); peak = 2 x "
                        + ("measured bf16 dense burst (MEASURED_PEAKS.json)" if src == "measured" else
                           "fallback bf16 dense burst 1590 TFLOP/s (MEASURED_PEAKS.json absent)")
                        + ", nominal int8 dense 4500"}

    cpu, parity = None, None
    if rank == 0 and world == 1 and not args.no_cpu:
        rows = panel.download(0, CPU_SAMPLE_SNPS)
        v, pairs_s, dt, cores, ref_masked, work = cpu_baseline(rows, spec, chr_, cm, bp, want_l2=True)
        cpu = {"value": v, "unit": "r2 pairs/s", "cores": cores, "kind": "port",
               "sample": f"first {CPU_SAMPLE_SNPS} SNPs of the panel ({pairs_s} pairs, {dt:.1f} s), same flags, f64",
               **cpu_gemm_fields(work)}
        if args.workload == "biobank":
            parity = oracle_parity(ctx, panel, spec, snps, chr_, cm, bp, l2_last[:, 0], ref_masked)

    # ---- serving latency at a stated rate (the metric's second half), 1 GPU ----
    serving = None
    if world == 1 and args.serve_seconds > 0 and not args.no_serving:
        try:
            sv = run_serving_workload(args, ctx, min(args.serve_seconds, 10.0), [args.serve_rate])[0]
            serving = {k: sv[k] for k in ("rate_req_s", "duration_s", "requests", "completed", "failed",
                                          "throughput_req_s", "l2_pairs_per_s", "latency_ms", "queue_ms",
                                          "by_kind_latency_ms", "slots", "graph_launches")}
            serving["config"] = sv["config"]
        except Exception as e:  # noqa: BLE001 -- reported in the line, the headline numbers stand
            serving = {"error": str(e)[:300]}
    regressions = None
    if world == 1 and not args.no_serving:
        try:
            regressions = run_regressions_workload(args)
        except Exception as e:  # noqa: BLE001 -- reported in the line, the headline numbers stand
            regressions = {"error": str(e)[:300]}

    if rank == 0:
        out = {"metric": METRIC, "value": value, "unit": "r2 pairs/s", "n_gpus": world, "steps": args.steps,
               "warmup": args.warmup, "ms_per_step": 1e3 * t_max / args.steps, "higher_is_better": True,
               "scaling": "strong" if sharded else "weak", "vs_baseline": None,
               "dtype": "int8 (int32 accumulate, f64 epilogue)",
               "data": "synthetic (seeded founder-mosaic panel generated on the device)",
               "config": config_dict(spec), "e2e": e2e, "gpu_launches": int(launches),
               "roofline": roofline, "cpu_baseline": cpu, "clocks": clocks, "serving": serving,
               "regressions": regressions,
               "int8_vs_oracle_max_rel_per_l2j": parity["int8_vs_oracle_max_rel_per_l2j"] if parity else None,
               "parity": parity,
               "forms": {"int8_pairs_per_s": value / world, "fp64_pairs_per_s": fp64_value,
                         "int8_over_fp64": (value / world) / fp64_value if fp64_value else None,
                         "int8_gram_ms": 1e3 * gram_avg, "fp64_gram_ms": 1e3 * float(np.mean(fp64_gram)),
                         "int8_decode_ms": 1e3 * float(np.mean(dec_s)),
                         "int8_device_ms_per_pass": float(np.mean(dev_ms)),
                         "n_pairs_per_rank": int(rank_pairs),
                         "int8_vs_fp64_l2_max_rel_err": int8_err,
                         "int8_fused_operands": fused}}
        print(json.dumps(out))
    panel.close()
    ctx.close()
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
