"""Benchmark of the l2 LD-score hot path: r^2-pairs/sec on one B200.

Workload (N = 1): the exact biobank-scale configuration -- synthetic panel
N = 50,000 individuals x M = 100,000 SNPs (200 founders, 1% missing, 100 cM),
--ld-wind-cm 1 --snp-level-masking.  One step = one full l2 pass over the
panel (decode + band Gram + r^2 epilogue + l2 back to the host) in the
INT8-exact form.  The plain FP64 form is timed on the same panel for the
INT8-vs-FP64 ratio.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

With --gpus N (launched by torchrun) each rank computes its own chromosome
(an independent 100,000-SNP panel, seed + rank): weak scaling, no collective
on the data path; the time is the max over ranks.  The reference arm
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


def cpu_baseline(body_rows, spec, chr_, cm, bp, n_threads=0):
    """The C restatement of the reference's l2 (OpenMP, all host threads) on
    the first CPU_SAMPLE_SNPS SNPs of the panel, same flags."""
    sys.path.insert(0, ROOT)
    from oracle import OracleL2Args, max_threads, oracle_l2
    m = body_rows.shape[0]
    a = OracleL2Args(bed_body=body_rows, n_file_indiv=spec.n_indiv, chr=chr_[:m], cm=cm[:m], bp=bp[:m],
                     mode="cm", wind=1.0, chunk_c=200, masking=True, per_chr=True, n_threads=n_threads)
    t0 = time.perf_counter()
    _, _, pairs, _ = oracle_l2(a)
    dt = time.perf_counter() - t0
    return pairs / dt, pairs, dt, (n_threads or max_threads())


def run_reference(args):
    """--impl reference: the reference's CPU path (C restatement) on host cores."""
    from ldsc_b200 import synth
    spec = workload_spec()
    chr_, cm, bp = synth.positions(spec)
    rows = synth.bed_body(spec, 0, CPU_SAMPLE_SNPS)
    for _ in range(args.warmup):
        cpu_baseline(rows[:200], spec, chr_, cm, bp)
    vals, tot_pairs, tot_t = [], 0, 0.0
    cores = None
    for _ in range(args.steps):
        v, pairs, dt, cores = cpu_baseline(rows, spec, chr_, cm, bp)
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
                            "sample": sample},
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
    the sketch pass rate, the scatter kernel's HBM roofline, and the error of
    the sketched l2 against exact l2 (INT8 form) on the same panel."""
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
    hbm, _, src = measured_peaks()
    for d in [int(x) for x in args.sketch_d.split(",")]:
        t, outs = _timed_passes(ctx, stream, lambda: run_l2(ctx, snps, panel, wm, 200, snp_level_masking=True,
                                                            sketch=d, yes_really=True), args.warmup, args.steps)
        sk = outs[-1][0][:, 0]
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
               "sketch_kernel_ms": 1e3 * sk_s, "sketch_gram_ms": 1e3 * gram_s, "decode_ms": 1e3 * perf.norm_secs,
               "sketch_roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                                   "frac": achieved / hbm, "algorithmic_bytes": alg_bytes, "peak_source": src},
               "vs_exact": {"pearson_r": float(np.corrcoef(sk, exact)[0, 1]),
                            "max_abs_err": float(np.max(np.abs(sk - exact))),
                            "mean_abs_err": float(np.mean(np.abs(sk - exact))),
                            "mean_exact_l2": float(np.mean(exact))}}
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
    chr_, cm, bp = synth.positions(spec)
    m = spec.m
    snps = BimTable(chr_, [f"rs{i}" for i in range(m)], cm, bp, np.arange(m, dtype=np.int64))
    annot = synth.partitioned_annot(m)
    panel = ctx.synth(spec.n_indiv, m, spec.founders, spec.switch_p, spec.miss, spec.seed)
    wm = WindowMode.Cm(1.0)
    npairs = pair_count(snps, wm, 200)
    res = {}
    for prec in ("int8", "fp64"):
        t, outs = _timed_passes(ctx, stream, lambda: run_l2(ctx, snps, panel, wm, 200, annot=annot,
                                                            precision=prec, yes_really=True),
                                args.warmup if prec == "int8" else 1, args.steps if prec == "int8" else 2)
        res[prec] = (t / (args.steps if prec == "int8" else 2), outs[-1])
    l2i = res["int8"][1][0]
    l2f = res["fp64"][1][0]
    # oracle on the three smallest chromosomes (independent in per-chromosome mode)
    start = int(np.searchsorted(chr_, 20))
    rows = panel.download(start, m)
    ref, _, _, _ = oracle_l2(OracleL2Args(bed_body=rows, n_file_indiv=spec.n_indiv, chr=chr_[start:], cm=cm[start:],
                                          bp=bp[start:], chunk_c=200, annot=annot[start:]))
    scale = np.maximum(np.abs(ref).max(axis=0, keepdims=True), 1.0)
    out = {"workload": "partitioned", "config": {"n_indiv": spec.n_indiv, "n_snp": m, "chromosomes": 22,
                                                 "annotations": annot.shape[1], "window": "1 cM", "chunk_size": 200},
           "metric": "r2 pairs/sec", "n_pairs": npairs,
           "int8": {"pairs_per_s": npairs / res["int8"][0], "ms_per_step": 1e3 * res["int8"][0],
                    "gram_ms": 1e3 * res["int8"][1][2].ab_dot_secs},
           "fp64": {"pairs_per_s": npairs / res["fp64"][0], "ms_per_step": 1e3 * res["fp64"][0],
                    "gram_ms": 1e3 * res["fp64"][1][2].ab_dot_secs},
           "int8_vs_oracle_chr20_22": float(np.max(np.abs(l2i[start:] - ref) / scale)),
           "fp64_vs_oracle_chr20_22": float(np.max(np.abs(l2f[start:] - ref) / scale)),
           "int8_vs_fp64_all": float(np.max(np.abs(l2i - l2f) / np.maximum(np.abs(l2f).max(axis=0, keepdims=True), 1.0))),
           "error_metric": "max |l2_jC - ref_jC| / max(max_j |ref_jC|, 1) per annotation column"}
    print(json.dumps(out), flush=True)
    panel.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=30)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--fp64-steps", type=int, default=2)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--workload", default="biobank", choices=["biobank", "profile", "sketch", "partitioned"])
    ap.add_argument("--sketch-d", default="200,1000,5000")
    ap.add_argument("--sketch-snps", type=int, default=0, help="truncate the sketch panel (profiling)")
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

    spec = workload_spec(seed_offset=rank, workload=args.workload)
    chr_, cm, bp = synth.positions(spec)
    m = spec.m
    snps = BimTable(chr_, [f"rs{i}" for i in range(m)], cm, bp, np.arange(m, dtype=np.int64))
    panel = ctx.synth(spec.n_indiv, m, spec.founders, spec.switch_p, spec.miss, spec.seed)
    wm = WindowMode.Cm(1.0)
    npairs = pair_count(snps, wm, 200, snp_level_masking=True)

    def step(precision):
        return run_l2(ctx, snps, panel, wm, 200, snp_level_masking=True, precision=precision, yes_really=True)

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
        _, _, perf = step("int8")
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
    if world > 1:
        tt = torch.tensor([t_local], device="cuda", dtype=torch.float64)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        pp = torch.tensor([npairs], device="cuda", dtype=torch.float64)
        dist.all_reduce(pp, op=dist.ReduceOp.SUM)
        t_max, pairs_all = float(tt.item()), float(pp.item())
    value = pairs_all * args.steps / t_max
    gram_avg = float(np.mean(gram_s))

    # ---- FP64 plain form, same panel ----
    fp64_value, fp64_gram = None, [float("nan")]
    if args.fp64_steps > 0:
        step("fp64")
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
        fp64_value = npairs * args.fp64_steps / t64

    # ---- end to end through the whole-file C ABI entry point, host buffers ----
    e2e = None
    if not args.no_e2e:
        rows = panel.download()
        bed = torch.empty(3 + rows.size, dtype=torch.uint8, pin_memory=True)
        bnp = bed.numpy()
        bnp[:3] = [0x6C, 0x1B, 0x01]
        bnp[3:] = rows.reshape(-1)
        del rows
        for _ in range(1):
            l2_from_bed_bytes(ctx, bnp, spec.n_indiv, snps, wm, 200, precision="int8", snp_level_masking=True)
        barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        e2e_perf = []
        for _ in range(args.steps):
            e2e_perf.append(l2_from_bed_bytes(ctx, bnp, spec.n_indiv, snps, wm, 200, precision="int8",
                                              snp_level_masking=True)[2])
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
    ops = 8.0 * spec.n_indiv * npairs   # 4 integer products x 2 ops x N per in-band pair
    achieved = ops / gram_avg / 1e12
    roofline = {"bound": "tensor", "achieved": achieved, "peak": int8_peak, "unit": "TFLOP/s",
                "frac": achieved / int8_peak, "traffic": committed_traffic("k_gram_i8"),
                "kernel": "k_gram_i8 (tcgen05.mma kind::i8)",
                "note": f"int8 ops counted like flops (2 per MAC, 4 products per pair); peak = 2 x {src} "
                        "bf16 dense burst (MEASURED_PEAKS.json), nominal int8 dense 4500"}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        rows = panel.download(0, CPU_SAMPLE_SNPS)
        v, pairs_s, dt, cores = cpu_baseline(rows, spec, chr_, cm, bp)
        cpu = {"value": v, "unit": "r2 pairs/s", "cores": cores, "kind": "port",
               "sample": f"first {CPU_SAMPLE_SNPS} SNPs of the panel ({pairs_s} pairs, {dt:.1f} s), same flags, f64"}

    if rank == 0:
        out = {"metric": METRIC, "value": value, "unit": "r2 pairs/s", "n_gpus": world, "steps": args.steps,
               "warmup": args.warmup, "ms_per_step": 1e3 * t_max / args.steps, "higher_is_better": True,
               "scaling": "weak", "vs_baseline": None, "dtype": "int8 (int32 accumulate, f64 epilogue)",
               "data": "synthetic (seeded founder-mosaic panel generated on the device)",
               "config": config_dict(spec), "e2e": e2e, "gpu_launches": int(launches),
               "roofline": roofline, "cpu_baseline": cpu, "clocks": clocks,
               "forms": {"int8_pairs_per_s": value / world, "fp64_pairs_per_s": fp64_value,
                         "int8_over_fp64": (value / world) / fp64_value if fp64_value else None,
                         "int8_gram_ms": 1e3 * gram_avg, "fp64_gram_ms": 1e3 * float(np.mean(fp64_gram)),
                         "int8_decode_ms": 1e3 * float(np.mean(dec_s)),
                         "int8_device_ms_per_pass": float(np.mean(dev_ms)),
                         "n_pairs_per_rank": npairs}}
        print(json.dumps(out))
    panel.close()
    ctx.close()
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
