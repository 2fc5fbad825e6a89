"""`l2` command line: the reference's `ldsc l2` (src/cli.rs:170-355,
src/l2/mod.rs:46-805) on the B200 engine.

    python -m ldsc_b200 l2 --bfile PREFIX --out PREFIX [--ld-wind-cm 1] ...

Same flags, same order of filters (--extract, --annot, --keep, the --maf /
--pq-exp prefilter, pq-scaled annotations), same outputs and messages.  The
GPU-only flags of the reference (--gpu, --gpu-tile-cols, --gpu-flex32,
--gpu-f64) are accepted and ignored: the engine always runs on the GPU, and
--gpu-precision picks its arithmetic (int8 exact, the default, or fp64).
--cts-bin builds annotations (the cts-annot tool) and is not part of this
engine.
"""
from __future__ import annotations

import argparse
import os
import sys
import time
from typing import List, Optional

import numpy as np

from . import io as lio
from .api import Context, LdscError, WindowMode, run_l2, snp_stats
from .sliced import call_bytes_per_record, run_l2_sliced
from .plink import BimTable, count_fam, parse_bim, parse_fam_text, read_bed


def build_parser() -> argparse.ArgumentParser:
    ap = argparse.ArgumentParser(prog="ldsc_b200 l2", description="LD scores on a B200 (ldsc l2)")
    ap.add_argument("--bfile", required=True)
    ap.add_argument("--out", required=True)
    ap.add_argument("--ld-wind-cm", type=float)
    ap.add_argument("--ld-wind-kb", type=float)
    ap.add_argument("--ld-wind-snps", type=int)
    ap.add_argument("--annot")
    ap.add_argument("--cts-bin")
    ap.add_argument("--cts-breaks")
    ap.add_argument("--cts-names")
    ap.add_argument("--thin-annot", action="store_true")
    ap.add_argument("--extract")
    ap.add_argument("--maf", type=float)
    ap.add_argument("--maf-pre", type=lambda s: s.lower() not in ("0", "false", "no"), default=True)
    ap.add_argument("--mmap", action="store_true")
    ap.add_argument("--global-pass", action="store_true")
    ap.add_argument("--snp-level-masking", action="store_true")
    ap.add_argument("--print-snps")
    ap.add_argument("--keep")
    ap.add_argument("--per-allele", action="store_true")
    ap.add_argument("--pq-exp", type=float)
    ap.add_argument("--no-print-annot", action="store_true")
    ap.add_argument("--chunk-size", type=int, default=200)
    ap.add_argument("--python-compat", action="store_true")
    ap.add_argument("--yes-really", action="store_true")
    ap.add_argument("--gpu", action="store_true")
    ap.add_argument("--gpu-tile-cols", type=int)
    ap.add_argument("--gpu-flex32", action="store_true")
    ap.add_argument("--gpu-f64", action="store_true")
    ap.add_argument("--fast-f32", action="store_true")
    ap.add_argument("--sketch", type=int, metavar="DIM")
    ap.add_argument("--sketch-maf-aware", action="store_true")
    ap.add_argument("--verbose-timing", action="store_true")
    ap.add_argument("--gpu-precision", choices=["int8", "fp64"], default="int8",
                    help="arithmetic of the exact form (engine flag; int8 is exact)")
    ap.add_argument("--device", type=int, default=0)
    ap.add_argument("--max-device-gb", type=float,
                    help="device memory for the panel and workspace (engine flag); a larger panel runs in "
                         "SNP slices.  Default: the free device memory less 4 GB, used only when needed")
    return ap


def _slice_budget(args, snps: BimTable, n_indiv: int, mode: WindowMode, chunk_c: int, annot, iid,
                  global_pass: bool) -> Optional[int]:
    """Device bytes for a sliced run, or None when the whole panel fits."""
    per = call_bytes_per_record(snps, n_indiv, mode, chunk_c, annot=annot, iid_indices=iid,
                                precision=args.gpu_precision, sketch=args.sketch,
                                snp_level_masking=args.snp_level_masking, global_pass=global_pass)
    need = per * len(snps)
    if args.max_device_gb is not None:
        budget = int(args.max_device_gb * 1e9)
        return budget if need > budget else None
    import torch
    free = torch.cuda.mem_get_info(args.device)[0] - (4 << 30)
    return int(free) if need > free else None


def _snp_stats_sliced(ctx: Context, snps: BimTable, body: np.ndarray, n_indiv: int, iid, budget: int):
    """compute_snp_stats on row slices of the panel (per-record, no halos)."""
    bpr = (n_indiv + 3) // 4
    rows = max(1, int(budget // max(bpr + 64, 1)))
    bed_idx = np.asarray(snps.bed_idx, dtype=np.int64)
    maf = np.zeros(len(snps))
    ok = np.zeros(len(snps), dtype=bool)
    rb = np.asarray(body).reshape(-1, bpr)
    a = 0
    while a < len(snps):
        b = int(np.searchsorted(bed_idx, bed_idx[a] + rows, side="left"))
        b = max(b, a + 1)
        r0, r1 = int(bed_idx[a]), int(bed_idx[b - 1]) + 1
        sub = snps.subset(np.arange(a, b))
        sub = BimTable(sub.chr, sub.snp, sub.cm, sub.bp, np.asarray(sub.bed_idx, dtype=np.int64) - r0)
        panel = ctx.upload(rb[r0:r1], n_indiv)
        try:
            maf[a:b], ok[a:b] = snp_stats(ctx, sub, panel, iid)
        finally:
            panel.close()
        a = b
    return maf, ok


def run(args, ctx: Optional[Context] = None) -> None:
    """l2::run (src/l2/mod.rs:46-805)."""
    # ---- flag checks (src/l2/mod.rs:55-97) ----
    if args.per_allele and args.pq_exp is not None:
        raise ValueError("Cannot set both --per-allele and --pq-exp (--per-allele is equivalent to --pq-exp 1).")
    if args.annot and args.cts_bin:
        raise ValueError("--annot and --cts-bin are currently incompatible.")
    if args.cts_bin:
        raise ValueError("--cts-bin builds annotations (cts-annot) and is not part of this engine; "
                         "build the .annot file first and pass --annot")
    if args.python_compat and args.snp_level_masking:
        raise ValueError("--python-compat is incompatible with --snp-level-masking")
    if args.sketch_maf_aware and args.sketch is None:
        raise ValueError("--sketch-maf-aware requires --sketch")
    pq_exp = 1.0 if args.per_allele else args.pq_exp
    n_wind = sum(x is not None for x in (args.ld_wind_cm, args.ld_wind_kb, args.ld_wind_snps))
    if n_wind > 1:
        raise ValueError("Must specify exactly one --ld-wind option")
    if args.ld_wind_kb is not None:
        mode = WindowMode.Kb(args.ld_wind_kb)
    elif args.ld_wind_snps is not None:
        mode = WindowMode.Snp(args.ld_wind_snps)
    else:
        mode = WindowMode.Cm(args.ld_wind_cm if args.ld_wind_cm is not None else 1.0)

    t_run0 = time.perf_counter()
    bim_path, fam_path, bed_path = args.bfile + ".bim", args.bfile + ".fam", args.bfile + ".bed"
    snps_raw = parse_bim(bim_path)
    n_indiv = count_fam(fam_path)
    print(f"Loaded {len(snps_raw)} SNPs, {n_indiv} individuals from '{args.bfile}'")

    snps = snps_raw
    if args.extract:
        keep_set = lio.load_snp_set(args.extract)
        rows = [i for i, s in enumerate(snps_raw.snp) if s in keep_set]
        snps = snps_raw.subset(rows)
        print(f"  After --extract: {len(snps)} SNPs")
    print_set = lio.load_print_snps(args.print_snps) if args.print_snps else None
    if args.annot and args.extract:
        print("WARNING: --annot with --extract is not supported. "
              "Ensure your annot files match the extracted SNP set.")

    annot, annot_names = None, None
    if args.annot:
        prefix = args.annot
        explicit = prefix.endswith((".annot", ".annot.gz", ".annot.bz2"))
        path = None
        if explicit:
            path = lio.resolve_annot_path(prefix)
        else:
            try:
                path = lio.resolve_annot_path(prefix)
            except FileNotFoundError:
                path = None
        if path is not None:
            annot, annot_names = lio.read_annot_path(path, args.thin_annot)
            where = path
        else:
            # per-chromosome files prefix{chr}.annot[.gz|.bz2], chromosomes in sorted order
            mats = []
            for c in sorted(set(int(x) for x in snps.chr)):
                m_c, names = lio.read_annot_path(lio.resolve_annot_path(f"{prefix}{c}"), args.thin_annot)
                annot_names = annot_names or names
                mats.append(m_c)
            annot = np.asfortranarray(np.concatenate(mats, axis=0))
            where = prefix + "*"
        if annot.shape[0] != len(snps):
            raise ValueError(f"Annotation file has {annot.shape[0]} rows but BIM has {len(snps)} SNPs "
                             "— they must match exactly")
        print(f"Read {len(annot_names)} annotations for {annot.shape[0]} SNPs from '{where}'")

    iid = None
    if args.keep:
        with open(fam_path) as f:
            fam_ids = parse_fam_text(f.read())
        iid = lio.load_individual_indices(args.keep, fam_ids)
    n_used = len(iid) if iid is not None else n_indiv

    # ---- the panel: resident for the prefilter and the compute, or, when it
    # does not fit the device budget, uploaded slice by slice ----
    own_ctx = ctx is None
    ctx = ctx or Context(args.device)
    chunk_c = 50 if args.python_compat else args.chunk_size
    global_pass = args.global_pass or args.python_compat
    t_bed0 = time.perf_counter()
    budget = _slice_budget(args, snps, n_indiv, mode, chunk_c, annot, iid, global_pass)
    body = read_bed(bed_path, n_indiv, len(snps_raw), mmap=budget is not None or args.mmap)
    panel = None if budget is not None else ctx.upload(body, n_indiv)
    t_bed = time.perf_counter() - t_bed0
    try:
        # ---- --maf / --pq-exp prefilter (src/l2/mod.rs:265-333) ----
        maf_pre_vals = None
        if args.maf_pre and (args.maf is not None or pq_exp is not None):
            if panel is None:
                maf_all, ok = _snp_stats_sliced(ctx, snps, body, n_indiv, iid, budget)
            else:
                maf_all, ok = snp_stats(ctx, snps, panel, iid)
            thr = args.maf if args.maf is not None else 0.0
            keep_mask = ok & (maf_all > thr)
            if not keep_mask.any():
                raise ValueError("SNP prefilter removed all SNPs")
            if not keep_mask.all():
                rows = np.nonzero(keep_mask)[0]
                snps = snps.subset(rows)
                if annot is not None:
                    annot = np.asfortranarray(annot[rows])
            if args.maf is not None:
                print(f"--maf-pre: kept {len(snps)} / {len(keep_mask)} SNPs (MAF > {lio.rust_f64(thr)})")
            maf_pre_vals = maf_all[keep_mask]
        pq_scaled = False
        if pq_exp is not None and maf_pre_vals is not None and annot is not None:
            annot = np.asfortranarray(annot * ((maf_pre_vals * (1.0 - maf_pre_vals)) ** pq_exp)[:, None])
            pq_scaled = True
        pq_for_compute = None if pq_scaled else pq_exp

        if args.python_compat:
            if args.chunk_size != 200:
                print(f"--python-compat overrides --chunk-size {args.chunk_size} with c=50 for Python LDSC parity",
                      file=sys.stderr)
            if not args.global_pass:
                print("--python-compat auto-enables --global-pass for Python LDSC parity", file=sys.stderr)
        if args.sketch is not None and not args.fast_f32:
            print("  --sketch auto-enables f32 (bit-identical to f64, ~1.3× faster)")
        if args.verbose_timing:
            print(f"[perf] maf_prefilter={time.perf_counter() - t_run0 - t_bed:.3f}s", file=sys.stderr)

        t_c0 = time.perf_counter()
        if panel is None:
            l2, maf, slices, perfs = run_l2_sliced(
                ctx, snps, body, n_indiv, mode, chunk_c, device_budget_bytes=budget, annot=annot,
                iid_indices=iid, pq_exp=pq_for_compute, sketch=args.sketch,
                sketch_maf_aware=args.sketch_maf_aware, snp_level_masking=args.snp_level_masking,
                global_pass=global_pass, precision=args.gpu_precision, use_f32=args.fast_f32)
            print(f"  panel larger than the device budget ({budget / 1e9:.1f} GB): computed in "
                  f"{len(slices)} SNP slices", file=sys.stderr)
            perf = perfs[-1]
        else:
            l2, maf, perf = run_l2(ctx, snps, panel, mode, chunk_c, annot=annot, iid_indices=iid,
                                   pq_exp=pq_for_compute, yes_really=args.yes_really, use_f32=args.fast_f32,
                                   sketch=args.sketch, sketch_maf_aware=args.sketch_maf_aware,
                                   snp_level_masking=args.snp_level_masking, global_pass=global_pass,
                                   precision=args.gpu_precision)
        if args.verbose_timing:
            print(f"[perf] bed_read={t_bed:.3f}s norm={perf.norm_secs:.3f}s "
                  f"ab_dot={perf.ab_dot_secs:.3f}s device={perf.device_ms / 1e3:.3f}s "
                  f"pairs={perf.n_pairs}", file=sys.stderr)
            print(f"[perf] compute_ldscore_total={time.perf_counter() - t_c0:.3f}s", file=sys.stderr)
    finally:
        if panel is not None:
            panel.close()
        if own_ctx:
            ctx.close()

    # ---- outputs (src/l2/mod.rs:584-805) ----
    t_w0 = time.perf_counter()
    suffix = f"_S{lio.rust_f64(pq_exp)}" if pq_exp is not None else ""
    col_names = [f"L2{suffix}"] if annot is None else [f"{n}L2{suffix}" for n in annot_names]
    pq_per_snp = None if pq_exp is None else (maf * (1.0 - maf)) ** pq_exp
    pq_for_m = None if pq_scaled else pq_per_snp
    m = len(snps)

    def should_output(i):
        ok = True
        if args.maf is not None:
            ok = maf[i] > args.maf
        if print_set is not None:
            ok = ok and snps.snp[i] in print_set
        return ok

    out_rows = np.array([i for i in range(m) if should_output(i)], dtype=np.int64)
    if print_set is not None and out_rows.size == 0:
        raise ValueError("After merging with --print-snps, no SNPs remain.")

    def m_vals(rows: np.ndarray):
        if annot is not None:
            base = annot[rows] if pq_for_m is None else annot[rows] * pq_for_m[rows][:, None]
            big = maf[rows] > 0.05
            return list(base.sum(axis=0)), list(base[big].sum(axis=0))
        if pq_per_snp is not None:
            return [float(pq_per_snp[rows].sum())], [float(pq_per_snp[rows][maf[rows] > 0.05].sum())]
        return [float(len(rows))], [float((maf[rows] > 0.05).sum())]

    out_path = f"{args.out}.l2.ldscore.gz"
    lio.write_ldscore(out_path, snps, out_rows, l2[out_rows], col_names)
    all_rows = np.arange(m)
    mv, m550 = m_vals(all_rows)
    with open(f"{args.out}.l2.M", "w") as f:
        f.write(lio.format_m_vals(mv))
    with open(f"{args.out}.l2.M_5_50", "w") as f:
        f.write(lio.format_m_vals(m550))
    for c in sorted(set(int(x) for x in snps.chr)):
        rows_all = np.nonzero(snps.chr == c)[0]
        rows_out = np.array([i for i in rows_all if should_output(i)], dtype=np.int64)
        cpath = f"{args.out}{c}.l2.ldscore.gz"
        lio.write_ldscore(cpath, snps, rows_out, l2[rows_out], col_names)
        mvc, m550c = m_vals(rows_all)
        with open(f"{args.out}{c}.l2.M", "w") as f:
            f.write(lio.format_m_vals(mvc))
        with open(f"{args.out}{c}.l2.M_5_50", "w") as f:
            f.write(lio.format_m_vals(m550c))
        print(f"chr {c}: {len(rows_out)} SNPs → {cpath} (M={','.join(lio.rust_f64(v) for v in mvc)}, "
              f"M_5_50={','.join(lio.rust_f64(v) for v in m550c)})")
    lio.print_ld_score_summary(out_path, maf[out_rows], l2[out_rows], col_names)
    if args.verbose_timing:
        print(f"[perf] write_outputs={time.perf_counter() - t_w0:.3f}s total={time.perf_counter() - t_run0:.3f}s",
              file=sys.stderr)


def main(argv: Optional[List[str]] = None) -> int:
    argv = list(sys.argv[1:] if argv is None else argv)
    if not argv or argv[0] != "l2":
        print("usage: python -m ldsc_b200 l2 --bfile PREFIX --out PREFIX [options]", file=sys.stderr)
        return 2
    args = build_parser().parse_args(argv[1:])
    try:
        run(args)
    except (LdscError, ValueError, FileNotFoundError) as e:
        print(f"Error: {e}", file=sys.stderr)
        return 1
    return 0
