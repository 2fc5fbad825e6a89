"""Sharded l2 over two ranks (gloo, CPU).  The compute step is the C oracle
standing in for each rank's GPU call; what is tested is the plan (cores
balanced by pair count, halos from the left limits, aligned to the chunk grid
without per-SNP windows) and the tensor all-gather of the core rows, against
one unsharded oracle run.
src/l2/mod.rs:477-553 (chromosomes are independent),
src/l2/compute.rs:1164-1184 (chunk windows), 1855-1867 (per-SNP windows)."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp


def _panel():
    from ldsc_b200 import synth
    spec = synth.PanelSpec(n_indiv=300, chrom_sizes=[900, 500, 700], chrom_cm=[6.0, 3.0, 5.0], founders=25,
                           miss=0.02, seed=61)
    chr_, cm, bp = synth.positions(spec)
    return spec, synth.bed_body(spec), chr_, cm, bp


def _worker(rank, world, port, masking, result_path):
    import torch.distributed as dist
    from ldsc_b200.api import WindowMode
    from ldsc_b200.parallel import plan_shards, run_sharded
    from ldsc_b200.plink import BimTable
    from oracle import OracleL2Args, oracle_l2
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        spec, body, chr_, cm, bp = _panel()
        m = spec.m
        snps = BimTable(chr_, [f"rs{i}" for i in range(m)], cm, bp, np.arange(m, dtype=np.int64))
        plan = plan_shards(snps, WindowMode.Cm(1.0), world, 200, snp_level_masking=masking)

        def compute(rec):
            l2, _, _, _ = oracle_l2(OracleL2Args(bed_body=body, n_file_indiv=spec.n_indiv, chr=rec.chr, cm=rec.cm,
                                                 bp=rec.bp, bed_idx=rec.bed_idx, chunk_c=200, masking=masking,
                                                 n_threads=1))
            return l2

        out = run_sharded(compute, snps, plan, rank)
        # the gather also takes torch tensors, and every rank can receive the result
        import torch
        every = run_sharded(lambda rec: torch.from_numpy(compute(rec)), snps, plan, rank, dst=None)
        np.testing.assert_array_equal(every, out if rank == 0 else every)
        if rank == 1:
            np.save(result_path + ".rank1.npy", every)
        if rank == 0:
            np.save(result_path, out)
            np.save(result_path + ".plan.npy", np.array([[s.core_lo, s.core_hi, s.call_lo, s.call_hi] for s in plan]))
    finally:
        dist.destroy_process_group()


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


@pytest.mark.parametrize("masking", [False, True])
def test_two_ranks_equal_one_run(tmp_path, masking):
    from oracle import OracleL2Args, oracle_l2
    res = str(tmp_path / "l2.npy")
    mp.spawn(_worker, args=(2, _free_port(), masking, res), nprocs=2, join=True)
    got = np.load(res)
    plan = np.load(res + ".plan.npy")
    np.testing.assert_array_equal(np.load(res + ".rank1.npy"), got)
    spec, body, chr_, cm, bp = _panel()
    ref, _, _, _ = oracle_l2(OracleL2Args(bed_body=body, n_file_indiv=spec.n_indiv, chr=chr_, cm=cm, bp=bp,
                                          chunk_c=200, masking=masking))
    np.testing.assert_allclose(got, ref, rtol=1e-10, atol=1e-12)
    assert plan[0, 1] == plan[1, 0] and plan[1, 1] == spec.m     # cores tile the records
    assert 0 < plan[0, 1] < spec.m and plan[0, 1] not in (900, 1400)   # cut inside a chromosome
    assert plan[1, 2] < plan[1, 0]                                # the second rank needs a left halo
    if not masking:
        assert (plan[1, 2] - 900) % 200 == 0                      # on chromosome 2's chunk grid


def test_global_pass_splits_on_the_global_grid():
    from ldsc_b200.api import WindowMode
    from ldsc_b200.parallel import plan_shards
    from ldsc_b200.plink import BimTable
    spec, body, chr_, cm, bp = _panel()
    snps = BimTable(chr_, [f"rs{i}" for i in range(spec.m)], cm, bp, np.arange(spec.m, dtype=np.int64))
    plan = plan_shards(snps, WindowMode.Cm(1.0), 2, global_pass=True)
    assert plan[0].core_hi == plan[1].core_lo and 0 < plan[1].core_lo < spec.m
    assert plan[1].call_lo % 200 == 0 and plan[1].call_lo < plan[1].core_lo
