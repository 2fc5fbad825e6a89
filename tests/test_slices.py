"""Record ranges for slices and ranks (ldsc_b200.parallel), CPU only.

The property every split rests on: a call over [call_lo, call_hi) gives each
record j >= core_lo of the call the same left limit as the whole run
(src/l2/compute.rs:1164-1184, 1855-1867), so every pair touching a core
record is accumulated exactly as in the whole run.  Checked with the host
planner on each call's records, and end to end with the C oracle: l2 stitched
from the slices' core rows equals one oracle run.
"""
import numpy as np
import pytest

MODES = [  # (snp_level_masking, global_pass)
    (False, False), (False, True), (True, False), (True, True)]


def _panel(seed=61):
    from ldsc_b200 import synth
    spec = synth.PanelSpec(n_indiv=300, chrom_sizes=[900, 500, 700], chrom_cm=[6.0, 3.0, 5.0], founders=25,
                           miss=0.02, seed=seed)
    chr_, cm, bp = synth.positions(spec)
    return spec, synth.bed_body(spec), chr_, cm, bp


def _snps(chr_, cm, bp):
    from ldsc_b200.plink import BimTable
    m = len(chr_)
    return BimTable(chr_, [f"rs{i}" for i in range(m)], cm, bp, np.arange(m, dtype=np.int64))


@pytest.mark.parametrize("masking,global_pass", MODES)
@pytest.mark.parametrize("budget", [550, 800, 1500])
def test_call_ranges_keep_the_left_limits(masking, global_pass, budget):
    from ldsc_b200.api import WindowMode, left_limits
    from ldsc_b200.parallel import plan_slices
    spec, _, chr_, cm, bp = _panel()
    snps = _snps(chr_, cm, bp)
    mode = WindowMode.Cm(1.0)
    left = left_limits(snps, mode, 100, snp_level_masking=masking, global_pass=global_pass)
    assert np.all(np.diff(left) >= 0)                     # non-decreasing, as the split assumes
    sl = plan_slices(snps, mode, budget, 100, masking, global_pass)
    assert sl[0].core_lo == 0 and sl[-1].core_hi == len(snps)
    assert all(a.core_hi == b.core_lo for a, b in zip(sl[:-1], sl[1:]))
    for s in sl:
        assert s.call_hi - s.call_lo <= budget
        assert s.call_lo <= s.core_lo < s.core_hi <= s.call_hi
        sub = snps.subset(np.arange(s.call_lo, s.call_hi))
        ls = left_limits(sub, mode, 100, snp_level_masking=masking, global_pass=global_pass) + s.call_lo
        j = np.arange(s.core_lo, s.call_hi)
        np.testing.assert_array_equal(ls[j - s.call_lo], left[j])
        # every record after the core that pairs with a core record is in the call
        if s.call_hi < len(snps):
            assert left[s.call_hi] >= s.core_hi


def test_budget_smaller_than_a_window_is_an_error():
    from ldsc_b200.api import WindowMode
    from ldsc_b200.parallel import plan_slices
    spec, _, chr_, cm, bp = _panel()
    with pytest.raises(ValueError):
        plan_slices(_snps(chr_, cm, bp), WindowMode.Cm(1.0), 50, 100)


@pytest.mark.parametrize("masking,global_pass", MODES)
def test_stitched_slices_equal_one_run(masking, global_pass):
    from ldsc_b200.api import WindowMode
    from ldsc_b200.parallel import plan_slices
    from oracle import OracleL2Args, oracle_l2
    spec, body, chr_, cm, bp = _panel()
    snps = _snps(chr_, cm, bp)
    rng = np.random.default_rng(5)
    annot = np.stack([np.ones(len(snps)), rng.integers(0, 2, len(snps)).astype(float)], axis=1)

    def run(rows):
        l2, maf, _, _ = oracle_l2(OracleL2Args(bed_body=body, n_file_indiv=spec.n_indiv, chr=chr_[rows],
                                               cm=cm[rows], bp=bp[rows], bed_idx=rows, chunk_c=100,
                                               masking=masking, per_chr=not global_pass, annot=annot[rows],
                                               n_threads=1))
        return l2, maf

    full, maf_full = run(np.arange(len(snps)))
    sl = plan_slices(snps, WindowMode.Cm(1.0), 600, 100, masking, global_pass)
    assert len(sl) >= 3
    got = np.zeros_like(full)
    maf = np.zeros_like(maf_full)
    for s in sl:
        l2, mf = run(np.arange(s.call_lo, s.call_hi))
        got[s.core_lo:s.core_hi] = l2[s.core_lo - s.call_lo: s.core_hi - s.call_lo]
        maf[s.core_lo:s.core_hi] = mf[s.core_lo - s.call_lo: s.core_hi - s.call_lo]
    np.testing.assert_allclose(got, full, rtol=1e-10, atol=1e-12)
    np.testing.assert_array_equal(maf, maf_full)


def test_shards_cut_inside_chromosomes_with_aligned_halos():
    from ldsc_b200.api import WindowMode
    from ldsc_b200.parallel import chunk_origin, plan_shards
    spec, _, chr_, cm, bp = _panel()
    snps = _snps(chr_, cm, bp)
    for global_pass in (False, True):
        plan = plan_shards(snps, WindowMode.Cm(1.0), 3, 100, global_pass=global_pass)
        origin = chunk_origin(snps, global_pass)
        assert plan[0].core_lo == 0 and plan[-1].core_hi == len(snps)
        for s in plan:
            assert (s.call_lo - origin[s.call_lo]) % 100 == 0     # halo starts on the chunk grid
        loads = [s.pairs for s in plan]
        assert max(loads) < 1.5 * min(loads)
