"""The serving loop: jobs of uneven size run concurrently on one resident
panel, and each job's result equals the same job run alone.

Tolerance: none.  Every pipeline sums in an order fixed by the data alone
(l2: per-tile sums added by a fixed-order reduction; regressions: block
sums in order), so each result is bit-identical alone and in the mix."""
import numpy as np
import pytest

from ldsc_b200 import synth
from ldsc_b200.plink import BimTable

pytestmark = pytest.mark.gpu

def relerr(a, b):
    return float(np.max(np.abs(a - b) / np.maximum(np.abs(b), 1.0)))


@pytest.fixture(scope="module")
def resident(ctx):
    """3 chromosomes, 4,000 individuals, 60,000 SNPs, 300 cM."""
    spec = synth.PanelSpec(n_indiv=4000, chrom_sizes=[30000, 20000, 10000], chrom_cm=[150.0, 100.0, 50.0],
                           founders=60, miss=0.01, seed=41)
    chr_, cm, bp = synth.positions(spec)
    panel = ctx.synth(spec.n_indiv, spec.m, spec.founders, spec.switch_p, spec.miss, spec.seed)
    snps = BimTable(chr_, [f"rs{i}" for i in range(spec.m)], cm, bp, np.arange(spec.m, dtype=np.int64))
    return spec, panel, snps


def _region(snps, b, e):
    return BimTable(snps.chr[b:e], snps.snp[b:e], snps.cm[b:e], snps.bp[b:e], np.arange(b, e, dtype=np.int64))


def test_jobs_alone_equal_jobs_in_the_mix(ctx, resident):
    import torch
    from ldsc_b200.api import WindowMode, h2_batch, rg_batch, run_l2
    from ldsc_b200.serve import Server
    spec, panel, snps = resident
    wm = WindowMode.Cm(1.0)
    m = spec.m
    annot = synth.partitioned_annot(m, seed=5, n_binary=6, n_cont=3)         # 10 columns
    d_annot = torch.from_numpy(np.ascontiguousarray(annot.T)).cuda()   # column c of SNP r at c * m + r
    # LD-score store and summary statistics for the regressions
    l2_all, _, _ = run_l2(ctx, snps, panel, wm, 200, snp_level_masking=True, precision="int8", yes_really=True)
    ld = l2_all[:, 0].copy()
    chi2, n_t, _ = synth.gwas_traits(ld, 1e6, 24, seed=6)
    z1, z2, n1, n2, _ = synth.gwas_pairs(ld, 1e6, 6, seed=7)
    # K = 10 LD scores for partitioned h2, in the l2 run's (K, n_snp) device layout
    l2k, _, _ = run_l2(ctx, snps, panel, wm, 200, annot=annot, snp_level_masking=True, precision="int8",
                       yes_really=True)
    m_vec = annot.sum(axis=0)
    from ldsc_b200.partitioned import default_chisq_max, h2_partitioned
    cmax = np.array([default_chisq_max(chi2[t], n_t[t]) for t in range(len(n_t))])
    dev = {k: torch.from_numpy(np.ascontiguousarray(v, dtype=np.float64)).cuda()
           for k, v in dict(chi2=chi2, n=n_t, ld=ld, z1=z1, z2=z2, n1=n1, n2=n2, l2k=l2k.T).items()}
    jobs = [
        ("l2", dict(b=0, e=9000, K=1, sk=None, prec="int8")),
        ("l2", dict(b=5000, e=35000, K=10, sk=None, prec="int8")),
        ("h2", dict(t0=0, t1=16)),
        ("l2", dict(b=31000, e=33000, K=1, sk=200, prec=None)),
        ("rg", dict(p0=0, p1=6)),
        ("l2", dict(b=40000, e=60000, K=3, sk=None, prec="fp64")),
        ("h2", dict(t0=16, t1=24)),
        ("l2", dict(b=12000, e=52000, K=1, sk=None, prec="int8")),
        ("l2", dict(b=100, e=2100, K=10, sk=None, prec="int8")),
        ("h2p", dict(t0=0, t1=4)),
        ("h2p", dict(t0=4, t1=12)),
    ]

    def alone(kind, p):
        if kind == "l2":
            reg = _region(snps, p["b"], p["e"])
            A = annot[p["b"]:p["e"], :p["K"]] if p["K"] > 1 else None
            return run_l2(ctx, reg, panel, wm, 200, annot=A, sketch=p["sk"], precision=p["prec"] or "fp64",
                          snp_level_masking=True, yes_really=True)[0]
        if kind == "h2":
            return h2_batch(ctx, chi2[p["t0"]:p["t1"]], n_t[p["t0"]:p["t1"]], ld, ld, 1e6, 200)
        if kind == "h2p":
            return h2_partitioned(ctx, chi2[p["t0"]:p["t1"]], n_t[p["t0"]:p["t1"]], l2k, ld, m_vec, 200)
        return rg_batch(ctx, z1[p["p0"]:p["p1"]], z2[p["p0"]:p["p1"]], n1[p["p0"]:p["p1"]],
                        n2[p["p0"]:p["p1"]], ld, ld, 1e6, 200)

    ref = [alone(k, p) for k, p in jobs]
    with Server(0, n_slots=4) as srv:
        tickets = []
        for rep in range(2):
            for kind, p in jobs:
                if kind == "l2":
                    reg = _region(snps, p["b"], p["e"])
                    ad = None
                    A = None
                    if p["K"] == 10:   # resident annotations, read in place
                        ad = (d_annot.data_ptr() + 8 * p["b"], m, 10)
                    elif p["K"] > 1:
                        A = annot[p["b"]:p["e"], :p["K"]]
                    t = srv.submit_l2(panel, reg, wm, 200, row_begin=p["b"], annot=A, annot_device=ad,
                                      sketch=p["sk"], precision=p["prec"] or "fp64", snp_level_masking=True)
                elif kind == "h2":
                    t = srv.submit_h2(dev["chi2"][p["t0"]:p["t1"]], dev["n"][p["t0"]:p["t1"]], dev["ld"],
                                      dev["ld"], 1e6, 200)
                elif kind == "h2p":
                    t = srv.submit_h2_partitioned(dev["chi2"][p["t0"]:p["t1"]], dev["n"][p["t0"]:p["t1"]],
                                                  dev["l2k"], dev["ld"], m_vec, cmax[p["t0"]:p["t1"]], 200)
                else:
                    t = srv.submit_rg(dev["z1"][p["p0"]:p["p1"]], dev["z2"][p["p0"]:p["p1"]],
                                      dev["n1"][p["p0"]:p["p1"]], dev["n2"][p["p0"]:p["p1"]], dev["ld"],
                                      dev["ld"], 1e6, 200)
                tickets.append((kind, t))
        slots = set()
        for i, (kind, t) in enumerate(tickets):
            got, timing = srv.wait(t)
            slots.add(timing.slot)
            want = ref[i % len(jobs)]
            if kind == "l2":
                np.testing.assert_array_equal(got[0], want, err_msg=str((i, jobs[i % len(jobs)])))
            elif kind == "h2p":
                for a, b in zip(got, want):
                    np.testing.assert_array_equal(a.est, b.est)
                    np.testing.assert_array_equal(a.cov, b.cov)
                    assert a.h2_total == b.h2_total
            else:
                for f in got.dtype.names:
                    np.testing.assert_array_equal(got[f], want[f])
        st = srv.stats()
        assert st["completed"] == len(tickets) and len(slots) > 1
        assert st["graph_launches"] > 0   # the regression pipelines replayed as graphs


def test_prewarm_runs_the_job_on_every_slot(ctx, resident):
    """ldsc_server_prewarm runs one job on each slot in turn (so every slot's
    workspace is sized for it before serving starts); its output is the job's
    own, and jobs submitted afterwards run as usual."""
    from ldsc_b200.api import WindowMode, run_l2
    from ldsc_b200.serve import Server
    spec, panel, snps = resident
    wm = WindowMode.Cm(1.0)
    reg = _region(snps, 20000, 40000)
    want = run_l2(ctx, reg, panel, wm, 200, snp_level_masking=True, precision="int8", yes_really=True)[0]
    with Server(0, n_slots=3) as srv:
        got = {}
        orig = srv._submit

        def keep(job, k):   # capture the prewarm job's output arrays
            got.update(k)
            return orig(job, k)

        srv._submit = keep
        srv.prewarm(srv.submit_l2, panel, reg, wm, 200, row_begin=20000, snp_level_masking=True)
        srv._submit = orig
        st = srv.stats()
        assert st["completed"] == 3 and st["submitted"] == 3
        np.testing.assert_array_equal(got["l2"], want)
        t = srv.submit_l2(panel, _region(snps, 25000, 30000), wm, 200, row_begin=25000, snp_level_masking=True)
        srv.wait(t)
        assert srv.stats()["completed"] == 4


def test_admission_by_device_budget(ctx, resident):
    """A budget that holds one large job at a time: every job still runs,
    the slots' workspace stays within the budget, and a job larger than the
    whole budget is refused at submission."""
    from ldsc_b200 import _lib as L
    from ldsc_b200.api import LdscError, WindowMode, _ArgPack
    from ldsc_b200.serve import Server
    import ctypes as C
    spec, panel, snps = resident
    wm = WindowMode.Cm(1.0)
    reg = _region(snps, 0, 20000)
    pack = _ArgPack(reg, wm, 200, None, None, None, True, False, None, False, True, "int8", False, None,
                    records_are_rows=True)
    need = C.c_uint64()
    assert L.load().ldsc_l2_workspace_bytes(C.byref(pack.args), spec.n_indiv, C.byref(need)) == 0
    budget = int(need.value * 1.5)
    with Server(0, n_slots=3, budget_bytes=budget) as srv:
        ts = [srv.submit_l2(panel, _region(snps, b, b + 20000), wm, row_begin=b, snp_level_masking=True)
              for b in (0, 10000, 20000, 30000, 40000)]
        small = srv.submit_l2(panel, _region(snps, 0, 1000), wm, row_begin=0, snp_level_masking=True)
        for t in ts + [small]:
            srv.wait(t)
        st = srv.stats()
        assert st["reserved_bytes"] <= budget and st["completed"] == 6
        with pytest.raises(LdscError):
            srv.submit_l2(panel, _region(snps, 0, 60000), wm, row_begin=0, snp_level_masking=True)


def test_failed_job_reports_and_server_continues(ctx, resident):
    from ldsc_b200.api import LdscError, WindowMode
    from ldsc_b200.serve import Server
    spec, panel, snps = resident
    wm = WindowMode.Cm(1.0)
    with Server(0, n_slots=2) as srv:
        bad = srv.submit_l2(panel, _region(snps, 50000, 60000), wm, row_begin=55000, snp_level_masking=True)
        good = srv.submit_l2(panel, _region(snps, 0, 3000), wm, row_begin=0, snp_level_masking=True)
        with pytest.raises(LdscError, match="more SNP records than panel rows"):
            srv.wait(bad)
        (l2, maf, perf), _ = srv.wait(good)
        assert perf.n_pairs > 0 and l2.shape == (3000, 1) and np.all(np.isfinite(l2))
