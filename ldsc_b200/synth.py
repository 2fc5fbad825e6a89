"""Seeded synthetic PLINK panels (Li-Stephens-style founder mosaic).

The reference's benchmark panels (1000G, a replicated 50K biobank) are not
available offline, so every measurement in this repository runs on panels
drawn here.  The generator is counter-based: every random draw is a pure
function of (seed, stream, a, b), so the numpy implementation below and the
CUDA kernel ``ldsc_synth_bed`` (csrc/synth.cu) produce byte-identical BED
bodies, and any SNP range of a panel can be drawn without drawing the rest.

Model (per SNP j, individual i, haplotype h = 2i, 2i+1):
  * target MAF p_j ~ U(0.01, 0.5); A1 frequency is p_j or 1 - p_j (coin flip);
  * F founder haplotypes with allele_f,j ~ Bernoulli(A1 frequency);
  * each haplotype copies one founder and switches to a uniformly drawn
    founder with probability ``switch_p`` at each SNP j >= 1;
  * genotype = number of A1 alleles over the two haplotypes;
  * each genotype is set missing with probability ``miss``;
  * cM positions: cumulative i.i.d. Exponential(1) gaps scaled to the
    chromosome's length; bp = 1 + floor(cM * 1e6).
"""
from __future__ import annotations

import dataclasses
from typing import List, Optional

import numpy as np

M64 = np.uint64(0xFFFFFFFFFFFFFFFF)
_G0 = np.uint64(0x9E3779B97F4A7C15)
_G1 = np.uint64(0xBF58476D1CE4E5B9)
_G2 = np.uint64(0x94D049BB133111EB)
_KS = np.uint64(0xD1B54A32D192ED03)  # stream multiplier
_KA = np.uint64(0xAEF17502108EF2D9)  # first-index multiplier

STREAM_ALLELE = 1
STREAM_SWITCH = 2
STREAM_FOUNDER = 3
STREAM_MISSING = 4
STREAM_GAP = 5
STREAM_MAF = 6
STREAM_ORIENT = 7
INITIAL = np.uint64(0xFFFFFFFFFFFFFFFF)


def _splitmix(x):
    with np.errstate(over="ignore"):
        z = x + _G0
        z = (z ^ (z >> np.uint64(30))) * _G1
        z = (z ^ (z >> np.uint64(27))) * _G2
        return z ^ (z >> np.uint64(31))


def draw(seed: int, stream: int, a, b):
    """64-bit draw for (seed, stream, a, b): two splitmix64 rounds."""
    a = np.asarray(a, dtype=np.uint64)
    b = np.asarray(b, dtype=np.uint64)
    with np.errstate(over="ignore"):
        k = np.uint64(seed) + np.uint64(stream) * _KS + a * _KA
        return _splitmix(_splitmix(k) + b)


def u01(h):
    return (h >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)


def bounded(h, n: int):
    return ((h >> np.uint64(32)) * np.uint64(n)) >> np.uint64(32)


@dataclasses.dataclass
class PanelSpec:
    n_indiv: int
    chrom_sizes: List[int]          # SNPs per chromosome, in order
    chrom_cm: List[float]           # cM length per chromosome
    chrom_ids: Optional[List[int]] = None
    founders: int = 50
    switch_p: float = 0.01
    miss: float = 0.005
    seed: int = 1

    @property
    def m(self) -> int:
        return int(sum(self.chrom_sizes))

    @property
    def bpr(self) -> int:
        return (self.n_indiv + 3) // 4


def snp_params(spec: PanelSpec):
    """Per-SNP A1 frequency (float64, length M)."""
    j = np.arange(spec.m, dtype=np.uint64)
    p = 0.01 + 0.49 * u01(draw(spec.seed, STREAM_MAF, 0, j))
    flip = (draw(spec.seed, STREAM_ORIENT, 0, j) & np.uint64(1)).astype(bool)
    return np.where(flip, 1.0 - p, p)


def founder_table(spec: PanelSpec):
    """allele[f, j] in {0, 1}, uint8 F x M."""
    pa1 = snp_params(spec)
    f = np.arange(spec.founders, dtype=np.uint64)[:, None]
    j = np.arange(spec.m, dtype=np.uint64)[None, :]
    return (u01(draw(spec.seed, STREAM_ALLELE, f, j)) < pa1[None, :]).astype(np.uint8)


def positions(spec: PanelSpec):
    """(chr uint8, cm float64, bp uint32) per SNP."""
    chrs, cms, bps = [], [], []
    ids = spec.chrom_ids or list(range(1, len(spec.chrom_sizes) + 1))
    start = 0
    for cid, size, length in zip(ids, spec.chrom_sizes, spec.chrom_cm):
        j = np.arange(start, start + size, dtype=np.uint64)
        gaps = -np.log(u01(draw(spec.seed, STREAM_GAP, 0, j)) + 2.0 ** -60)
        cum = np.cumsum(gaps)
        cm = length * cum / cum[-1]
        chrs.append(np.full(size, cid, dtype=np.uint8))
        cms.append(cm)
        bps.append((1 + np.floor(cm * 1e6)).astype(np.uint32))
        start += size
    return np.concatenate(chrs), np.concatenate(cms), np.concatenate(bps)


_CODE = np.array([0b11, 0b10, 0b00], dtype=np.uint8)  # genotype 0,1,2 -> BED code
_MISSING = np.uint8(0b01)


def bed_body(spec: PanelSpec, snp_begin: int = 0, snp_end: Optional[int] = None,
             block: int = 256) -> np.ndarray:
    """BED body rows [snp_begin, snp_end) as uint8 (rows x bpr), numpy reference
    of the CUDA generator.  Meant for small panels (tests)."""
    if snp_end is None:
        snp_end = spec.m
    n, F = spec.n_indiv, spec.founders
    table = founder_table(spec)
    nh = 2 * n
    hap = np.arange(nh, dtype=np.uint64)
    # founder state entering snp_begin: scan back to the last switch
    state = bounded(draw(spec.seed, STREAM_FOUNDER, hap, INITIAL), F).astype(np.int64)
    if snp_begin > 0:
        for jj in range(1, snp_begin):
            sw = u01(draw(spec.seed, STREAM_SWITCH, hap, np.uint64(jj))) < spec.switch_p
            nf = bounded(draw(spec.seed, STREAM_FOUNDER, hap, np.uint64(jj)), F).astype(np.int64)
            state = np.where(sw, nf, state)
    rows = snp_end - snp_begin
    out = np.zeros((rows, spec.bpr), dtype=np.uint8)
    iid = np.arange(n, dtype=np.uint64)
    for b0 in range(snp_begin, snp_end, block):
        b1 = min(b0 + block, snp_end)
        js = np.arange(b0, b1, dtype=np.uint64)
        sw = u01(draw(spec.seed, STREAM_SWITCH, hap[:, None], js[None, :])) < spec.switch_p
        sw[:, js == 0] = False
        nf = bounded(draw(spec.seed, STREAM_FOUNDER, hap[:, None], js[None, :]), F).astype(np.int64)
        col = np.where(sw, np.arange(b1 - b0)[None, :], -1)
        last = np.maximum.accumulate(col, axis=1)
        fidx = np.where(last >= 0, np.take_along_axis(nf, np.maximum(last, 0), axis=1),
                        state[:, None])
        state = fidx[:, -1].copy()
        alle = table[fidx, js[None, :].astype(np.int64)]       # (2n, b)
        g = alle[0::2] + alle[1::2]                            # (n, b)
        miss = u01(draw(spec.seed, STREAM_MISSING, iid[:, None], js[None, :])) < spec.miss
        codes = np.where(miss, _MISSING, _CODE[g])             # (n, b)
        pad = spec.bpr * 4 - n
        if pad:
            codes = np.concatenate([codes, np.zeros((pad, b1 - b0), dtype=np.uint8)], axis=0)
        c4 = codes.T.reshape(b1 - b0, spec.bpr, 4)
        out[b0 - snp_begin:b1 - snp_begin] = (c4[:, :, 0] | (c4[:, :, 1] << 2) |
                                              (c4[:, :, 2] << 4) | (c4[:, :, 3] << 6))
    return out


# ---- the configurations measured in this repository ----------------------

def spec_small(seed: int = 11) -> PanelSpec:
    """Plain exact l2 at small size: N=2,490, M=18,627 on one chromosome,
    50 founders, 0.5% missing, 70 cM."""
    return PanelSpec(n_indiv=2490, chrom_sizes=[18627], chrom_cm=[70.0], founders=50,
                     miss=0.005, seed=seed)


def spec_biobank(seed: int = 12) -> PanelSpec:
    """Exact biobank scale: N=50,000, M=100,000, 200 founders, 1% missing, 100 cM."""
    return PanelSpec(n_indiv=50000, chrom_sizes=[100000], chrom_cm=[100.0], founders=200,
                     miss=0.01, seed=seed)


def spec_sketch(seed: int = 13) -> PanelSpec:
    """Fused CountSketch scale: N=100,000, M=200,000, 1% missing, 150 cM."""
    return PanelSpec(n_indiv=100000, chrom_sizes=[200000], chrom_cm=[150.0], founders=200,
                     miss=0.01, seed=seed)


def spec_partitioned(seed: int = 14) -> PanelSpec:
    """Partitioned LD scores: N=10,000 over 22 chromosomes, M=500,000 with
    M_chr proportional to 23 - chr.  Chromosome length (unspecified by the
    workload) is set proportional to M_chr for a 3,500 cM genome, about 143
    SNPs per cM."""
    M = 500000
    sizes = [M * (23 - c) // 253 for c in range(1, 23)]
    sizes[0] += M - sum(sizes)
    cms = [3500.0 * s / M for s in sizes]
    return PanelSpec(n_indiv=10000, chrom_sizes=sizes, chrom_cm=cms, founders=200, miss=0.01,
                     seed=seed)


def spec_resident(seed: int = 15) -> PanelSpec:
    """Serving panel: N=20,000 x M=1,200,000 over 22 chromosomes (M_chr
    proportional to 23 - chr, 3,500 cM genome), 1% missing."""
    M = 1200000
    sizes = [M * (23 - c) // 253 for c in range(1, 23)]
    sizes[0] += M - sum(sizes)
    cms = [3500.0 * s / M for s in sizes]
    return PanelSpec(n_indiv=20000, chrom_sizes=sizes, chrom_cm=cms, founders=200, miss=0.01,
                     seed=seed)


def partitioned_annot(m: int, seed: int = 21, n_binary: int = 80, n_cont: int = 16) -> np.ndarray:
    """97 annotations: all-ones, 80 binary runs (density U(0.01, 0.2),
    geometric run length with mean 20 SNPs), 16 N(0,1) clipped to +-3."""
    rng = np.random.default_rng(seed)
    cols = [np.ones(m)]
    for _ in range(n_binary):
        dens = rng.uniform(0.01, 0.2)
        # alternating on/off runs: on-runs mean 20, off-runs mean 20*(1-d)/d
        col = np.zeros(m)
        pos = int(rng.integers(0, 40))
        on_mean = 20.0
        off_mean = on_mean * (1.0 - dens) / dens
        while pos < m:
            on = int(rng.geometric(1.0 / on_mean))
            col[pos:pos + on] = 1.0
            pos += on + int(rng.geometric(1.0 / off_mean))
        cols.append(col)
    for _ in range(n_cont):
        cols.append(np.clip(rng.standard_normal(m), -3.0, 3.0))
    return np.asfortranarray(np.stack(cols, axis=1))


def gwas_traits(l2: np.ndarray, m_snps: float, n_traits: int, seed: int = 31):
    """Synthetic GWAS chi^2 statistics over LD scores l2: per trait
    h2 ~ U(0.05, 0.5), N log-uniform in [1e4, 5e5], z_j = sqrt(N h2 l2_j / M) b_j
    + e_j with b_j, e_j ~ N(0, 1), chi2 = z^2 (so E[chi2] = 1 + N h2 l2 / M).
    Returns (chi2 [T x M], N [T], h2 [T])."""
    rng = np.random.default_rng(seed)
    h2 = rng.uniform(0.05, 0.5, n_traits)
    n = np.exp(rng.uniform(np.log(1e4), np.log(5e5), n_traits))
    lm = np.maximum(l2, 0.0)[None, :]
    z = np.sqrt(n[:, None] * h2[:, None] * lm / m_snps) * rng.standard_normal((n_traits, len(l2))) \
        + rng.standard_normal((n_traits, len(l2)))
    return z * z, n, h2


def gwas_pairs(l2: np.ndarray, m_snps: float, n_pairs: int, seed: int = 32):
    """Synthetic z-score pairs with genetic correlation rg ~ U(-0.8, 0.8):
    z_t = sqrt(N_t h_t l2 / M) b_t + e_t with corr(b_1, b_2) = rg.
    Returns (z1, z2, n1, n2, rg)."""
    rng = np.random.default_rng(seed)
    h1, h2 = rng.uniform(0.05, 0.5, n_pairs), rng.uniform(0.05, 0.5, n_pairs)
    n1 = np.exp(rng.uniform(np.log(1e4), np.log(5e5), n_pairs))
    n2 = np.exp(rng.uniform(np.log(1e4), np.log(5e5), n_pairs))
    rg = rng.uniform(-0.8, 0.8, n_pairs)
    m = len(l2)
    b1 = rng.standard_normal((n_pairs, m))
    b2 = rg[:, None] * b1 + np.sqrt(1 - rg[:, None] ** 2) * rng.standard_normal((n_pairs, m))
    lm = np.maximum(l2, 0.0)[None, :]
    z1 = np.sqrt(n1[:, None] * h1[:, None] * lm / m_snps) * b1 + rng.standard_normal((n_pairs, m))
    z2 = np.sqrt(n2[:, None] * h2[:, None] * lm / m_snps) * b2 + rng.standard_normal((n_pairs, m))
    return z1, z2, n1, n2, rg
