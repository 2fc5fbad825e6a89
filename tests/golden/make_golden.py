"""Generate the committed golden fixtures under tests/golden/.

    python tests/golden/make_golden.py

* micro.npz -- the reference's known-answer micro BED (src/l2/mod.rs:1191-1225):
  4 individuals x 2 identical SNPs, bytes 6c 1b 01 f0 f0, 100 kb window,
  chunk 2; expected l2 = [2, 2], MAF = [0.5, 0.5].  The expected values are the
  reference test's own assertions.
* small_panel.npz -- a 3-chromosome synthetic panel (N = 203, M = 1,400) with
  planted edge cases (monomorphic, all-missing, all-heterozygous SNPs, a
  chromosome of two SNPs) and expected l2 / MAF from the C oracle in the modes
  the tests cover.  The oracle itself is checked against the brute-force
  definition in tests/test_oracle.py.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from ldsc_b200 import synth  # noqa: E402
from oracle import OracleL2Args, oracle_l2  # noqa: E402


def small_panel():
    spec = synth.PanelSpec(n_indiv=203, chrom_sizes=[700, 450, 248, 2], chrom_cm=[6.0, 4.0, 2.0, 0.1],
                           chrom_ids=[1, 2, 5, 7], founders=12, switch_p=0.02, miss=0.02, seed=77)
    body = synth.bed_body(spec)
    chr_, cm, bp = synth.positions(spec)
    bpr = spec.bpr
    # planted edge cases
    body[10] = 0xFF            # all genotype 0: monomorphic
    body[11] = 0x55            # all missing
    body[12] = 0xAA            # all heterozygous: monomorphic with g = 1
    body[700] = 0x00           # first SNP of chr 2: all genotype 2
    # fix trailing padding bits of the planted rows (individuals 203..207 do not exist)
    for r in (10, 11, 12, 700):
        last = body[r, bpr - 1]
        body[r, bpr - 1] = last & 0b00111111
    return spec, body, chr_, cm, bp


MODES = {
    # name: (mode, wind, chunk, masking, per_chr, use_f32, sketch, annot?, pq)
    "cm1_chunk50": ("cm", 1.0, 50, False, True, False, 0, False, None),
    "cm1_masked": ("cm", 1.0, 50, True, True, False, 0, False, None),
    "cm1_global": ("cm", 1.0, 64, False, False, False, 0, False, None),
    "kb500_chunk40": ("kb", 500.0, 40, False, True, False, 0, False, None),
    "snp25_masked": ("snp", 25, 30, True, True, False, 0, False, None),
    "cm1_annot3": ("cm", 1.0, 50, False, True, False, 0, True, None),
    "cm1_perallele": ("cm", 1.0, 50, True, True, False, 0, False, 1.0),
    "cm1_f32": ("cm", 1.0, 50, False, True, True, 0, False, None),
    "cm1_sketch50": ("cm", 1.0, 50, True, True, True, 50, False, None),
    "cm1_sketch200": ("cm", 1.0, 50, True, True, True, 200, False, None),
    "cm1_sketch50_maf": ("cm", 1.0, 50, True, True, True, 50, False, None),
    "cm1_sketch200_maf": ("cm", 1.0, 50, True, True, True, 200, False, None),
}
# sketch modes run with --sketch-maf-aware (the kurtosis-shifted correction)
MAF_AWARE = {"cm1_sketch50_maf", "cm1_sketch200_maf"}


def annot3(m, seed=5):
    rng = np.random.default_rng(seed)
    return np.asfortranarray(np.stack([np.ones(m), (rng.random(m) < 0.3).astype(float),
                                       np.clip(rng.standard_normal(m), -3, 3)], axis=1))


def oracle_args(name, body, n, chr_, cm, bp):
    mode, wind, chunk, masking, per_chr, f32, sk, has_annot, pq = MODES[name]
    return OracleL2Args(bed_body=body, n_file_indiv=n, chr=chr_, cm=cm, bp=bp, mode=mode,
                        wind=wind if mode != "snp" else 0.0, wind_snp=int(wind) if mode == "snp" else 0,
                        chunk_c=chunk, masking=masking, per_chr=per_chr, use_f32=f32, sketch_d=sk,
                        annot=annot3(len(chr_)) if has_annot else None, pq_exp=pq,
                        sketch_maf_aware=name in MAF_AWARE)


def main():
    np.savez_compressed(os.path.join(HERE, "micro.npz"),
                        bed=np.array([0x6C, 0x1B, 0x01, 0xF0, 0xF0], dtype=np.uint8),
                        chr=np.array([1, 1], dtype=np.uint8), cm=np.zeros(2), bp=np.array([100, 200], dtype=np.uint32),
                        n_indiv=4, l2=np.array([2.0, 2.0]), maf=np.array([0.5, 0.5]))
    spec, body, chr_, cm, bp = small_panel()
    out = dict(body=body, chr=chr_, cm=cm, bp=bp, n_indiv=spec.n_indiv)
    for name in MODES:
        l2, maf, npairs, _ = oracle_l2(oracle_args(name, body, spec.n_indiv, chr_, cm, bp))
        out[f"l2_{name}"] = l2
        out[f"maf_{name}"] = maf
        out[f"pairs_{name}"] = npairs
    np.savez_compressed(os.path.join(HERE, "small_panel.npz"), **out)
    print("wrote", sorted(out))


if __name__ == "__main__":
    main()
