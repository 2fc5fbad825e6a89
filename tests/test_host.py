"""Host-side checks that need no GPU: the C ABI library loads and exports its
declared symbols, BED validation, window planning, the CountSketch hash."""
import os
import re

import numpy as np
import pytest

from ldsc_b200.build import build

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")


@pytest.fixture(scope="module")
def lib():
    build()
    from ldsc_b200 import _lib
    return _lib.load()


def declared_symbols():
    text = open(os.path.join(ROOT, "include", "ldsc_b200.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(ldsc_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol(lib):
    syms = declared_symbols()
    assert len(syms) >= 15
    missing = [s for s in syms if not hasattr(lib, s)]
    assert not missing, missing
    from ldsc_b200._lib import SIGNATURES
    assert sorted(SIGNATURES) == syms


def test_abi_version(lib):
    assert lib.ldsc_abi_version() == 1


def test_bed_validation_messages(lib):
    from ldsc_b200.api import LdscError, bed_validate
    z = np.load(os.path.join(GOLDEN, "micro.npz"))
    bed_validate(z["bed"], 4, 2)
    bad = z["bed"].copy()
    bad[0] = 0xFF
    with pytest.raises(LdscError, match="invalid magic bytes"):
        bed_validate(bad, 4, 2)
    with pytest.raises(LdscError, match="invalid length"):
        bed_validate(z["bed"][:-1], 4, 2)
    mode = z["bed"].copy()
    mode[2] = 0
    with pytest.raises(LdscError, match="not SNP-major"):
        bed_validate(mode, 4, 2)
    with pytest.raises(LdscError, match="too short"):
        bed_validate(z["bed"][:2], 4, 2)


def test_python_bed_validation_matches(lib):
    from ldsc_b200.plink import validate_bed
    z = np.load(os.path.join(GOLDEN, "micro.npz"))
    assert validate_bed(z["bed"], 4, 2).tolist() == [0xF0, 0xF0]
    with pytest.raises(ValueError, match="invalid length"):
        validate_bed(z["bed"][:-1], 4, 2)


def test_left_limits_and_pair_counts_match_oracle(lib):
    from golden.make_golden import MODES
    from ldsc_b200.api import WindowMode, left_limits, pair_count
    from ldsc_b200.plink import BimTable
    from test_oracle import py_left_limits
    z = np.load(os.path.join(GOLDEN, "small_panel.npz"))
    chr_, cm, bp = z["chr"], z["cm"], z["bp"]
    m = len(chr_)
    snps = BimTable(chr_, [f"rs{i}" for i in range(m)], cm, bp, np.arange(m, dtype=np.int64))
    for name, (mode, wind, chunk, masking, per_chr, *_rest) in MODES.items():
        wm = {"cm": WindowMode.Cm, "kb": WindowMode.Kb, "snp": WindowMode.Snp}[mode](wind)
        got = left_limits(snps, wm, chunk, masking, not per_chr)
        exp = py_left_limits(chr_, cm, bp, mode, wind if mode != "snp" else 0.0,
                             int(wind) if mode == "snp" else 0, chunk, masking, per_chr)
        assert np.array_equal(got, exp), name
        assert pair_count(snps, wm, chunk, masking, not per_chr) == int(z[f"pairs_{name}"]), name


def test_countsketch_hash_restatements_agree(lib):
    """The engine's and the oracle's restatements of fastrand's WyRand stream
    (written independently) produce the same buckets and signs."""
    from ldsc_b200.api import countsketch_hash
    from oracle import countsketch_hash as ocs
    for n, d in [(10, 7), (503, 50), (100000, 1000), (4099, 4098)]:
        b1, s1 = countsketch_hash(n, d, 42)
        b2, s2 = ocs(n, d, 42)
        assert np.array_equal(b1, b2) and np.array_equal(s1, s2)
        assert b1.max() < d


def test_wyrand_stream_properties():
    from oracle import wyrand_stream
    x = wyrand_stream(42, 200000)
    bits = np.unpackbits(x.view(np.uint8))
    assert abs(bits.mean() - 0.5) < 0.005
    assert len(np.unique(x)) == len(x)


def test_context_creation_fails_loudly_without_gpu(lib):
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except ImportError:
        pass
    from ldsc_b200.api import Context, LdscError
    with pytest.raises(LdscError):
        Context(0)


def test_synth_panel_statistics():
    from ldsc_b200 import synth
    from ldsc_b200.plink import decode_genotypes
    spec = synth.PanelSpec(n_indiv=301, chrom_sizes=[400], chrom_cm=[5.0], founders=30, miss=0.01, seed=3)
    body = synth.bed_body(spec)
    G = decode_genotypes(body, spec.n_indiv)
    assert abs(np.isnan(G).mean() - 0.01) < 0.004
    f = np.nanmean(G, axis=1) / 2
    maf = np.minimum(f, 1 - f)
    assert maf.max() <= 0.5 and np.median(maf) > 0.1
    chr_, cm, bp = synth.positions(spec)
    assert np.all(np.diff(cm) > 0) and abs(cm[-1] - 5.0) < 1e-9
    # drawing a SNP range on its own gives the same rows
    part = synth.bed_body(spec, 150, 260)
    assert np.array_equal(part, body[150:260])
