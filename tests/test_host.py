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


def test_left_limits_on_tied_and_unsorted_coordinates(lib):
    """Window limits for sorted coordinates with many ties (the interleaved
    sorted-coordinate walk) and for unsorted ones (the plain two-pointer
    walk), in cM and kb modes, against the Python restatement."""
    from ldsc_b200.api import WindowMode, left_limits
    from ldsc_b200.plink import BimTable
    from test_oracle import py_left_limits
    rng = np.random.default_rng(17)
    m = 3000
    chr_ = np.repeat(np.array([1, 2, 5], dtype=np.uint8), [1700, 40, 1260])
    tied = np.round(np.cumsum(rng.exponential(0.004, m)), 2)           # sorted, many equal values
    shuffled = tied.copy()
    shuffled[1740:] = rng.permutation(shuffled[1740:])                  # chromosome 5 unsorted
    bp = np.sort(rng.integers(0, 3_000_000, m)).astype(np.uint32)
    bp[:1700] = np.sort(rng.integers(0, 900, 1700) * 1000)              # kb ties
    for cm in (tied, shuffled):
        snps = BimTable(chr_, [f"rs{i}" for i in range(m)], cm, bp, np.arange(m, dtype=np.int64))
        for mode, wind in (("cm", 0.5), ("cm", 0.0), ("kb", 40.0)):
            wm = WindowMode.Cm(wind) if mode == "cm" else WindowMode.Kb(wind)
            for masking in (True, False):
                got = left_limits(snps, wm, 100, masking, False)
                exp = py_left_limits(chr_, cm, bp, mode, wind, 0, 100, masking, True)
                assert np.array_equal(got, exp), (mode, wind, masking)


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


# ---- struct layouts: header vs the ctypes mirror vs the Rust binding ----

_STRUCTS = {"ldsc_progress": "Progress", "ldsc_perf": "Perf", "ldsc_l2_args": "L2Args",
            "ldsc_synth_spec": "SynthSpec", "ldsc_h2_args": "H2Args", "ldsc_h2_result": "H2Result",
            "ldsc_h2p_args": "H2PArgs", "ldsc_h2p_result": "H2PResult", "ldsc_rg_args": "RgArgs",
            "ldsc_rg_result": "RgResult", "ldsc_job": "Job", "ldsc_job_result": "JobResult",
            "ldsc_server_stats": "ServerStats"}
_RUST = {"LdscProgress": "ldsc_progress", "LdscPerf": "ldsc_perf", "LdscL2Args": "ldsc_l2_args",
         "LdscH2Args": "ldsc_h2_args", "LdscH2Result": "ldsc_h2_result", "LdscH2pArgs": "ldsc_h2p_args",
         "LdscH2pResult": "ldsc_h2p_result", "LdscRgArgs": "ldsc_rg_args", "LdscRgResult": "ldsc_rg_result"}


def header_structs():
    """{typedef name: [field names in order]} from include/ldsc_b200.h."""
    text = open(os.path.join(ROOT, "include", "ldsc_b200.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    out = {}
    for body, name in re.findall(r"typedef struct\s*\{(.*?)\}\s*(\w+)\s*;", text, flags=re.S):
        fields = []
        for decl in body.split(";"):
            decl = decl.strip()
            if not decl:
                continue
            for piece in decl.split(","):
                fields.append(re.findall(r"[A-Za-z_]\w*", piece)[-1])
        out[name] = fields
    return out


def test_ctypes_mirror_matches_the_header_layout(tmp_path):
    """offsetof / sizeof of every mirrored struct, from gcc on the header,
    against the ctypes classes the Python binding passes."""
    import ctypes
    import subprocess
    from ldsc_b200 import _lib
    hs = header_structs()
    assert set(_STRUCTS) <= set(hs)
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "ldsc_b200.h"', "int main(void) {"]
    for cname in _STRUCTS:
        lines.append(f'printf("{cname} sizeof %zu\\n", sizeof({cname}));')
        for f in hs[cname]:
            lines.append(f'printf("{cname} {f} %zu\\n", offsetof({cname}, {f}));')
    lines.append("return 0; }")
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), "-o", str(exe), str(src)], check=True)
    got = {}
    for line in subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.splitlines():
        s, f, v = line.split()
        got[(s, f)] = int(v)
    for cname, pyname in _STRUCTS.items():
        cls = getattr(_lib, pyname)
        assert [f for f, _ in cls._fields_] == hs[cname], cname
        assert ctypes.sizeof(cls) == got[(cname, "sizeof")], cname
        for f, _ in cls._fields_:
            assert getattr(cls, f).offset == got[(cname, f)], (cname, f)


def test_rust_binding_fields_match_the_header():
    text = open(os.path.join(ROOT, "include", "ldsc_b200.rs")).read()
    hs = header_structs()
    found = dict(re.findall(r"pub struct (Ldsc\w+)\s*\{(.*?)\}", text, flags=re.S))
    for rname, cname in _RUST.items():
        assert rname in found, rname
        fields = re.findall(r"pub (\w+)\s*:", found[rname])
        assert fields == hs[cname], (rname, fields, hs[cname])


def test_rust_binding_functions_are_declared_in_the_header():
    rs = open(os.path.join(ROOT, "include", "ldsc_b200.rs")).read()
    h = open(os.path.join(ROOT, "include", "ldsc_b200.h")).read()
    names = re.findall(r"pub fn (ldsc_\w+)\(", rs)
    assert len(names) >= 10
    for name in names:
        assert re.search(r"\b" + name + r"\s*\(", h), name
