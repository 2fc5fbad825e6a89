"""Build libldsc_b200.so in-tree with nvcc for sm_100a.

    python -m ldsc_b200.build [--force]

Objects go to ldsc_b200/_build/, the library to ldsc_b200/libldsc_b200.so.
The CUDA runtime is linked statically so the library only needs the driver.
"""
from __future__ import annotations

import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
INC = os.path.join(os.path.dirname(HERE), "include")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libldsc_b200.so")

NVCC = os.environ.get("NVCC", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CUFLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-I", CSRC, "-I", INC,
                  "--expt-relaxed-constexpr"]
CXXFLAGS = ["-O3", "-std=c++17", "-fPIC", "-Wall", "-I", CSRC, "-I", INC]


def _sources():
    srcs = sorted(f for f in os.listdir(CSRC) if f.endswith((".cu", ".cpp")))
    return [os.path.join(CSRC, f) for f in srcs]


def _headers():
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    hs.append(os.path.join(INC, "ldsc_b200.h"))
    return hs


def _compile(src: str, force: bool, extra: list) -> str:
    obj = os.path.join(BUILD, os.path.basename(src) + ".o")
    newest_dep = max([os.path.getmtime(src)] + [os.path.getmtime(h) for h in _headers()])
    if not force and os.path.exists(obj) and os.path.getmtime(obj) >= newest_dep:
        return obj
    if src.endswith(".cu"):
        cmd = [NVCC, "-c", src, "-o", obj] + CUFLAGS + extra
    else:
        cuda_inc = os.path.join(os.path.dirname(os.path.dirname(
            subprocess.check_output(["which", NVCC]).decode().strip())), "include")
        cmd = ["g++", "-c", src, "-o", obj, "-I", cuda_inc] + CXXFLAGS
    subprocess.check_call(cmd)
    return obj


def build(force: bool = False, extra_cuflags: list | None = None) -> str:
    os.makedirs(BUILD, exist_ok=True)
    extra = list(extra_cuflags or [])
    srcs = _sources()
    with ThreadPoolExecutor(max_workers=min(8, len(srcs))) as ex:
        objs = list(ex.map(lambda s: _compile(s, force, extra), srcs))
    newest = max(os.path.getmtime(o) for o in objs)
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < newest:
        tmp = LIB + ".tmp"
        subprocess.check_call([NVCC, "-shared", "-o", tmp] + ARCH + objs +
                              ["-cudart", "static", "-lrt", "-ldl", "-lpthread"])
        os.replace(tmp, LIB)
    return LIB


def ptxas_report() -> str:
    """Registers / spills / shared memory of every kernel (-Xptxas -v)."""
    out = []
    for src in _sources():
        if src.endswith(".cu"):
            r = subprocess.run([NVCC, "-c", src, "-o", os.devnull, "-Xptxas", "-v"] + CUFLAGS,
                               capture_output=True, text=True)
            out.append(r.stderr)
    return "\n".join(out)


if __name__ == "__main__":
    if "--ptxas" in sys.argv:
        print(ptxas_report())
    else:
        print(build(force="--force" in sys.argv))
