"""Build recipe for the CPU oracle (test infrastructure, not the product).

Compiles ``oracle/ldsc_oracle.c`` into ``oracle/_build/libldsc_oracle.so``
with gcc + OpenMP.  The reference itself (Rust) cannot be compiled in this
image -- there is no cargo/rustc -- so there is no ``oracle/_ref`` build.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "ldsc_oracle.c")
OUT_DIR = os.path.join(HERE, "_build")
OUT = os.path.join(OUT_DIR, "libldsc_oracle.so")


def build(force: bool = False) -> str:
    os.makedirs(OUT_DIR, exist_ok=True)
    if not force and os.path.exists(OUT) and os.path.getmtime(OUT) >= os.path.getmtime(SRC):
        return OUT
    cmd = [
        "gcc", "-O3", "-mavx2", "-mfma", "-fopenmp", "-fPIC", "-shared",
        "-std=gnu11", "-Wall", "-Wno-unused-function", SRC, "-o", OUT + ".tmp", "-lm",
    ]
    subprocess.check_call(cmd)
    os.replace(OUT + ".tmp", OUT)
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))
