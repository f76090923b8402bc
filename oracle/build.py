"""Build recipe for the CPU oracle (test infrastructure only).

Compiles ``oracle/fx_oracle.c`` into ``oracle/_build/libfxoracle.so`` with
``-ffp-contract=off`` so that the only fused multiply-adds are the explicit
``fma()`` calls that restate the reference's ``f64::mul_add``.  The reference
itself (Rust) cannot be compiled here, so there is no ``oracle/_ref`` build.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT_DIR = os.path.join(HERE, "_build")
LIB = os.path.join(OUT_DIR, "libfxoracle.so")


def build(verbose: bool = False) -> str:
    os.makedirs(OUT_DIR, exist_ok=True)
    src = os.path.join(HERE, "fx_oracle.c")
    cmd = [
        "gcc", "-O3", "-std=c11", "-fPIC", "-shared", "-fopenmp",
        "-ffp-contract=off", "-mavx2", "-mfma", "-fno-math-errno",
        "-Wall", "-Wno-unused-function",
        src, "-o", LIB + ".tmp", "-lm",
    ]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
