"""Build ``libfluxion_cuda.so`` (the C-ABI CUDA library) in-tree for sm_100a.

Every ``csrc/*.cu`` file is compiled with nvcc for ``compute_100a``/``sm_100a``
and linked into ``fluxion_b200/libfluxion_cuda.so``.  Kernels are compiled with
``-fmad=false`` (and host code with ``-ffp-contract=off``): the only fused
multiply-adds are the explicit ``fma`` calls that restate the reference's
``f64::mul_add``, which keeps F64 results bitwise comparable with the CPU path.
The architecture can be overridden with ``FLUXION_CUDA_ARCH`` (e.g. ``sm_100a``).

``build(checked=True)`` compiles the same sources with ``FX_CHECKED`` into
``libfluxion_cuda_checked.so``: kernels that test every index they compute and record, never
trap on, an out-of-range one (``fx_checked_status``).  ``FLUXION_CHECKED=1`` makes the package
load it instead of the default library.
"""
from __future__ import annotations

import concurrent.futures as cf
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD_DIR = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libfluxion_cuda.so")
LIB_CHECKED = os.path.join(HERE, "libfluxion_cuda_checked.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")


def _arch_flags():
    arch = os.environ.get("FLUXION_CUDA_ARCH", "sm_100a")
    num = arch.replace("sm_", "")
    return ["-gencode", f"arch=compute_{num},code=sm_{num}"]


COMMON = [
    "-O3", "-std=c++17", "-lineinfo", "--extended-lambda", "-fmad=false",
    "-Xcompiler", "-fPIC,-ffp-contract=off,-O3",
    "-Xptxas", "-O3",
]


def _needs(obj: str, src: str, deps) -> bool:
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return any(os.path.getmtime(p) > t for p in [src, *deps])


def build(verbose: bool = False, force: bool = False, ptxas_verbose: bool = False, checked: bool = False) -> str:
    build_dir = os.path.join(BUILD_DIR, "checked") if checked else BUILD_DIR
    lib = LIB_CHECKED if checked else LIB
    os.makedirs(build_dir, exist_ok=True)
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    deps = sorted(glob.glob(os.path.join(CSRC, "*.cuh"))) + [
        os.path.join(os.path.dirname(HERE), "include", "fluxion_cuda.h")]
    objs = []
    jobs = []
    for s in srcs:
        o = os.path.join(build_dir, os.path.basename(s)[:-3] + ".o")
        objs.append(o)
        if force or _needs(o, s, deps):
            cmd = [NVCC, *_arch_flags(), *COMMON, *(["-DFX_CHECKED"] if checked else []), "-c", s, "-o", o]
            if ptxas_verbose:
                cmd += ["-Xptxas", "-v"]
            jobs.append(cmd)

    def run(cmd):
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0 or (verbose and r.stderr):
            sys.stderr.write(r.stderr)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed for {cmd[-3]}")
        return r.stderr

    if jobs:
        with cf.ThreadPoolExecutor(max_workers=min(8, len(jobs))) as ex:
            list(ex.map(run, jobs))
    if force or jobs or not os.path.exists(lib):
        link = [NVCC, *_arch_flags(), "-shared", "-o", lib + ".tmp", *objs, "-lcudart", "-ldl"]
        if verbose:
            print(" ".join(link), flush=True)
        subprocess.run(link, check=True)
        os.replace(lib + ".tmp", lib)
    return lib


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv, force="-f" in sys.argv, ptxas_verbose="--ptxas" in sys.argv,
                checked="--checked" in sys.argv))
