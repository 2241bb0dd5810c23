"""Builds libfrpa.so (the C-ABI library) from csrc/*.cu for sm_100a, in-tree.

    python -m fast_rpa_eval_b200.build [--force]

Each translation unit is compiled with nvcc (-gencode arch=compute_100a,code=sm_100a,
static CUDA runtime) and linked into fast_rpa_eval_b200/lib/libfrpa.so.  Objects are
rebuilt only when a source or header is newer.  The sum-up's per-l_max Horner
bodies (kelvin_horner.cuh) are generated into the build directory first by
csrc/gen_kelvin.py.
"""
from __future__ import annotations

import concurrent.futures as cf
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIBDIR = os.path.join(HERE, "lib")
LIB = os.path.join(LIBDIR, "libfrpa.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
         "-I" + os.path.join(ROOT, "include"), "-I" + CSRC, "-I" + BUILD]


def generate_headers() -> list:
    """Writes the generated headers into the build directory (unchanged
    files are left alone, so their timestamps do not force rebuilds)."""
    sys.path.insert(0, CSRC)
    try:
        import gen_kelvin
    finally:
        sys.path.pop(0)
    dst = os.path.join(BUILD, "kelvin_horner.cuh")
    gen_kelvin.write(dst)
    return [dst]


def _newer(target: str, deps) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    os.makedirs(LIBDIR, exist_ok=True)
    generated = generate_headers()
    sources = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    headers = glob.glob(os.path.join(CSRC, "*.cuh")) + [os.path.join(ROOT, "include", "frpa.h")] + generated
    objs, jobs = [], []
    for src in sources:
        obj = os.path.join(BUILD, os.path.basename(src) + ".o")
        objs.append(obj)
        if force or _newer(obj, [src] + headers):
            jobs.append([NVCC, *ARCH, *FLAGS, "-c", src, "-o", obj])
    with cf.ThreadPoolExecutor(max_workers=min(8, max(1, len(jobs)))) as ex:
        for cmd, res in zip(jobs, ex.map(lambda c: subprocess.run(c, capture_output=True, text=True), jobs)):
            if verbose or res.returncode:
                sys.stderr.write(res.stdout + res.stderr)
            if res.returncode:
                raise RuntimeError("nvcc failed: " + " ".join(cmd))
    if force or jobs or _newer(LIB, objs):
        cmd = [NVCC, *ARCH, "-shared", "-cudart", "static", "-o", LIB, *objs]
        res = subprocess.run(cmd, capture_output=True, text=True)
        if res.returncode:
            sys.stderr.write(res.stdout + res.stderr)
            raise RuntimeError("link failed")
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
