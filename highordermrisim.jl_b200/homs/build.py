"""Build libhoms.so (sm_100a) in-tree with nvcc.

    python -m homs.build            # from highordermrisim.jl_b200/
    python highordermrisim.jl_b200/homs/build.py

The plain kernels are compiled with -fmad=false (no multiply-add
contraction, so FP64 results follow the reference's rounding order); the
split kernel and the runtime use default contraction.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(ROOT, "csrc")
BUILD = os.path.join(ROOT, "_build")
LIB = os.path.join(PKG, "libhoms.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-O2",
          "--expt-relaxed-constexpr", "-Xptxas", "-v"]
UNITS = {
    "homs_plain.cu": ["-fmad=false"],
    "homs_split.cu": [],
    "homs_api.cu": [],
    "homs_kspace.cu": [],
    "homs_phantom.cu": [],
    "homs_noalloc.cu": [],
    "homs_server.cu": [],
}


def nvcc() -> str:
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(cand):
        raise RuntimeError("nvcc not found; libhoms needs the CUDA toolkit to build")
    return cand


def sources():
    return [os.path.join(CSRC, f) for f in sorted(os.listdir(CSRC)) if f.endswith((".cu", ".cuh"))] + [
        os.path.join(os.path.dirname(ROOT), "include", "homs.h")]


def up_to_date() -> bool:
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    return all(os.path.getmtime(s) <= t for s in sources())


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and up_to_date():
        return LIB
    os.makedirs(BUILD, exist_ok=True)
    cc = nvcc()
    objs = []
    for unit, extra in UNITS.items():
        obj = os.path.join(BUILD, unit.replace(".cu", ".o"))
        cmd = [cc, *ARCH, *COMMON, *extra, "-c", os.path.join(CSRC, unit), "-o", obj]
        res = subprocess.run(cmd, capture_output=True, text=True)
        log = os.path.join(BUILD, unit + ".ptxas.txt")
        with open(log, "w") as fh:
            fh.write(res.stdout + res.stderr)
        if res.returncode != 0:
            sys.stderr.write(res.stdout + res.stderr)
            raise RuntimeError(f"nvcc failed for {unit}")
        if verbose:
            sys.stdout.write(res.stderr)
        objs.append(obj)
    tmp = LIB + ".tmp"
    cmd = [cc, *ARCH, "-shared", "--cudart", "static", "-o", tmp, *objs]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        sys.stderr.write(res.stdout + res.stderr)
        raise RuntimeError("nvcc link failed")
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
