"""Builds the overlap_b200 CUDA library for B200 (sm_100a) with nvcc.

    python -m overlap_b200.build [--verbose]

Output: overlap_b200/_lib/libovl_b200.so, loaded by overlap_b200._lib.  The
library is built in-tree so that it ships with the source tree to GPU hosts.
"""
from __future__ import annotations

import argparse
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
OUT_DIR = PKG / "_lib"
LIB = OUT_DIR / "libovl_b200.so"
SOURCES = ["ovl_capi.cu", "ovl_wilson.cu", "ovl_gauge.cu", "ovl_modes.cu", "ovl_noalloc.cu", "ovl_overlap.cu",
           "ovl_chebyshev.cu", "ovl_zolotarev.cpp", "ovl_force.cu", "ovl_ritz.cu", "ovl_batch.cu",
           "ovl_stochastic.cu", "ovl_su3.cu", "ovl_quasi.cu", "ovl_eigen.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def flags(verbose: bool = False) -> list[str]:
    f = ARCH + ["-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr", "-Xcompiler", "-fPIC",
                "-I", str(ROOT / "include"), "-I", str(CSRC)]
    if verbose:
        f += ["-Xptxas", "-v"]
    return f


def build(verbose: bool = False, force: bool = False) -> Path:
    OUT_DIR.mkdir(exist_ok=True)
    deps = [CSRC / s for s in SOURCES] + list(CSRC.glob("*.cuh")) + list(CSRC.glob("*.h")) + [ROOT / "include" / "ovl.h"]
    if not force and LIB.exists() and all(LIB.stat().st_mtime >= d.stat().st_mtime for d in deps):
        return LIB
    objs = []
    for s in SOURCES:
        obj = OUT_DIR / (Path(s).stem + ".o")
        cmd = [nvcc(), *flags(verbose), "-c", str(CSRC / s), "-o", str(obj)]
        res = subprocess.run(cmd, capture_output=True, text=True)
        if res.returncode != 0:
            raise RuntimeError(f"nvcc failed on {s}:\n{res.stderr}")
        if verbose and res.stderr:
            print(res.stderr, file=sys.stderr)
        objs.append(str(obj))
    tmp = LIB.with_suffix(".so.tmp")
    cmd = [nvcc(), *ARCH, "-shared", "-o", str(tmp), *objs, "-lcudart", "-lcusolver", "-lcublas"]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"link failed:\n{res.stderr}")
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--force", action="store_true")
    a = ap.parse_args()
    print(build(verbose=a.verbose, force=a.force))
