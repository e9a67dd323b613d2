"""
Build libqpopdiff.so in-tree with nvcc for sm_100a (B200).

    python -m qpop_diffraction_b200.build        (or build() from Python)

The library is a plain shared object with a C ABI (include/qpopdiff.h); no torch
headers are involved, so it is loaded with ctypes.
"""

from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
INCLUDE = ROOT / "include"
LIB = PKG / "libqpopdiff.so"

SOURCES = ["qpd_api.cu", "qpd_noalloc.cu", "qpd_rsm.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc():
    cand = os.environ.get("NVCC") or shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(cand).exists() and shutil.which(cand) is None:
        raise RuntimeError("nvcc not found: the CUDA toolkit is needed to build libqpopdiff.so")
    return cand


def sources():
    return [CSRC / s for s in SOURCES]


def inputs():
    return sorted(CSRC.glob("*.cu")) + sorted(CSRC.glob("*.cuh")) + sorted(CSRC.glob("*.h")) + sorted(INCLUDE.glob("*.h"))


def up_to_date(lib=LIB):
    if not lib.exists():
        return False
    t = lib.stat().st_mtime
    return all(p.stat().st_mtime <= t for p in inputs())


def build(force=False, verbose=False, extra=()):
    """Compile every CUDA source into libqpopdiff.so next to this file; returns its path."""
    if not force and up_to_date():
        return LIB
    # per-process temporary: concurrent builds each write their own file and the last rename wins
    tmp = LIB.with_suffix(f".so.tmp{os.getpid()}")
    cmd = [nvcc(), *ARCH, "-O3", "-std=c++17", "-lineinfo", "-shared", "-Xcompiler", "-fPIC",
           "-Xcompiler", "-fvisibility=hidden", "-I", str(INCLUDE), "-I", str(CSRC),
           "-DQPD_BUILD", *extra, *map(str, sources()), "-o", str(tmp)]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    try:
        subprocess.run(cmd, check=True)
        os.replace(tmp, LIB)
    finally:
        tmp.unlink(missing_ok=True)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True,
                extra=["-Xptxas", "-v"] if "--ptxas" in sys.argv else []))
