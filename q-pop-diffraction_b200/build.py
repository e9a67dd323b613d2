"""
Build libqpopdiff.so in-tree with nvcc for sm_100a (B200).

    python -m qpop_diffraction_b200.build        (or build() from Python)

The library is a plain shared object with a C ABI (include/qpopdiff.h); no torch
headers are involved, so it is loaded with ctypes.  Every CUDA source compiles to its own
object under _build/ (in parallel, each one only when it or a header it includes changed, from
the dependency file nvcc writes beside it), and the objects link into the library.
"""

from __future__ import annotations

import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
INCLUDE = ROOT / "include"
LIB = PKG / "libqpopdiff.so"
OBJ = PKG / "_build"

SOURCES = ["qpd_api.cu", "qpd_noalloc.cu", "qpd_rsm.cu", "qpd_n4000.cu", "qpd_probe.cu"]
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


def _deps(dfile: Path):
    """Files named in an nvcc/gcc dependency file (make syntax)."""
    try:
        text = dfile.read_text()
    except OSError:
        return None
    text = text.replace("\\\n", " ")
    out = []
    for line in text.splitlines():
        if ":" not in line:
            continue
        out += [Path(t) for t in line.split(":", 1)[1].split()]
    return out


def _obj_current(src: Path, obj: Path, flags_file: Path, flags: str):
    if not obj.exists() or not flags_file.exists() or flags_file.read_text() != flags:
        return False
    deps = _deps(obj.with_suffix(".d"))
    if not deps:
        return False
    t = obj.stat().st_mtime
    return all(d.exists() and d.stat().st_mtime <= t for d in deps + [src])


def _compile(src: Path, common, force, verbose):
    obj = OBJ / (src.stem + ".o")
    flags_file = OBJ / (src.stem + ".flags")
    flags = " ".join(common)
    if not force and _obj_current(src, obj, flags_file, flags):
        return obj
    tmp = obj.with_suffix(f".o.tmp{os.getpid()}")
    cmd = [nvcc(), *common, "-MD", "-MF", str(obj.with_suffix(".d")), "-c", str(src), "-o", str(tmp)]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    try:
        subprocess.run(cmd, check=True)
        os.replace(tmp, obj)
        flags_file.write_text(flags)
    finally:
        tmp.unlink(missing_ok=True)
    return obj


def build(force=False, verbose=False, extra=()):
    """Compile every CUDA source and link libqpopdiff.so next to this file; returns its path."""
    if not force and up_to_date():
        return LIB
    OBJ.mkdir(exist_ok=True)
    common = [*ARCH, "-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
              "-I", str(INCLUDE), "-I", str(CSRC), "-DQPD_BUILD", *extra]
    with ThreadPoolExecutor(max_workers=max(1, min(len(SOURCES), os.cpu_count() or 1))) as ex:
        objs = list(ex.map(lambda s: _compile(s, common, force, verbose), sources()))
    # per-process temporary: concurrent builds each write their own file and the last rename wins
    tmp = LIB.with_suffix(f".so.tmp{os.getpid()}")
    cmd = [nvcc(), *ARCH, "-shared", "-Xcompiler", "-fPIC", *map(str, objs), "-o", str(tmp)]
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
