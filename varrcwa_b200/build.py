"""Build the in-tree CUDA shared library ``varrcwa_b200/libvrc.so`` for sm_100a.

Usage: ``python -m varrcwa_b200.build`` (or ``__graft_entry__.build()``).
Objects go to ``_build/`` at the repository root; the library is written next
to this file so that it travels with the source tree.
"""
from __future__ import annotations

import concurrent.futures
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
BUILD = ROOT / "_build"
LIB = PKG / "libvrc.so"

SOURCES = ["gemm.cu", "inverse.cu", "eig.cu", "hessenberg.cu", "qr.cu", "assembly.cu", "segment.cu", "engine.cu", "drivers.cu",
           "capi.cu", "noalloc.cu", "adjoint.cu", "stack.cu", "gds.cu"]
HEADERS = ["common.cuh", "kernels.h", "engine.h", "householder.cuh"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-Wall",
         "-Xcompiler", "-Wno-unused-function", "--expt-relaxed-constexpr"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def _newest_dep() -> float:
    deps = [CSRC / h for h in HEADERS] + [ROOT / "include" / "vrc.h"]
    return max(p.stat().st_mtime for p in deps if p.exists())


def _compile(src: str, verbose: bool) -> Path:
    obj = BUILD / (Path(src).stem + ".o")
    s = CSRC / src
    if obj.exists() and obj.stat().st_mtime >= max(s.stat().st_mtime, _newest_dep()):
        return obj
    cmd = [nvcc(), *ARCH, *FLAGS, "-I", str(ROOT / "include"), "-c", str(s), "-o", str(obj)]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{r.stdout}\n{r.stderr}")
    return obj


def build(verbose: bool = False, force: bool = False) -> Path:
    BUILD.mkdir(exist_ok=True)
    if force:
        for o in BUILD.glob("*.o"):
            o.unlink()
    with concurrent.futures.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        objs = list(ex.map(lambda s: _compile(s, verbose), SOURCES))
    if LIB.exists() and LIB.stat().st_mtime >= max(o.stat().st_mtime for o in objs):
        return LIB
    tmp = LIB.with_suffix(".so.tmp")
    cmd = [nvcc(), *ARCH, "-shared", "-o", str(tmp), *map(str, objs), "-lcudart"]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv, force="-f" in sys.argv))
