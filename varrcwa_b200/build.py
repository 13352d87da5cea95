"""Build the in-tree CUDA shared library ``varrcwa_b200/libvrc.so`` for sm_100a.

Usage: ``python -m varrcwa_b200.build`` (or ``__graft_entry__.build()``).
Objects go to ``_build/`` at the repository root; the library is written next
to this file so that it travels with the source tree.

Reuse is decided by content, not by file times: every object carries the
SHA-256 of its source, the shared headers and the compiler flags
(``_build/<name>.o.sha``), and the library carries the hash over all of them
(``libvrc.so.sha``).  ``source_hash()`` recomputes the latter from the tree,
so a loader can refuse a library built from other sources.
"""
from __future__ import annotations

import concurrent.futures
import hashlib
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
STAMP = PKG / "libvrc.so.sha"

SOURCES = ["gemm.cu", "inverse.cu", "eig.cu", "hessenberg.cu", "qr.cu", "assembly.cu", "segment.cu", "engine.cu",
           "drivers.cu", "capi.cu", "noalloc.cu", "adjoint.cu", "stack.cu", "gds.cu", "geom_adjoint.cu", "chain.cu"]
HEADERS = ["common.cuh", "kernels.h", "engine.h", "householder.cuh", "batch.h"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-Wall",
         "-Xcompiler", "-Wno-unused-function", "--expt-relaxed-constexpr"]
LINK = ["-lcudart"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def _sources() -> list:
    return [s for s in SOURCES if (CSRC / s).exists()]


def _deps_hash() -> "hashlib._Hash":
    h = hashlib.sha256()
    for p in [CSRC / x for x in HEADERS] + [ROOT / "include" / "vrc.h"]:
        h.update(p.name.encode())
        h.update(p.read_bytes() if p.exists() else b"")
    h.update(" ".join(ARCH + FLAGS).encode())
    return h


def _object_hash(src: str) -> str:
    h = _deps_hash()
    h.update(src.encode())
    h.update((CSRC / src).read_bytes())
    return h.hexdigest()


def source_hash() -> str:
    """Hash of everything the library is built from (sources, headers, flags)."""
    h = hashlib.sha256()
    for s in _sources():
        h.update(_object_hash(s).encode())
    h.update(" ".join(LINK).encode())
    return h.hexdigest()


def _compile(src: str, verbose: bool) -> Path:
    obj = BUILD / (Path(src).stem + ".o")
    stamp = BUILD / (Path(src).stem + ".o.sha")
    want = _object_hash(src)
    if obj.exists() and stamp.exists() and stamp.read_text().strip() == want:
        return obj
    cmd = [nvcc(), *ARCH, *FLAGS, "-I", str(ROOT / "include"), "-c", str(CSRC / src), "-o", str(obj)]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{r.stdout}\n{r.stderr}")
    stamp.write_text(want + "\n")
    return obj


def is_current() -> bool:
    """True when the library exists and was built from the sources in the tree."""
    return LIB.exists() and STAMP.exists() and STAMP.read_text().strip() == source_hash()


def build(verbose: bool = False, force: bool = False) -> Path:
    BUILD.mkdir(exist_ok=True)
    if force:
        for o in list(BUILD.glob("*.o")) + list(BUILD.glob("*.o.sha")):
            o.unlink()
    with concurrent.futures.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        objs = list(ex.map(lambda s: _compile(s, verbose), _sources()))
    if not force and is_current():
        return LIB
    tmp = LIB.with_suffix(".so.tmp")
    cmd = [nvcc(), *ARCH, "-shared", "-o", str(tmp), *map(str, objs), *LINK]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    os.replace(tmp, LIB)
    STAMP.write_text(source_hash() + "\n")
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv, force="-f" in sys.argv))
