"""Build the product library (CUDA for sm_100a + host C++) in-tree.

``python -m ccpol23_plus_2025_mbmd_b200.build`` compiles ``csrc/*.cu`` and ``csrc/*.cpp``
with nvcc into ``ccpol23_plus_2025_mbmd_b200/lib/libccpol23_b200.so``.  Each translation unit
is compiled separately (objects in ``_build/``) and rebuilt only when its sources change.
"""
from __future__ import annotations

import hashlib
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
INCLUDE = PKG.parent / "include"
LIBDIR = PKG / "lib"
LIB = LIBDIR / "libccpol23_b200.so"
OBJDIR = PKG.parent / "_build" / "obj"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC,-O2",
              "--expt-relaxed-constexpr", "-Xptxas", "-O3"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def _sources():
    return sorted(CSRC.glob("*.cu")) + sorted(CSRC.glob("*.cpp"))


def _headers():
    return sorted(CSRC.glob("*.h")) + sorted(CSRC.glob("*.cuh")) + sorted(INCLUDE.glob("*.h"))


def _digest(src: Path) -> str:
    h = hashlib.sha256()
    for p in [src, *_headers()]:
        h.update(p.read_bytes())
    h.update(" ".join(ARCH + NVCC_FLAGS).encode())
    return h.hexdigest()[:16]


def build(verbose: bool = False, ptxas_verbose: bool = False) -> Path:
    OBJDIR.mkdir(parents=True, exist_ok=True)
    LIBDIR.mkdir(parents=True, exist_ok=True)
    objs = []
    changed = not LIB.exists()
    for src in _sources():
        obj = OBJDIR / f"{src.stem}.{_digest(src)}.o"
        objs.append(obj)
        if obj.exists() and not ptxas_verbose:
            continue
        changed = True
        cmd = [nvcc(), *ARCH, *NVCC_FLAGS, "-I", str(INCLUDE), "-c", str(src), "-o", str(obj)]
        if ptxas_verbose and src.suffix == ".cu":
            cmd[1:1] = ["-Xptxas", "-v"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    # relink whenever the library was linked from a different set of objects (a source
    # reverted to an earlier state reuses that state's cached object without recompiling)
    stamp = LIBDIR / ".objects"
    listing = "\n".join(o.name for o in objs)
    if changed or not stamp.exists() or stamp.read_text() != listing:
        cmd = [nvcc(), *ARCH, "-shared", "-o", str(LIB), *map(str, objs), "-lcudart_static",
               "-lrt", "-ldl", "-lpthread"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
        stamp.write_text(listing)
    return LIB


if __name__ == "__main__":
    build(verbose=True, ptxas_verbose="-v" in sys.argv)
    print(LIB)
