"""Build the sm_100a shared library of this package in-tree.

    python pavel-s_svd_b200/build.py          # or __graft_entry__.build()

Produces ``pavel-s_svd_b200/_lib/libjacobi_b200.so`` from ``csrc/*.cu`` with
``nvcc -gencode arch=compute_100a,code=sm_100a``.  The library links the CUDA
runtime statically and exports only the C ABI of include/jacobi_b200.h, so it
has no dependency on torch; the Python side loads it with ctypes.
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
LIBDIR = PKG / "_lib"
LIBNAME = "libjacobi_b200.so"
SOURCES = ["jb_batched.cu", "jb_tensor.cu", "jb_mlp.cu", "jb_block.cu", "jb_eigh.cu", "jb_qr.cu", "jb_complex.cu", "jb_lab.cu", "jb_null.cu", "jb_peak.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found: the CUDA toolkit is required to build the library")


def library_path() -> Path:
    return LIBDIR / LIBNAME


def _stale(out: Path) -> bool:
    if not out.exists():
        return True
    t = out.stat().st_mtime
    deps = list(CSRC.glob("*.cu")) + list(CSRC.glob("*.cuh")) + list((ROOT / "include").glob("*.h"))
    return any(p.stat().st_mtime > t for p in deps)


def build(force: bool = False, verbose: bool = False, extra: list[str] | None = None) -> Path:
    out = library_path()
    if not force and not _stale(out):
        return out
    LIBDIR.mkdir(exist_ok=True)
    tmp = out.with_suffix(".so.tmp")
    cmd = [nvcc(), *ARCH, "-O3", "-lineinfo", "-std=c++17", "-shared", "-Xcompiler", "-fPIC",
           "-Xcompiler", "-fvisibility=hidden", "-I", str(ROOT / "include"), "-I", str(CSRC),
           "-o", str(tmp), *[str(CSRC / s) for s in SOURCES], *(extra or [])]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    tmp.replace(out)
    return out


if __name__ == "__main__":
    v = "-v" in sys.argv
    xs = ["-Xptxas", "-v"] if "--ptxas" in sys.argv else None
    print(build(force=True, verbose=v, extra=xs))
