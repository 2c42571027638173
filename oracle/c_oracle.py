"""ctypes front end of the C oracle (oracle/jacobi_oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline legs of bench.py.  Builds the oracle with ``make -C oracle`` on
first use when the shared object is missing.
"""
from __future__ import annotations

import ctypes
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "_build" / "libjacobi_oracle.so"
FULL_MATRICES, VALUES_ONLY = 1, 2

_lib = None


def build(force=False):
    """make -C oracle (rebuilds when the sources or include/jacobi_b200.h
    changed).  Without make/gcc an existing library is used as is."""
    try:
        subprocess.run(["make", "-s", "-C", str(HERE)] + (["-B"] if force else []), check=True)
    except (OSError, subprocess.CalledProcessError):
        if not LIB.exists():
            raise
    return LIB


def lib():
    global _lib
    if _lib is None:
        build()
        l = ctypes.CDLL(str(LIB))
        P, I32, I64, F64 = ctypes.c_void_p, ctypes.c_int32, ctypes.c_int64, ctypes.c_double
        for name in ("jo_svd_batched_f32", "jo_svd_batched_f64"):
            f = getattr(l, name)
            f.restype = ctypes.c_int
            f.argtypes = [P, P, P, P, I64, I32, I32, I32, I32, F64, I32, P, P, I32]
        l.jo_svd_uneven_f32.restype = ctypes.c_int
        l.jo_svd_uneven_f32.argtypes = [P, P, P, P, P, I64, F64, I32, P, P, I32]
        l.jo_max_threads.restype = ctypes.c_int
        _lib = l
    return _lib


def _p(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


def svd_batched(a, rank=None, full_matrices=False, values_only=False, tol=None, max_sweeps=60, threads=0):
    """Oracle svd(a, 'jacobi') of a (B, m, n) float32/float64 array.

    Returns U, S, Vh (None with values_only), sweeps (B,), status (B,)."""
    a = np.ascontiguousarray(a)
    if a.ndim == 2:
        a = a[None]
    b, m, n = a.shape
    k = min(m, n)
    rank = k if rank is None else rank
    flags = (FULL_MATRICES if full_matrices else 0) | (VALUES_ONLY if values_only else 0)
    ucols = m if full_matrices else rank
    vrows = n if full_matrices else rank
    u = None if values_only else np.zeros((b, m, ucols), a.dtype)
    vh = None if values_only else np.zeros((b, vrows, n), a.dtype)
    s = np.zeros((b, rank), a.dtype)
    sweeps = np.zeros(b, np.int32)
    status = np.zeros(b, np.int32)
    f = lib().jo_svd_batched_f64 if a.dtype == np.float64 else lib().jo_svd_batched_f32
    if a.dtype not in (np.float32, np.float64):
        raise TypeError("oracle takes float32/float64")
    rc = f(_p(a), _p(u), _p(s), _p(vh), b, m, n, rank, flags, float(tol or 0.0), max_sweeps, _p(sweeps),
           _p(status), threads)
    if rc:
        raise ValueError(f"oracle rejected the arguments (code {rc})")
    return u, s, vh, sweeps, status


def svd_uneven(flat, desc, tol=None, max_sweeps=60, threads=0, u_size=None, s_size=None, v_size=None):
    """Oracle over an uneven batch: flat float32 input, `desc` a numpy
    structured array with the jb_matrix_desc layout.  Returns flat U, S, Vh,
    sweeps, status."""
    flat = np.ascontiguousarray(flat, np.float32)
    desc = np.ascontiguousarray(desc)
    count = len(desc)
    k = np.minimum(desc["m"], desc["n"]).astype(np.int64)
    u_size = u_size or int((desc["u_off"] + desc["m"].astype(np.int64) * k).max()) if count else 1
    s_size = s_size or int((desc["s_off"] + k).max()) if count else 1
    v_size = v_size or int((desc["v_off"] + k * desc["n"]).max()) if count else 1
    u = np.zeros(max(u_size, 1), np.float32)
    s = np.zeros(max(s_size, 1), np.float32)
    vh = np.zeros(max(v_size, 1), np.float32)
    sweeps = np.zeros(count, np.int32)
    status = np.zeros(count, np.int32)
    rc = lib().jo_svd_uneven_f32(_p(flat), _p(u), _p(s), _p(vh), _p(desc), count, float(tol or 0.0), max_sweeps,
                                 _p(sweeps), _p(status), threads)
    if rc:
        raise ValueError(f"oracle rejected the arguments (code {rc})")
    return u, s, vh, sweeps, status


def max_threads():
    return lib().jo_max_threads()
