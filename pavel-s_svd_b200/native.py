"""ctypes binding of the C ABI in include/jacobi_b200.h.

The shared library is built in-tree by ``build.py``.  There is no CPU or
PyTorch fallback: when the library is missing or a CUDA device is absent,
``lib()`` raises and every solver call fails loudly.
"""
from __future__ import annotations

import ctypes
import threading
from pathlib import Path

from .build import library_path

# Return codes and per-matrix status words (include/jacobi_b200.h).
JB_OK, JB_EINVAL, JB_ETOOBIG, JB_EWORKSPACE, JB_ECUDA = 0, 1, 2, 3, 4
ST_OK, ST_NOT_CONVERGED, ST_NONFINITE_IN, ST_NULL_FAILED, ST_NONFINITE_OUT, ST_BAD_DESC, ST_TIMEOUT = (
    0, 1, 2, 3, 4, 5, 6)
FULL_MATRICES, VALUES_ONLY, ROUND_ROBIN, BLOCK_WIDTH_8, ONE_SIZE_CLASS = 1, 2, 4, 8, 16
PREC_NATIVE, PREC_MIXED = 0, 1

RC_NAMES = {JB_EINVAL: "invalid argument", JB_ETOOBIG: "shape too large for this entry point",
            JB_EWORKSPACE: "workspace missing or too small", JB_ECUDA: "CUDA runtime error"}

# Exported symbols, in declaration order of include/jacobi_b200.h.
SYMBOLS = ("jb_version", "jb_device_sm_count", "jb_workspace_bytes", "jb_svd_batched_f32",
           "jb_svd_batched_f64", "jb_uneven_workspace_bytes", "jb_svd_uneven_f32", "jb_svd_uneven_f32_ex",
           "jb_gemm_bf16", "jb_gemm_bf16x", "jb_gemm_bf16x_rows", "jb_gemm_bf16x_rows2", "jb_split_bf16", "jb_split3_bf16",
           "jb_warm_prep_f32", "jb_svd_warm_f32", "jb_transpose_bf16", "jb_bias_act", "jb_relu_backward",
           "jb_col_sum", "jb_mse_grad", "jb_adam", "jb_gram_sketch", "jb_block_eig_f64", "jb_block_eig_workspace_bytes",
           "jb_block_eig_ws", "jb_block_eig_f64_ex", "jb_rows_scatter",
           "jb_rows_combine", "jb_gemm_f64acc", "jb_block_finish", "jb_eigh_workspace_bytes", "jb_eigh_f32",
           "jb_eigh_f64", "jb_eigh_complex_workspace_bytes", "jb_eigh_c64", "jb_eigh_c128",
           "jb_qr_workspace_bytes", "jb_qr_f32", "jb_qr_f64", "jb_qr_c64", "jb_qr_c128",
           "jb_svd_complex_workspace_bytes", "jb_svd_batched_c64", "jb_svd_batched_c128", "jb_jacobi_rounds",
           "jb_complete_null_workspace_bytes", "jb_complete_null", "jb_fma_loop_flops", "jb_fma_loop",
           "jb_svd_batched_f32_noalloc")
GEMM_PLAIN, GEMM_SPLIT3, GEMM_SPLIT6, GEMM_B_MN, GEMM_CHAIN128, GEMM_SYRK = 0, 1, 2, 4, 8, 16
EIG_FP32 = 128  # JB_EIG_FP32
EIG_DEFER_Q = 256  # JB_EIG_DEFER_Q
NOALLOC_SCRATCH_BYTES = 16 << 20  # JB_NOALLOC_SCRATCH_BYTES


class MatrixDesc(ctypes.Structure):
    """jb_matrix_desc: one matrix of an uneven batch (offsets in elements)."""
    _fields_ = [("m", ctypes.c_int32), ("n", ctypes.c_int32), ("rank", ctypes.c_int32),
                ("flags", ctypes.c_int32), ("a_off", ctypes.c_int64), ("u_off", ctypes.c_int64),
                ("s_off", ctypes.c_int64), ("v_off", ctypes.c_int64), ("x_off", ctypes.c_int64)]


DESC_BYTES = ctypes.sizeof(MatrixDesc)  # 56

_lock = threading.Lock()
_lib = None

P, I32, I64, F64, SZ = ctypes.c_void_p, ctypes.c_int32, ctypes.c_int64, ctypes.c_double, ctypes.c_size_t


def _declare(l):
    l.jb_version.restype = ctypes.c_int
    l.jb_version.argtypes = []
    l.jb_device_sm_count.restype = ctypes.c_int
    l.jb_device_sm_count.argtypes = []
    l.jb_workspace_bytes.restype = SZ
    l.jb_workspace_bytes.argtypes = [I32, I32, I64, I32, I32, I32]
    l.jb_uneven_workspace_bytes.restype = SZ
    l.jb_uneven_workspace_bytes.argtypes = [I32, I32, I64, I32, I32, I64]
    l.jb_eigh_workspace_bytes.restype = SZ
    l.jb_eigh_workspace_bytes.argtypes = [I32, I64]
    l.jb_eigh_complex_workspace_bytes.restype = SZ
    l.jb_eigh_complex_workspace_bytes.argtypes = [I32, I64]
    for name in ("jb_eigh_f32", "jb_eigh_f64", "jb_eigh_c64", "jb_eigh_c128"):
        getattr(l, name).restype = ctypes.c_int
        getattr(l, name).argtypes = [P, P, P, P, P, I64, I32, F64, I32, P, SZ, P]
    l.jb_qr_workspace_bytes.restype = SZ
    l.jb_qr_workspace_bytes.argtypes = [I32, I32, I64, I32]
    for name in ("jb_qr_f32", "jb_qr_f64", "jb_qr_c64", "jb_qr_c128"):
        getattr(l, name).restype = ctypes.c_int
        getattr(l, name).argtypes = [P, P, P, I64, I32, I32, P, SZ, P]
    l.jb_svd_complex_workspace_bytes.restype = SZ
    l.jb_svd_complex_workspace_bytes.argtypes = [I32, I32, I64, I32]
    for name in ("jb_svd_batched_c64", "jb_svd_batched_c128"):
        getattr(l, name).restype = ctypes.c_int
        getattr(l, name).argtypes = [P, P, P, P, I64, I32, I32, F64, I32, P, P, P, SZ, P]
    l.jb_jacobi_rounds.restype = ctypes.c_int
    l.jb_jacobi_rounds.argtypes = [P, P, I32, I32, I32, I32, I32, F64, P, P]
    l.jb_svd_batched_f32.restype = ctypes.c_int
    l.jb_svd_batched_f32.argtypes = [P, P, P, P, I64, I32, I32, I32, I32, F64, I32, I32, P, P, P, SZ, P]
    l.jb_svd_batched_f64.restype = ctypes.c_int
    l.jb_svd_batched_f64.argtypes = [P, P, P, P, I64, I32, I32, I32, I32, F64, I32, P, P, P, SZ, P]
    l.jb_svd_uneven_f32.restype = ctypes.c_int
    l.jb_svd_uneven_f32.argtypes = [P, P, P, P, P, P, I64, I32, I32, F64, I32, I32, P, P, P, SZ, P]
    l.jb_svd_uneven_f32_ex.restype = ctypes.c_int
    l.jb_svd_uneven_f32_ex.argtypes = [P, P, P, P, P, P, I64, I32, I32, F64, I32, I32, I32, F64, P, P, P, SZ, P]
    l.jb_gemm_bf16.restype = ctypes.c_int
    l.jb_gemm_bf16.argtypes = [P, P, P, P, I32, P, I64, I64, I64, I64, I64, I64, I64, I64, I64, I64,
                               ctypes.c_float, ctypes.c_float, I32, P, P]
    l.jb_split_bf16.restype = ctypes.c_int
    l.jb_split_bf16.argtypes = [P, P, P, I64, P]
    l.jb_split3_bf16.restype = ctypes.c_int
    l.jb_split3_bf16.argtypes = [P, P, P, P, I64, P]
    l.jb_gemm_bf16x.restype = ctypes.c_int
    l.jb_gemm_bf16x.argtypes = [ctypes.POINTER(ctypes.c_void_p), ctypes.POINTER(ctypes.c_void_p), I32, P, I64, I64,
                                I64, I64, I64, I64, I64, I64, I64, I64, ctypes.c_float, ctypes.c_float, I32, P, P]
    l.jb_gemm_bf16x_rows.restype = ctypes.c_int
    l.jb_gemm_bf16x_rows.argtypes = [ctypes.POINTER(ctypes.c_void_p), ctypes.POINTER(ctypes.c_void_p), I32,
                                     ctypes.POINTER(ctypes.c_void_p), I32, P, I64, I64, I64, I64, I64, I64, I64,
                                     I64, I64, ctypes.c_float, P, P]
    VP = ctypes.POINTER(ctypes.c_void_p)
    l.jb_gemm_bf16x_rows2.restype = ctypes.c_int
    l.jb_gemm_bf16x_rows2.argtypes = [VP, VP, VP, I32, VP, VP, I32, P, I64, I64, I64, I64, I64, I64, I64, I64, I64,
                                      I64, I64, I64, I64, ctypes.c_float, P, P]
    FL = ctypes.c_float
    for name, args in (("jb_warm_prep_f32", [P, P, P, P, P, P, I64, I32, I32, P]),
                       ("jb_svd_warm_f32", [P, P, P, P, P, I64, I32, I32, I32, I32, F64, I32, I32, P, P, P, SZ, P]),
                       ("jb_transpose_bf16", [P, I32, P, I64, I64, I64, P]),
                       ("jb_bias_act", [P, P, P, I64, I64, I32, I32, P]),
                       ("jb_relu_backward", [P, P, P, I32, I64, P]),
                       ("jb_col_sum", [P, P, I64, I64, P]),
                       ("jb_mse_grad", [P, P, P, P, I64, FL, P]),
                       ("jb_adam", [P, P, P, P, P, P, I64, I64, FL, FL, FL, FL, I32, P]),
                       ("jb_gram_sketch", [P, P, I64, I32, I32, P]),
                       ("jb_block_eig_f64", [P, P, P, P, P, P, P, I64, I32, I32, F64, P, P]),
                       ("jb_block_eig_f64_ex", [P, P, P, P, P, P, P, I64, I32, I32, F64, P, I32, P]),
                       ("jb_block_eig_ws", [P, P, P, P, P, P, P, I64, I32, I32, F64, P, I32, P, SZ, P]),
                       ("jb_rows_scatter", [P, P, P, P, P, P, I64, I64, P]),
                       ("jb_rows_combine", [P, P, P, P, P, I64, I64, P]),
                       ("jb_gemm_f64acc", [P, P, P, I64, I64, I64, I64, I64, I64, P]),
                       ("jb_block_finish", [P, P, P, P, P, P, P, I64, I64, I32, I32, I32, P])):
        f = getattr(l, name)
        f.restype = ctypes.c_int
        f.argtypes = args
    l.jb_block_eig_workspace_bytes.restype = SZ
    l.jb_block_eig_workspace_bytes.argtypes = [I64, I32, I32]
    l.jb_complete_null_workspace_bytes.restype = SZ
    l.jb_complete_null_workspace_bytes.argtypes = [I32, I64, I64, I64]
    l.jb_complete_null.restype = ctypes.c_int
    l.jb_complete_null.argtypes = [P, P, I32, I64, I64, I64, P, P, SZ, P]
    l.jb_fma_loop_flops.restype = F64
    l.jb_fma_loop_flops.argtypes = [I32, I32]
    l.jb_fma_loop.restype = ctypes.c_int
    l.jb_fma_loop.argtypes = [I32, I32, I32, P, P]
    l.jb_svd_batched_f32_noalloc.restype = ctypes.c_int
    l.jb_svd_batched_f32_noalloc.argtypes = [P, P, P, P, I64, I32, I32, I32, I32, F64, I32, I32, P, P, P]
    return l


def load(path: Path | None = None):
    """Load the shared library (no device needed).  Raises if it is missing."""
    global _lib
    with _lock:
        if _lib is None:
            p = Path(path) if path else library_path()
            if not p.exists():
                raise RuntimeError(f"B200 Jacobi library not built: {p} is missing "
                                   "(run pavel-s_svd_b200/build.py); there is no CPU fallback")
            _lib = _declare(ctypes.CDLL(str(p)))
        return _lib


def lib():
    """The loaded library, for compute calls: also requires a CUDA device."""
    import torch
    if not torch.cuda.is_available():
        raise RuntimeError("the B200 Jacobi solver needs a CUDA device; there is no CPU fallback")
    return load()


def check(rc: int, what: str):
    if rc != JB_OK:
        raise RuntimeError(f"{what} failed: {RC_NAMES.get(rc, rc)} (code {rc})")
