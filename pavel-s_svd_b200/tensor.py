"""Thin torch-facing wrappers of the tensor-core entry points (jb_gemm_bf16,
jb_split_bf16).  Buffers are torch tensors on the current device; the work is
enqueued on the current stream."""
from __future__ import annotations

import torch

from . import native as N


def _ptr(t):
    return None if t is None else t.data_ptr()


def split_bf16(x: torch.Tensor):
    """(hi, lo) BF16 parts of a float32 tensor: hi = bf16(x), lo = bf16(x - hi)."""
    x = x.contiguous()
    hi = torch.empty(x.shape, dtype=torch.bfloat16, device=x.device)
    lo = torch.empty(x.shape, dtype=torch.bfloat16, device=x.device)
    N.check(N.lib().jb_split_bf16(x.data_ptr(), hi.data_ptr(), lo.data_ptr(), x.numel(),
                                  torch.cuda.current_stream(x.device).cuda_stream), "jb_split_bf16")
    return hi, lo


def gemm(a, b, c=None, *, a_lo=None, b_lo=None, alpha=1.0, beta=0.0, split_k=1, error_flag=None):
    """C = alpha * A @ B^T (+ beta C) on the tensor cores.

    a: (..., M, K) bf16, b: (..., N, K) bf16 (row-major, K contiguous).  With
    a_lo/b_lo the compensated 3xBF16 product (a + a_lo)(b + b_lo)^T without
    the lo*lo term.  Returns C (..., M, N) float32."""
    if a.dtype != torch.bfloat16 or b.dtype != torch.bfloat16:
        raise TypeError("gemm takes bf16 operands")
    batch_shape = a.shape[:-2]
    M, K = a.shape[-2:]
    Nn = b.shape[-2]
    bsz = 1
    for d in batch_shape:
        bsz *= d
    a3 = a.reshape(bsz, M, K)
    b3 = b.reshape(-1, Nn, K)
    if b3.shape[0] != bsz:
        raise ValueError("batch shapes of a and b differ")
    if c is None:
        c = torch.empty(*batch_shape, M, Nn, dtype=torch.float32, device=a.device)
        beta = 0.0
    mode = N.GEMM_SPLIT3 if a_lo is not None else N.GEMM_PLAIN
    lda = a3.stride(1)
    ldb = b3.stride(1)
    rc = N.lib().jb_gemm_bf16(_ptr(a3), _ptr(a_lo), _ptr(b3), _ptr(b_lo), mode, c.data_ptr(), M, Nn, K, lda, ldb,
                              c.stride(-2), bsz, a3.stride(0), b3.stride(0), M * Nn if c.dim() == 2 else c.stride(-3),
                              float(alpha), float(beta), int(split_k), _ptr(error_flag),
                              torch.cuda.current_stream(a.device).cuda_stream)
    N.check(rc, "jb_gemm_bf16")
    return c
