"""Thin torch-facing wrappers of the tensor-core entry points (jb_gemm_bf16,
jb_split_bf16).  Buffers are torch tensors on the current device; the work is
enqueued on the current stream."""
from __future__ import annotations

import ctypes

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


def split3_bf16(x: torch.Tensor):
    """(hi, mid, lo) BF16 parts of a float32 tensor (x ~ hi + mid + lo)."""
    x = x.contiguous()
    parts = [torch.empty(x.shape, dtype=torch.bfloat16, device=x.device) for _ in range(3)]
    N.check(N.lib().jb_split3_bf16(x.data_ptr(), parts[0].data_ptr(), parts[1].data_ptr(), parts[2].data_ptr(),
                                   x.numel(), torch.cuda.current_stream(x.device).cuda_stream), "jb_split3_bf16")
    return tuple(parts)


def _mode(ns, b_mn, chain128, syrk):
    return ({1: N.GEMM_PLAIN, 2: N.GEMM_SPLIT3, 3: N.GEMM_SPLIT6}[ns] | (N.GEMM_B_MN if b_mn else 0) |
            (N.GEMM_CHAIN128 if chain128 else 0) | (N.GEMM_SYRK if syrk else 0))


def gemm_parts(a_parts, b_parts, c=None, *, b_mn=False, alpha=1.0, beta=0.0, split_k=1, error_flag=None,
               chain128=False, syrk=False):
    """General entry over split parts (1, 2 or 3 of them): C = alpha A B^T (+ beta C).

    a parts: (batch, M, K) bf16; b parts: (batch, N, K) bf16, or with b_mn
    (batch, K, N) bf16 (N contiguous).  With syrk, B is A (C = A A^T) and
    b_parts is ignored.  chain128 keeps every accumulation chain <= 128 long
    (several tensor-memory accumulators per CTA).  Returns C (batch, M, N)
    float32."""
    if syrk:
        b_parts = a_parts
    a0, b0 = a_parts[0], b_parts[0]
    if a0.dim() == 2:
        a_parts = [x[None] for x in a_parts]
    if b0.dim() == 2:
        b_parts = [x[None] for x in b_parts]
    a0, b0 = a_parts[0], b_parts[0]
    bsz, M, K = a0.shape
    Nn = b0.shape[-1] if b_mn else b0.shape[-2]
    if c is None:
        c = torch.empty(bsz, M, Nn, dtype=torch.float32, device=a0.device)
        beta = 0.0
    c3 = c if c.dim() == 3 else c[None]
    ns = len(a_parts)
    mode = _mode(ns, b_mn, chain128, syrk)
    A = (ctypes.c_void_p * 3)(*[x.data_ptr() for x in a_parts] + [None] * (3 - ns))
    B = (ctypes.c_void_p * 3)(*[x.data_ptr() for x in b_parts] + [None] * (3 - ns))
    rc = N.lib().jb_gemm_bf16x(A, B, mode, c3.data_ptr(), M, Nn, K, a0.stride(1), b0.stride(1), c3.stride(1),
                               bsz, a0.stride(0), b0.stride(0), c3.stride(0), float(alpha), float(beta), int(split_k),
                               _ptr(error_flag), torch.cuda.current_stream(a0.device).cuda_stream)
    N.check(rc, "jb_gemm_bf16x")
    return c


def gemm_parts_rows(a_parts, b_parts, out_parts, row_map=None, *, b_mn=False, alpha=1.0, chain128=True,
                    error_flag=None):
    """alpha A B^T written as BF16 split parts into mapped rows:
    row r of batch z -> row row_map[z * M + r] of every out part (2-D,
    rows x L, L >= N).  len(out_parts) parts (1..3) are written."""
    a0, b0 = a_parts[0], b_parts[0]
    bsz, M, K = a0.shape
    Nn = b0.shape[-1] if b_mn else b0.shape[-2]
    ns = len(a_parts)
    A = (ctypes.c_void_p * 3)(*[x.data_ptr() for x in a_parts] + [None] * (3 - ns))
    B = (ctypes.c_void_p * 3)(*[x.data_ptr() for x in b_parts] + [None] * (3 - ns))
    O = (ctypes.c_void_p * 3)(*[x.data_ptr() for x in out_parts] + [None] * (3 - len(out_parts)))
    rc = N.lib().jb_gemm_bf16x_rows(A, B, _mode(ns, b_mn, chain128, False), O, len(out_parts), _ptr(row_map),
                                    out_parts[0].shape[-1], M, Nn, K, a0.stride(1), b0.stride(1), bsz,
                                    a0.stride(0), b0.stride(0), float(alpha), _ptr(error_flag),
                                    torch.cuda.current_stream(a0.device).cuda_stream)
    N.check(rc, "jb_gemm_bf16x_rows")


def gemm_parts_rows2(a_parts, b_parts, out_parts, b2_parts, out2_parts, row_map=None, *, b_mn=False, alpha=1.0,
                     chain128=True, error_flag=None):
    """Two gemm_parts_rows products sharing A and the row map, in one launch
    (jb_gemm_bf16x_rows2): alpha A B^T into out_parts and alpha A B2^T into
    out2_parts."""
    a0, b0, c0 = a_parts[0], b_parts[0], b2_parts[0]
    bsz, M, K = a0.shape
    Nn = b0.shape[-1] if b_mn else b0.shape[-2]
    N2 = c0.shape[-1] if b_mn else c0.shape[-2]
    ns = len(a_parts)
    arr = lambda xs: (ctypes.c_void_p * 3)(*[x.data_ptr() for x in xs] + [None] * (3 - len(xs)))
    rc = N.lib().jb_gemm_bf16x_rows2(arr(a_parts), arr(b_parts), arr(b2_parts), _mode(ns, b_mn, chain128, False),
                                     arr(out_parts), arr(out2_parts), len(out_parts), _ptr(row_map),
                                     out_parts[0].shape[-1], out2_parts[0].shape[-1], M, Nn, N2, K, a0.stride(1),
                                     b0.stride(1), c0.stride(1), bsz, a0.stride(0), b0.stride(0), c0.stride(0),
                                     float(alpha), _ptr(error_flag), torch.cuda.current_stream(a0.device).cuda_stream)
    N.check(rc, "jb_gemm_bf16x_rows2")


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
