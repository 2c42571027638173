"""Batched symmetric eigen-solver: the reference's jacobi_eigh on the GPU.

Counterpart of ``svdbench.standalone.primitives.jacobi_eigh(H, tol=None,
max_sweeps=30)`` (primitives.py:370-427, the syevj structure), which the
reference's gram_jacobi and polar_* families call (solvers.py:109, 170): a
two-sided cyclic Jacobi with round-robin pairs, one plane rotation per
active pair (|g_pq| > tol * max|G|), V accumulated, eigenvalues ascending.
Same signature, return value ``(w, V, sweeps)`` and error
(``RuntimeError('Hermitian Jacobi did not converge in N sweeps')``).  Real
float32/float64 or complex64/complex128 (Hermitian) CUDA tensors of shape
(b, n, n), n <= 255; the arithmetic is FP64 (complex128) for all of them;
eigenvalues come out real.  Other devices raise Unsupported: there is no CPU
fallback.
"""
from __future__ import annotations

import torch

from . import native as N
from .solvers import Unsupported


def jacobi_eigh(H: torch.Tensor, tol=None, max_sweeps=30):
    if H.ndim != 3 or H.shape[-1] != H.shape[-2]:
        raise ValueError('jacobi_eigh takes a (b, n, n) batch of square matrices')
    if H.device.type != 'cuda':
        raise Unsupported('the B200 eigen-solver runs on CUDA tensors only; there is no CPU fallback')
    if H.dtype not in (torch.float32, torch.float64, torch.complex64, torch.complex128):
        raise TypeError('supported dtypes: float32/64, complex64/128')
    if max_sweeps < 1:
        raise ValueError('max_sweeps must be positive')
    b, n, _ = H.shape
    if n > 255:
        raise Unsupported('jacobi_eigh on the B200 solver takes n <= 255')
    x = H.detach().resolve_conj().contiguous()      # the kernel reads memory: no lazy conjugate view
    real = H.real.dtype if H.is_complex() else H.dtype
    w = torch.empty(b, n, dtype=real, device=H.device)
    V = torch.empty(b, n, n, dtype=H.dtype, device=H.device)
    info = torch.zeros(2, max(b, 1), dtype=torch.int32, device=H.device)
    if b == 0:
        return w, V, 0
    lib = N.lib()
    ws_bytes = int(lib.jb_eigh_complex_workspace_bytes(n, b) if H.is_complex() else lib.jb_eigh_workspace_bytes(n, b))
    ws = torch.empty(max(ws_bytes, 8), dtype=torch.uint8, device=H.device)
    fn = {torch.float32: lib.jb_eigh_f32, torch.float64: lib.jb_eigh_f64, torch.complex64: lib.jb_eigh_c64,
          torch.complex128: lib.jb_eigh_c128}[H.dtype]
    with torch.cuda.device(H.device):
        st = torch.cuda.current_stream(H.device).cuda_stream
        N.check(fn(x.data_ptr(), w.data_ptr(), V.data_ptr(), info[0].data_ptr(), info[1].data_ptr(), b, n,
                   float(tol or 0.0), int(max_sweeps), ws.data_ptr(), ws.numel(), st), 'jb_eigh')
        host = info[:, :b].cpu()
    if bool((host[1] != N.ST_OK).any()):
        raise RuntimeError(f"Hermitian Jacobi did not converge in {max_sweeps} sweeps")  # primitives.py:422-423
    return w, V, int(host[0].max())
