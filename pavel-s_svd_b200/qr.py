"""Householder QR on the GPU and the reference's Jacobi-based solvers built on
it: 'qr' and 'tsqr' (a QR, then the one-sided Jacobi of the small R factor)
and the projected 'randomized', 'subspace' and 'block_krylov' solvers (a
range basis from QRs of sketches, then the Jacobi of the projected matrix).

Mirrors svdbench/standalone of uncle-Slava/Pavel-s_SVD:
  qr       primitives.py:41-89 (householder_vec, qr) -> jb_qr_f32 / _f64 / _c64 / _c128
  tsqr     solvers.py:71-96
  partial  solvers.py:185-220 (with _sketch, :179-182)
  raw      solvers.py:224-230, 245-248, 253-254 for these methods
The QRs and the small Jacobi solves run on this library's sm_100a kernels;
the products around them (A @ Omega, Q @ U, ...) are plain library GEMMs in
the input dtype, as the reference's matmuls are.
"""
from __future__ import annotations

import torch

from . import native as N

PARTIAL = ('randomized', 'subspace', 'block_krylov')
_QR = {torch.float32: 'jb_qr_f32', torch.float64: 'jb_qr_f64', torch.complex64: 'jb_qr_c64',
       torch.complex128: 'jb_qr_c128'}
METHODS = ('qr', 'tsqr') + PARTIAL

_ws = {}


def _workspace(nbytes, device):
    """The QR scratch of the current stream on `device` (launches on different
    streams may run at the same time and must not share it)."""
    key = (torch.device(device), torch.cuda.current_stream(device).cuda_stream)
    buf = _ws.get(key)
    nbytes = max(int(nbytes), 256)
    if buf is None or buf.numel() < nbytes:
        buf = torch.empty(nbytes, dtype=torch.uint8, device=device)
        _ws[key] = buf
    return buf


def qr(a: torch.Tensor):
    """Householder QR of a batch of tall matrices (b, m, n), m >= n, float32,
    float64, complex64 or complex128 on a CUDA device: Q (b, m, n), R (b, n,
    n) upper triangular, in the input dtype (primitives.py:74-89, computed as
    the reference does, in that dtype)."""
    if a.ndim != 3 or a.shape[-2] < a.shape[-1]:
        raise ValueError('qr expects a (batch, m, n) tensor with m >= n')
    if a.dtype not in _QR:
        raise TypeError('qr supports float32, float64, complex64 and complex128')
    if a.device.type != 'cuda':
        raise RuntimeError('the B200 QR runs on CUDA tensors only; there is no CPU fallback')
    b, m, n = a.shape
    x = a.resolve_conj().contiguous()   # the kernel reads memory: no lazy conjugate view
    q = torch.empty(b, m, n, dtype=a.dtype, device=a.device)
    r = torch.empty(b, n, n, dtype=a.dtype, device=a.device)
    if b == 0:
        return q, r
    lib = N.lib()
    elem = x.element_size()
    ws = _workspace(lib.jb_qr_workspace_bytes(m, n, b, elem), a.device)
    stream = torch.cuda.current_stream(a.device).cuda_stream
    fn = getattr(lib, _QR[a.dtype])
    N.check(fn(x.data_ptr(), q.data_ptr(), r.data_ptr(), b, m, n, ws.data_ptr(), ws.numel(), stream), 'jb_qr')
    return q, r


def tsqr(a: torch.Tensor, rows: int, stats: dict):
    """Tall-skinny QR (solvers.py:71-96): QRs of row tiles of `rows` rows (a
    last tile shorter than n joins the one before), then a binary reduction
    tree over the stacked R factors with the tree back-transformation of Q.
    The leaf QRs of equal height run as one batched launch, as do the QRs of
    one tree level."""
    b, m, n = a.shape
    rows = max(rows, n)
    if m <= rows:
        return qr(a)
    spans = []
    for start in range(0, m, rows):
        end = min(start + rows, m)
        if end - start < n:
            start = spans.pop()[0]
        spans.append((start, end))
    stats['tsqr_leaves'] = len(spans)
    leaves = [None] * len(spans)
    heights = sorted({e - s for s, e in spans})
    for h in heights:
        idx = [i for i, (s, e) in enumerate(spans) if e - s == h]
        q, r = qr(torch.cat([a[:, s:e] for s, e in (spans[i] for i in idx)], 0))
        for k, i in enumerate(idx):
            leaves[i] = (q[k * b:(k + 1) * b], r[k * b:(k + 1) * b])
    nodes = leaves
    while len(nodes) > 1:
        pairs = [(nodes[i], nodes[i + 1]) for i in range(0, len(nodes) - 1, 2)]
        q, r = qr(torch.cat([torch.cat([r1, r2], -2) for (_, r1), (_, r2) in pairs], 0))
        nxt = []
        for k, ((q1, _), (q2, _)) in enumerate(pairs):
            qk, rk = q[k * b:(k + 1) * b], r[k * b:(k + 1) * b]
            nxt.append((torch.cat([q1 @ qk[:, :n], q2 @ qk[:, n:]], -2), rk))
        if len(nodes) % 2:
            nxt.append(nodes[-1])
        nodes = nxt
    return nodes[0]


def sketch(a: torch.Tensor, columns: int, seed: int):
    """The reference's Gaussian test matrix (solvers.py:179-182): the same
    generator, seed and call, so on the same device the same numbers."""
    gen = torch.Generator(device=a.device).manual_seed(seed)
    return torch.randn(a.shape[0], a.shape[-1], columns, dtype=a.dtype, device=a.device, generator=gen)


def partial(a: torch.Tensor, stats: dict, opts: dict, method: str, jacobi):
    """'randomized', 'subspace', 'block_krylov' (solvers.py:185-220): a range
    basis Q from QRs of A Omega and of its power / Krylov iterations, then the
    Jacobi SVD of Q^H A (wide: solved through its transpose); returns the
    first `rank` triplets.  `jacobi(x)` is the small solve."""
    k = opts.get('rank', min(a.shape[-2:]))
    ell = min(k + opts.get('oversample', 8), min(a.shape[-2:]))
    omega = opts.get('initial_basis')
    if omega is None:
        omega = sketch(a, ell, opts.get('seed', 20261011))
    else:
        if omega.ndim == 2:
            omega = omega[None]
        if omega.shape != (a.shape[0], a.shape[-1], ell):
            raise ValueError('initial_basis shape must match batch, n, rank+oversample')
        omega = omega.to(device=a.device, dtype=a.dtype)
        stats['warm_started'] = True
    q, _ = qr(a @ omega)
    bases = [q]
    iterations = opts.get('iterations', 2)
    for _ in range(iterations):
        z, _ = qr(a.mH @ q)
        y = a @ z
        if method == 'block_krylov':
            joined = torch.cat(bases, -1)
            available = a.shape[-2] - joined.shape[-1]
            if available <= 0:
                break
            for _ in range(2):
                y = y - joined @ (joined.mH @ y)
            q, _ = qr(y[:, :, :min(ell, available)].contiguous())
            bases.append(q)
        else:
            q, _ = qr(y)
    if method == 'block_krylov':
        q, _ = qr(torch.cat(bases, -1))
    small = q.mH @ a
    u, s, v = jacobi(small)
    stats.update(sketch_columns=ell, range_columns=q.shape[-1], power_iterations=iterations)
    return (q @ u)[:, :, :k], s[:, :k], v[:, :, :k]


def raw(x: torch.Tensor, method: str, stats: dict, opts: dict, jacobi):
    """The reference's _raw for these methods (solvers.py:224-230, 245-248,
    253-254): wide input through its transpose except for the projected
    solvers; 'qr' / 'tsqr' solve R by Jacobi and return U = Q U_R."""
    if x.shape[-2] < x.shape[-1] and method not in PARTIAL:
        u, s, v = raw(x.mH.resolve_conj().contiguous(), method, stats, opts, jacobi)
        return v, s, u
    if method in ('qr', 'tsqr'):
        q, r = qr(x) if method == 'qr' else tsqr(x, opts.get('tile_rows', 4 * x.shape[-1]), stats)
        u, s, v = jacobi(r)
        return q @ u, s, v
    return partial(x, stats, opts, method, jacobi)
