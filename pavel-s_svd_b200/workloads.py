"""Seeded synthetic inputs for the five Jacobi workloads.

Conventions follow the reference input generator (svdbench/matrices.py:8-62):
NumPy ``default_rng(seed)``, generation in float64, one cast to the target
dtype at the end, orthogonal factors from ``np.linalg.qr`` of Gaussian draws.
The draw order inside each generator is part of its definition and is fixed.

  plain_single     256x128 f32, s_i = 10^(-4 i/127), seed 0
  uneven_batch     8192 f32 matrices, n ~ U{8..64}, m ~ U{n..2n}, N(0,1), seed 1
  clustered_large  4096x1024 f32, 64 clusters x 16 values, seed 2
  tall_lowrank     8192x2048 f32 rank-64 product + N(0, (1e-6)^2) noise, seed 3
  warm_family      65536 f32 128x64 matrices, V = expm(0.3 L(theta)), seed 4
"""
from __future__ import annotations

import numpy as np

__all__ = ["plain_single", "uneven_batch", "uneven_sizes", "clustered_large",
           "tall_lowrank", "warm_family", "pack_uneven"]


def plain_single(seed=0, m=256, n=128, decades=4.0):
    """A = U diag(s) V^T, U = qr(G m x n).Q, V = qr(G n x n).Q, s_i = 10^(-decades i/(n-1))."""
    rng = np.random.default_rng(seed)
    u, _ = np.linalg.qr(rng.standard_normal((m, n)), mode="reduced")
    v, _ = np.linalg.qr(rng.standard_normal((n, n)), mode="reduced")
    s = 10.0 ** (-decades * np.arange(n) / (n - 1))
    return np.ascontiguousarray(((u * s) @ v.T).astype(np.float32))


def uneven_sizes(count=8192, seed=1, n_lo=8, n_hi=64):
    """Shapes of the uneven batch: all n first, then all m (m ~ U{n..2n})."""
    rng = np.random.default_rng(seed)
    n = rng.integers(n_lo, n_hi + 1, size=count)
    m = rng.integers(n, 2 * n + 1)
    return rng, m.astype(np.int64), n.astype(np.int64)


def uneven_batch(count=8192, seed=1, n_lo=8, n_hi=64, dtype=np.float32):
    """List of `count` matrices with iid N(0,1) entries; draws follow the shapes
    in matrix order (row-major m x n per matrix)."""
    rng, m, n = uneven_sizes(count, seed, n_lo, n_hi)
    return [rng.standard_normal((int(mi), int(ni))).astype(dtype) for mi, ni in zip(m, n)]


def pack_uneven(mats):
    """Concatenate row-major matrices into one flat buffer.

    Returns (flat, m, n, offsets) with offsets in elements.  Each matrix starts
    on a 4-element boundary so vector loads stay aligned."""
    m = np.array([a.shape[0] for a in mats], np.int64)
    n = np.array([a.shape[1] for a in mats], np.int64)
    sizes = (m * n + 3) // 4 * 4
    offsets = np.zeros(len(mats), np.int64)
    offsets[1:] = np.cumsum(sizes)[:-1]
    flat = np.zeros(int(sizes.sum()), mats[0].dtype)
    for a, o in zip(mats, offsets):
        flat[o:o + a.size] = a.ravel()
    return flat, m, n, offsets


def clustered_large(seed=2, m=4096, n=1024, clusters=64, size=16, decades=6.0, gap=1e-6):
    """Haar-like U (m x n), V (n x n); 64 cluster centres log-spaced over 10^-6;
    inside a cluster consecutive values differ by the relative gap 1e-6."""
    rng = np.random.default_rng(seed)
    u, _ = np.linalg.qr(rng.standard_normal((m, n)), mode="reduced")
    v, _ = np.linalg.qr(rng.standard_normal((n, n)), mode="reduced")
    centres = np.logspace(0.0, -decades, clusters)
    s = (centres[:, None] * (1.0 - gap) ** np.arange(size)[None, :]).ravel()[:n]
    return np.ascontiguousarray(((u * s) @ v.T).astype(np.float32))


def tall_lowrank(seed=3, m=8192, n=2048, rank=64, noise=1e-6):
    """B = G1 (m x r) G2 (r x n) scaled to spectral norm 1, plus iid N(0, noise^2)."""
    rng = np.random.default_rng(seed)
    g1 = rng.standard_normal((m, rank))
    g2 = rng.standard_normal((rank, n))
    # ||G1 G2||_2 from the r x r core: G1 = Q1 R1, G2^T = Q2 R2 -> sigma(R1 R2^T).
    r1 = np.linalg.qr(g1, mode="r")
    r2 = np.linalg.qr(g2.T, mode="r")
    top = np.linalg.svd(r1 @ r2.T, compute_uv=False)[0]
    b = (g1 @ g2) / top
    b += noise * rng.standard_normal((m, n))
    return np.ascontiguousarray(b.astype(np.float32))


def skew_basis(seed=4, n=64, dims=16):
    """The fixed seeded linear map L: R^dims -> skew(n), as `dims` skew matrices
    K_i = (G_i - G_i^T) / sqrt(2 n), drawn first from the generator."""
    rng = np.random.default_rng(seed)
    g = rng.standard_normal((dims, n, n))
    return rng, (g - np.swapaxes(g, -1, -2)) / np.sqrt(2.0 * n)


def _expm_skew(k):
    """exp(K) for real skew-symmetric K, batched: K = i H with H Hermitian, so
    exp(K) = Q diag(exp(i w)) Q^H from the Hermitian eigendecomposition."""
    w, q = np.linalg.eigh(-1j * k)
    e = np.exp(1j * w)
    return np.real((q * e[..., None, :]) @ np.conj(np.swapaxes(q, -1, -2)))


def family_v(theta, seed=4, n=64, dims=16, strength=0.3, device=None):
    """The generator's V(theta) = expm(strength * sum_i theta_i K_i) for given
    theta (count, dims): the smooth frame of the warm-start family."""
    _, basis = skew_basis(seed, n, dims)
    k = strength * np.einsum("bd,dij->bij", np.asarray(theta), basis)
    if device is None:
        return _expm_skew(k)
    import torch
    return torch.linalg.matrix_exp(torch.from_numpy(k).to(device)).float()


def warm_family(count=65536, seed=4, m=128, n=64, dims=16, strength=0.3, decades=3.0,
                chunk=4096, device=None):
    """A = U diag(s) V^T with U = qr(G m x n).Q, log10 s ~ U[-decades, 0] (unsorted),
    V = expm(strength * sum_i theta_i K_i), theta ~ N(0, I_dims).

    Returns (A float32 (count, m, n), theta float64 (count, dims)).  Draw order:
    the skew basis, then all theta, then per chunk the U Gaussians and the
    spectra.  With `device` (a CUDA torch device) the QR and exp steps run
    in float64 on that device (same draws; results equal to rounding)."""
    rng, basis = skew_basis(seed, n, dims)
    theta = rng.standard_normal((count, dims))
    out = np.empty((count, m, n), np.float32)
    for lo in range(0, count, chunk):
        hi = min(lo + chunk, count)
        g = rng.standard_normal((hi - lo, m, n))
        s = 10.0 ** (-decades * rng.random((hi - lo, n)))
        k = strength * np.einsum("bd,dij->bij", theta[lo:hi], basis)
        if device is None:
            u, _ = np.linalg.qr(g, mode="reduced")
            v = _expm_skew(k)
            out[lo:hi] = ((u * s[:, None, :]) @ np.swapaxes(v, -1, -2)).astype(np.float32)
        else:
            import torch
            gt = torch.from_numpy(g).to(device)
            u = torch.linalg.qr(gt, mode="reduced")[0]
            v = torch.linalg.matrix_exp(torch.from_numpy(k).to(device))
            a = (u * torch.from_numpy(s).to(device)[:, None, :]) @ v.transpose(-1, -2)
            out[lo:hi] = a.float().cpu().numpy()
    return out, theta
