"""The reference's block Jacobi in rounds (svdbench/standalone/solvers.py:30-68
of uncle-Slava/Pavel-s_SVD) for float64, complex64 and complex128 input and
for float32 matrices too small for the tensor-core solver (blocked.py).

The columns are cut into groups of ``block_size``; a sweep plays the
round-robin tournament of the groups (primitives.py:309-313), and each pair
(i, j) of a round is orthogonalised by the one-sided Jacobi of its columns
W[:, cols]: W[:, cols] <- W[:, cols] V_ij, V[:, cols] <- V[:, cols] V_ij.
The pairs of one round touch disjoint columns, so applying them one after
the other (the reference) or all at once (here) gives the same result:

  * all pair subproblems of a round with the same column count are ONE call
    of this library's batched Jacobi (b x pairs matrices of m x |cols|,
    jb_svd_batched_f64 / _c64 / _c128, or the mixed FP32/FP64 kernels for
    float32), instead of one solve per pair;
  * only V_ij of a pair solve is used, and a one-sided Jacobi sees its matrix
    only through the column Gram W^H W; so pair subproblems taller than
    QR_ROWS are first reduced to their R factor (this library's Householder
    QR, W = Q R, R^H R = W^H W) and the Jacobi runs on the |cols| x |cols| R:
    the same rotations and sweeps in exact arithmetic, far less work;
  * the rotations W[:, cols] V_ij and V[:, cols] V_ij and the convergence
    check's Gram W^H W are library GEMMs in the input dtype, as the
    reference's matmuls are.

After a sweep the largest correlation |g_pq| / sqrt(g_pp g_qq) between live
columns decides convergence (tol defaults to 40 eps); then the columns are
sorted by norm and normalised, null columns completed (solvers.py:18-21).
"""
from __future__ import annotations

import torch

from . import qr as Q

QR_ROWS = 128   # pair subproblems with more rows than this are reduced to R first


def round_robin(n):
    """Circle-method tournament of n (even) players: n - 1 rounds of n // 2
    disjoint pairs (p < q); player 0 stays, the last moves to slot 1
    (primitives.py:309-313)."""
    players = list(range(n))
    for _ in range(n - 1):
        yield [(min(players[i], players[n - 1 - i]), max(players[i], players[n - 1 - i])) for i in range(n // 2)]
        players = [players[0]] + [players[-1]] + players[1:-1]


def groups_of(n, width):
    """Column groups of `width` (the last one shorter), padded with an empty
    group to an even count (solvers.py:35, 38-39)."""
    groups = [list(range(j, min(j + width, n))) for j in range(0, n, width)]
    if len(groups) % 2:
        groups.append([])
    return groups


def schedule(n, width, device):
    """Per round, the pairs that have at least two columns (solvers.py:46-48),
    bucketed by column count: a list of (pairs, count) index tensors."""
    groups = groups_of(n, width)
    rounds = []
    for pairs in round_robin(len(groups)):
        by_count = {}
        for i, j in pairs:
            cols = groups[i] + groups[j]
            if len(cols) >= 2:
                by_count.setdefault(len(cols), []).append(cols)
        rounds.append([torch.tensor(c, dtype=torch.long, device=device) for c in by_count.values()])
    return rounds


def finish_columns(w, s, complete):
    """U = W / sigma for the columns above eps * max(m, n) * sigma_1, the
    others zeroed in sigma and completed in U (solvers.py:18-21)."""
    eps = torch.finfo(w.real.dtype).eps
    keep = s > eps * max(w.shape[-2:]) * s[:, :1]
    u = w / torch.where(keep, s, torch.ones_like(s))[:, None, :].to(w.dtype)
    return complete(u, keep), torch.where(keep, s, torch.zeros_like(s))


def block_jacobi(a, stats, opts, jacobi, check, complete):
    """Block Jacobi of a batch of tall matrices a (b, m, n), m >= n, with at
    least two column groups.  `jacobi(y)` enqueues the one-sided Jacobi of a
    batch of pair subproblems and returns (_, _, v) with v (., c, c)
    orthogonal / unitary, columns by descending sigma; `check()` raises the
    errors of the solves enqueued since its last call (called once per
    sweep); `complete(u, keep)` fills the columns of u not in keep.  Returns
    U (b, m, n), sigma (b, n) descending, V (b, n, n).  Raises
    RuntimeError('block Jacobi did not converge') after max_sweeps (default
    30) sweeps (solvers.py:59-60)."""
    b, m, n = a.shape
    if b == 0:
        stats['block_sweeps'] = 0
        return a.new_zeros(b, m, n), a.real.new_zeros(b, n), a.new_zeros(b, n, n)
    width = opts.get('block_size', 4)
    dev = a.device
    rounds = schedule(n, width, dev)
    w = a.clone()
    v = torch.eye(n, dtype=a.dtype, device=dev).expand(b, n, n).clone()
    eps = torch.finfo(a.real.dtype).eps
    tol = opts.get('tol') or 40 * eps
    tiny = torch.finfo(a.real.dtype).tiny
    max_sweeps = opts.get('max_sweeps', 30)
    converged = False
    sweep = 0
    for sweep in range(max_sweeps):
        for buckets in rounds:
            for idx in buckets:
                k, c = idx.shape
                flat = idx.reshape(-1)
                wy = w[:, :, flat].reshape(b, m, k, c).permute(2, 0, 1, 3)     # (pairs, b, m, c)
                vy = v[:, :, flat].reshape(b, n, k, c).permute(2, 0, 1, 3)
                y = wy.reshape(k * b, m, c)
                if m > QR_ROWS:
                    y = Q.qr(y)[1]
                _, _, vv = jacobi(y)
                vv = vv.reshape(k, b, c, c)
                w[:, :, flat] = (wy @ vv).permute(1, 2, 0, 3).reshape(b, m, k * c)
                v[:, :, flat] = (vy @ vv).permute(1, 2, 0, 3).reshape(b, n, k * c)
        check()
        g = w.mH @ w
        d = g.diagonal(dim1=-2, dim2=-1).real.clamp_min(0)
        root = d.sqrt()
        denom = root[:, :, None] * root[:, None, :]
        g.diagonal(dim1=-2, dim2=-1).zero_()
        live = d > (eps * max(m, n)) ** 2 * d.amax(-1, keepdim=True)
        corr = torch.where(live[:, :, None] & live[:, None, :], g.abs() / denom.clamp_min(tiny),
                           torch.zeros_like(denom))
        if bool(corr.max() <= tol):
            converged = True
            break
    if not converged:
        raise RuntimeError('block Jacobi did not converge')
    s = w.abs().square().sum(1).sqrt()
    order = s.argsort(-1, descending=True)
    s = s.gather(1, order)
    w = w.gather(2, order[:, None].expand_as(w))
    v = v.gather(2, order[:, None].expand_as(v))
    u, s = finish_columns(w, s, complete)
    stats['block_sweeps'] = sweep + 1
    return u, s, v


def raw(x, stats, opts, jacobi, check, complete):
    """Wide input through its conjugate transpose (solvers.py:224-227).  The
    caller sends a matrix with a single column group to the plain Jacobi
    (:36-37)."""
    if x.shape[-2] < x.shape[-1]:
        u, s, v = raw(x.mH.resolve_conj().contiguous(), stats, opts, jacobi, check, complete)
        return v, s, u
    return block_jacobi(x, stats, opts, jacobi, check, complete)
