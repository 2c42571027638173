"""CPU oracle: NumPy restatement of the reference one-sided Jacobi SVD path.

TEST INFRASTRUCTURE ONLY.  Only ``tests/``, ``__graft_entry__.smoke()`` and the
``cpu_baseline`` / ``--impl reference`` legs of ``bench.py`` may import this
module, and only as the checker (or the timed CPU baseline).  The product path
(``pavel-s_svd_b200``) never imports it and has no CPU fallback.

Every function restates the algorithm of the reference project
(uncle-Slava/Pavel-s_SVD) step by step with NumPy arrays, batched in lock-step
exactly like the PyTorch original:

  round_robin            svdbench/standalone/primitives.py:309-313
  jacobi_svd             svdbench/standalone/primitives.py:316-367
  jacobi_eigh            svdbench/standalone/primitives.py:370-427 (real dtypes)
  complete_null_columns  svdbench/standalone/primitives.py:430-455
  complete_basis         svdbench/standalone/primitives.py:458-467
  householder_vec / qr   svdbench/standalone/primitives.py:41-89
  tsqr                   svdbench/standalone/solvers.py:71-96
  partial                svdbench/standalone/solvers.py:185-220 (given initial_basis)
  finish_columns         svdbench/standalone/solvers.py:18-21
  block_jacobi           svdbench/standalone/solvers.py:30-68
  svd                    svdbench/standalone/solvers.py:264-310 ('jacobi', 'block_jacobi', 'qr',
                         'tsqr', 'randomized', 'subspace', 'block_krylov')
  raw                    svdbench/standalone/solvers.py:224-248
  reference / validate   svdbench/metrics.py:6-66 (FP64 LAPACK gesvd truth)

Parity of this restatement is pinned against fixtures produced by the
reference itself (tests/golden/make_golden.py, tests/test_oracle.py).
"""
from __future__ import annotations

import numpy as np

__all__ = ["round_robin", "jacobi_svd", "jacobi_eigh", "complete_null_columns", "complete_basis",
           "householder_vec", "qr", "tsqr", "partial", "svd", "raw", "reference", "validate", "eps"]


def _real(dt):
    dt = np.dtype(dt)
    return {np.dtype(np.complex64): np.dtype(np.float32),
            np.dtype(np.complex128): np.dtype(np.float64)}.get(dt, dt)


def eps(dt):
    """Machine epsilon of the real part type (primitives.py:26-31)."""
    return float(np.finfo(_real(dt)).eps)


def tiny(dt):
    return float(np.finfo(_real(dt)).tiny)


def round_robin(n):
    """Circle-method tournament: n-1 rounds of n//2 disjoint (p<q) pairs.

    Player 0 stays fixed; the last player moves to slot 1 each round
    (primitives.py:309-313)."""
    players = list(range(n))
    for _ in range(n - 1):
        yield [(min(players[i], players[n - 1 - i]), max(players[i], players[n - 1 - i]))
               for i in range(n // 2)]
        players = [players[0]] + [players[-1]] + players[1:-1]


def jacobi_svd(A, tol=None, max_sweeps=30):
    """One-sided Hestenes Jacobi, round-robin ordering, lock-step batch.

    A: (b, m, n) with m >= n.  Returns U (b,m,n), s (b,n) descending, V (b,n,n),
    sweeps (primitives.py:316-367).  Raises RuntimeError when not converged
    (primitives.py:354-355)."""
    A = np.asarray(A)
    dt = A.dtype
    rdt = _real(dt)
    b, m, n = A.shape
    padded = n % 2 == 1
    W = A.copy()
    if padded:                                                    # :320-323
        W = np.concatenate([W, np.zeros((b, m, 1), dt)], -1)
        n += 1
    V = np.broadcast_to(np.eye(n, dtype=dt), (b, n, n)).copy()    # :324
    e = eps(dt)
    tol = tol or 10 * e                                           # :325
    sched = [(np.array([p for p, _ in prs]), np.array([q for _, q in prs])) for prs in round_robin(n)]
    sweeps = 0
    off = rdt.type(0)
    one = rdt.type(1)
    for sweeps in range(1, max_sweeps + 1):                       # :328
        off = rdt.type(0)
        for P, Q in sched:                                        # :330
            wp, wq = W[:, :, P], W[:, :, Q]
            app = (np.abs(wp) ** 2).sum(1, dtype=rdt)             # :332
            aqq = (np.abs(wq) ** 2).sum(1, dtype=rdt)
            apq = (np.conj(wp) * wq).sum(1, dtype=dt)             # :333
            den = np.sqrt(app) * np.sqrt(aqq)                     # :334
            ratio = np.abs(apq) / np.maximum(den, rdt.type(tiny(dt)))     # :335
            floor = rdt.type(e) ** 2 * np.maximum(app, aqq).max(-1, keepdims=True)   # :337
            active = (ratio > tol) & (np.minimum(app, aqq) > floor)       # :338
            off = max(off, np.where(active, ratio, rdt.type(0)).max())    # :339
            a = np.where(active, np.abs(apq), one)                # :340
            tau = (aqq - app) / (2 * a)                           # :341
            t = np.sign(tau) / (np.abs(tau) + np.hypot(tau, one))         # :342
            t = np.where(tau == 0, one, t).astype(rdt)            # :343
            c = (one / np.sqrt(one + t * t)).astype(rdt)          # :344
            s = (t * c).astype(dt) * (apq / a.astype(dt))         # :345
            c = np.where(active, c, one).astype(dt)               # :346
            s = np.where(active, s, 0).astype(dt)                 # :347
            c = c[:, None, :]
            s = s[:, None, :]
            W[:, :, P], W[:, :, Q] = c * wp - np.conj(s) * wq, s * wp + c * wq   # :349
            vp, vq = V[:, :, P], V[:, :, Q]
            V[:, :, P], V[:, :, Q] = c * vp - np.conj(s) * vq, s * vp + c * vq   # :350-351
        if off <= tol:                                            # :352
            break
    if off > tol:                                                 # :354-355
        raise RuntimeError(f"one-sided Jacobi did not converge in {max_sweeps} sweeps")
    s_vals = np.sqrt((np.abs(W) ** 2).sum(1, dtype=rdt))          # :356
    if padded:                                                    # :357-358
        W, V, s_vals = W[:, :, :-1], V[:, :-1, :-1], s_vals[:, :-1]
    order = np.argsort(-s_vals, axis=1, kind="stable")            # :359
    s_vals = np.take_along_axis(s_vals, order, 1)
    W = np.take_along_axis(W, order[:, None, :], 2)
    V = np.take_along_axis(V, order[:, None, :], 2)
    # n here is the padded width, as in the reference (:319, :323, :362).
    cut = rdt.type(e) * max(m, n) * s_vals[:, :1]                 # :362
    keep = s_vals > cut                                           # :363
    U = W / np.where(keep, s_vals, one)[:, None, :]               # :364
    U = complete_null_columns(U, keep)                            # :365
    s_vals = np.where(keep, s_vals, rdt.type(0))                  # :366
    return U, s_vals, V, sweeps


def complete_null_columns(u, keep):
    """Fill columns with keep==False by projected coordinate vectors
    (primitives.py:430-455): largest leftover row leverage picks the
    coordinate, two projections against all columns, normalise."""
    if keep.all():                                                # :432
        return u
    u = np.where(keep[:, None, :], u, 0).astype(u.dtype)          # :434-436
    b, m, n = u.shape
    rdt = _real(u.dtype)
    e = eps(u.dtype)
    for j in range(n):                                            # :438
        missing = ~keep[:, j]
        if not missing.any():
            continue
        leverage = 1 - (np.abs(u) ** 2).sum(-1, dtype=rdt)        # :444
        idx = leverage.argmax(-1)                                 # :445
        v = np.zeros((b, m, 1), u.dtype)
        v[np.arange(b), idx, 0] = 1                               # :446-447
        for _ in range(2):                                        # :448-449
            v = v - u @ (np.conj(np.swapaxes(u, -1, -2)) @ v)
        length = np.sqrt((np.abs(v) ** 2).sum(-2, keepdims=True, dtype=rdt))  # :450
        if (length[missing] < 10 * e).any():                      # :451-452
            raise RuntimeError("null-space completion failed: supplied live columns are not independent")
        v = v / np.maximum(length, rdt.type(tiny(u.dtype)))       # :453
        u[:, :, j] = np.where(missing[:, None], v[:, :, 0], u[:, :, j])   # :454
    return u


def complete_basis(q, size):
    """Extend an orthonormal basis to `size` columns (primitives.py:458-467)."""
    if size == q.shape[-1]:
        return q
    b, m, k = q.shape
    if not k <= size <= m:
        raise ValueError("invalid basis size")
    z = np.zeros((b, m, size - k), q.dtype)
    keep = np.broadcast_to(np.arange(size)[None, :] < k, (b, size))
    return complete_null_columns(np.concatenate([q, z], -1), keep)


def householder_vec(x):
    """Reflector of the rows of x (b, k), LAPACK xLARFG convention
    (primitives.py:41-59): v (v_0 = 1), tau, beta with
    (I - tau v v^H)^H x = beta e_1; a row with nothing below its first entry
    (and a real first entry) gets v = 0, tau = 0, beta = x_0."""
    b, k = x.shape
    rdt = _real(x.dtype)
    alpha = x[:, 0]
    xnorm = np.sqrt((np.abs(x[:, 1:]) ** 2).sum(-1)).astype(rdt) if k > 1 else np.zeros(b, rdt)
    ar = alpha.real.astype(rdt)
    ai = alpha.imag.astype(rdt) if np.iscomplexobj(x) else np.zeros_like(ar)
    beta = (-np.sign(ar + (ar == 0)) * np.hypot(np.abs(alpha).astype(rdt), xnorm)).astype(rdt)
    trivial = (xnorm == 0) & (ai == 0)
    beta = np.where(trivial, ar, beta).astype(rdt)
    bx = beta.astype(x.dtype)
    denom = np.where(trivial, np.ones_like(alpha), alpha - bx)
    tau = np.where(trivial, np.zeros_like(alpha), (bx - alpha) / np.where(beta != 0, bx, np.ones_like(bx)))
    v = x / denom[:, None]
    v[:, 0] = 1
    v = np.where(trivial[:, None], np.zeros_like(v), v)
    return v.astype(x.dtype), tau.astype(x.dtype), beta


def _apply_left(A, v, tau):
    """(I - tau v v^H) A for A (b, k, c) (primitives.py:62-65)."""
    w = (np.conj(v)[:, :, None] * A).sum(-2)
    return A - tau[:, None, None] * v[:, :, None] * w[:, None, :]


def qr(A):
    """Householder QR of tall A (b, m, n): Q (b, m, n), R (b, n, n), Q by
    backward accumulation (primitives.py:74-89)."""
    A = np.array(A, copy=True)
    b, m, n = A.shape
    vs, taus = [], []
    for j in range(n):
        v, tau, beta = householder_vec(A[:, j:, j])
        A[:, j:, j + 1:] = _apply_left(A[:, j:, j + 1:], v, np.conj(tau))
        A[:, j, j] = beta
        A[:, j + 1:, j] = 0
        vs.append(v)
        taus.append(tau)
    R = np.triu(A[:, :n, :])
    Q = np.zeros((b, m, n), A.dtype)
    Q[:, :n, :] = np.eye(n, dtype=A.dtype)
    for j in range(n - 1, -1, -1):
        Q[:, j:, :] = _apply_left(Q[:, j:, :], vs[j], taus[j])
    return Q, R


def tsqr(a, rows, stats):
    """Tall-skinny QR: QR of row tiles of `rows` rows (a short last tile joins
    the one before), a binary reduction tree over the stacked R factors and
    the tree back-transformation of Q (solvers.py:71-96)."""
    b, m, n = a.shape
    rows = max(rows, n)
    if m <= rows:
        return qr(a)
    leaves = []
    for start in range(0, m, rows):
        end = min(start + rows, m)
        if end - start < n:
            start = leaves.pop()[0]
        q, r = qr(a[:, start:end])
        leaves.append((start, q, r))
    stats["tsqr_leaves"] = len(leaves)
    nodes = [(q, r) for _, q, r in leaves]
    while len(nodes) > 1:
        nxt = []
        for i in range(0, len(nodes), 2):
            if i + 1 == len(nodes):
                nxt.append(nodes[i])
                continue
            (q1, r1), (q2, r2) = nodes[i], nodes[i + 1]
            q, r = qr(np.concatenate([r1, r2], -2))
            nxt.append((np.concatenate([q1 @ q[:, :n], q2 @ q[:, n:]], -2), r))
        nodes = nxt
    return nodes[0]


def partial(a, stats, opts, method):
    """Projected solvers 'randomized', 'subspace', 'block_krylov'
    (solvers.py:185-220) from a given start basis opts['initial_basis']
    (b, n, rank + oversample): the reference draws it from torch's generator
    otherwise, which NumPy cannot reproduce."""
    k = opts.get("rank", min(a.shape[-2:]))
    ell = min(k + opts.get("oversample", 8), min(a.shape[-2:]))
    omega = np.asarray(opts["initial_basis"])
    if omega.ndim == 2:
        omega = omega[None]
    if omega.shape != (a.shape[0], a.shape[-1], ell):
        raise ValueError("initial_basis shape must match batch, n, rank+oversample")
    omega = omega.astype(a.dtype)
    stats["warm_started"] = True
    q, _ = qr(a @ omega)
    bases = [q]
    iterations = opts.get("iterations", 2)
    ah = np.conj(np.swapaxes(a, -1, -2))
    for _ in range(iterations):
        z, _ = qr(ah @ q)
        y = a @ z
        if method == "block_krylov":
            joined = np.concatenate(bases, -1)
            available = a.shape[-2] - joined.shape[-1]
            if available <= 0:
                break
            jh = np.conj(np.swapaxes(joined, -1, -2))
            for _ in range(2):
                y = y - joined @ (jh @ y)
            q, _ = qr(y[:, :, :min(ell, available)])
            bases.append(q)
        else:
            q, _ = qr(y)
    if method == "block_krylov":
        q, _ = qr(np.concatenate(bases, -1))
    small = np.conj(np.swapaxes(q, -1, -2)) @ a
    u, s, v = raw(small, opts, stats, "jacobi")
    stats.update(sketch_columns=ell, range_columns=q.shape[-1], power_iterations=iterations)
    return (q @ u)[:, :, :k], s[:, :k], v[:, :, :k]


PARTIAL = ("randomized", "subspace", "block_krylov")


def finish_columns(w, s):
    """U = W / sigma above eps * max(m, n) * sigma_1, the rest completed
    (solvers.py:18-21)."""
    keep = s > s.dtype.type(eps(w.dtype)) * max(w.shape[-2:]) * s[:, :1]
    u = w / np.where(keep, s, s.dtype.type(1))[:, None, :]
    return complete_null_columns(u, keep), np.where(keep, s, s.dtype.type(0))


def block_jacobi(a, stats, opts):
    """Block one-sided Jacobi (solvers.py:30-68): column groups of
    block_size in a round-robin tournament, each pair orthogonalised by the
    Jacobi SVD of its columns, until the largest correlation of live columns
    is at most tol (40 eps by default); pairs applied one after the other
    as in the reference."""
    b, m, n = a.shape
    width = opts.get("block_size", 4)                              # :32
    if width < 1:
        raise ValueError("block_size must be positive")
    groups = [list(range(j, min(j + width, n))) for j in range(0, n, width)]   # :35
    if len(groups) == 1:                                           # :36-37
        return raw(a, opts, stats, "jacobi")
    if len(groups) % 2:                                            # :38-39
        groups.append([])
    w = a.copy()
    v = np.broadcast_to(np.eye(n, dtype=a.dtype), (b, n, n)).copy()
    e = eps(a.dtype)
    tol = opts.get("tol") or 40 * e                               # :41
    rdt = _real(a.dtype)
    for sweep in range(opts.get("max_sweeps", 30)):               # :42
        for pairs in round_robin(len(groups)):                     # :43-44
            for i, j in pairs:
                cols = groups[i] + groups[j]
                if len(cols) < 2:                                  # :46-47
                    continue
                _, _, vv, sweeps = jacobi_svd(w[:, :, cols], tol=opts.get("tol"),
                                              max_sweeps=opts.get("max_sweeps", 60))   # :48, :24-27
                stats["jacobi_sweeps"] = max(stats.get("jacobi_sweeps", 0), sweeps)
                w[:, :, cols] = w[:, :, cols] @ vv                 # :49
                v[:, :, cols] = v[:, :, cols] @ vv                 # :50
        g = np.conj(np.swapaxes(w, -1, -2)) @ w                    # :51
        d = np.clip(np.real(np.diagonal(g, axis1=-2, axis2=-1)), 0, None)   # :52
        denom = np.sqrt(d)[:, :, None] * np.sqrt(d)[:, None, :]     # :53
        g = g.copy()
        idx = np.arange(n)
        g[:, idx, idx] = 0                                         # :54
        live = d > (e * max(m, n)) ** 2 * d.max(-1, keepdims=True)  # :55
        corr = np.where(live[:, :, None] & live[:, None, :],
                        np.abs(g) / np.maximum(denom, tiny(rdt)), 0)   # :56
        if corr.max() <= tol:                                      # :57-58
            break
    else:
        raise RuntimeError("block Jacobi did not converge")       # :59-60
    s = np.sqrt((np.abs(w) ** 2).sum(1, dtype=rdt))               # :61
    order = np.argsort(-s, axis=1, kind="stable")                 # :62
    s = np.take_along_axis(s, order, 1)
    w = np.take_along_axis(w, order[:, None, :], 2)
    v = np.take_along_axis(v, order[:, None, :], 2)
    u, s = finish_columns(w, s)                                    # :66
    stats["block_sweeps"] = sweep + 1                             # :67
    return u, s, v


def raw(x, opts, stats, method="jacobi"):
    """Wide inputs are solved through their adjoint, except by the projected
    solvers (solvers.py:224-230); then 'jacobi' (:229-230), 'block_jacobi'
    (:231-232), 'qr' / 'tsqr' (:245-248) or the projected solvers (:253-254)."""
    if x.shape[-2] < x.shape[-1] and method not in PARTIAL:
        u, s, v = raw(np.conj(np.swapaxes(x, -1, -2)), opts, stats, method)
        return v, s, u
    if method in ("qr", "tsqr"):
        q, r = qr(x) if method == "qr" else tsqr(x, opts.get("tile_rows", 4 * x.shape[-1]), stats)
        u, s, v = raw(r, opts, stats, "jacobi")
        return q @ u, s, v
    if method in PARTIAL:
        return partial(x, stats, opts, method)
    if method == "block_jacobi":
        return block_jacobi(x, stats, opts)
    u, s, v, sweeps = jacobi_svd(x, tol=opts.get("tol"), max_sweeps=opts.get("max_sweeps", 60))
    stats["jacobi_sweeps"] = max(stats.get("jacobi_sweeps", 0), sweeps)   # solvers.py:24-27
    return u, s, v


def svd(a, algorithm="jacobi", *, full_matrices=False, values_only=False, return_info=False, **opts):
    """NumPy restatement of the public entry (solvers.py:264-310) for the
    Jacobi-based algorithms."""
    a = np.asarray(a)
    if algorithm not in ("jacobi", "block_jacobi", "qr", "tsqr") + PARTIAL:
        raise ValueError("the oracle restates the Jacobi-based algorithms only")
    if a.ndim < 2 or min(a.shape[-2:]) < 1:
        raise ValueError("nonempty matrix dimensions required")
    if a.dtype not in (np.float32, np.float64, np.complex64, np.complex128):
        raise TypeError("supported dtypes: float32/64, complex64/128")
    rank = opts.get("rank", min(a.shape[-2:]))
    if not 1 <= rank <= min(a.shape[-2:]):
        raise ValueError("rank outside [1,min(m,n)]")
    if full_matrices and rank != min(a.shape[-2:]):
        raise ValueError("full_matrices and truncated rank cannot be combined")
    for key in ("max_iter", "max_sweeps", "leaf_size"):
        if key in opts and opts[key] < 1:
            raise ValueError(f"{key} must be positive")
    for key in ("oversample", "iterations"):
        if key in opts and opts[key] < 0:
            raise ValueError(f"{key} must be nonnegative")
    shape = a.shape[:-2]
    x = a.reshape(-1, *a.shape[-2:])
    if not np.isfinite(x).all():
        raise ValueError("input contains NaN or infinity")
    scale = np.abs(x).max((-2, -1), keepdims=True)                # solvers.py:294-295
    scale = np.where(scale > 0, scale, 1).astype(_real(a.dtype))
    stats = {"algorithm": algorithm, "vendor_factorizations": 0, "converged": True}
    u, s, v = raw((x / scale).astype(a.dtype), opts, stats, algorithm)
    s = s * scale[:, 0, 0][:, None]
    if full_matrices:
        u = complete_basis(u, a.shape[-2])
        v = complete_basis(v, a.shape[-1])
    else:
        u, s, v = u[:, :, :rank], s[:, :rank], v[:, :, :rank]
    if not all(np.isfinite(z).all() for z in (u, s, v)):
        raise RuntimeError("standalone solver produced nonfinite output")
    vh = np.conj(np.swapaxes(v, -1, -2))
    result = (None if values_only else u.reshape(*shape, *u.shape[-2:]),
              s.reshape(*shape, s.shape[-1]),
              None if values_only else vh.reshape(*shape, *vh.shape[-2:]))
    return (*result, stats) if return_info else result


def reference(a):
    """FP64 LAPACK gesvd truth on the rounded input (metrics.py:6-10)."""
    import scipy.linalg
    dtype = np.complex128 if np.iscomplexobj(a) else np.float64
    arrays = a[None] if a.ndim == 2 else a
    return [scipy.linalg.svd(x.astype(dtype), full_matrices=False, lapack_driver="gesvd",
                             check_finite=True) for x in arrays]


def validate(a, result, refs):
    """Accuracy metrics against the FP64 truth (metrics.py:13-66): worst case
    over the batch of each key, plus the per-matrix rows."""
    u, s, vh = result
    arrays = a[None] if a.ndim == 2 else a
    if a.ndim == 2:
        s = s[None]
        u, vh = (u[None], vh[None]) if u is not None else (None, None)
    rows = []
    for i, (x, (ur, sr, vhr)) in enumerate(zip(arrays, refs)):
        dtype = np.complex128 if np.iscomplexobj(x) else np.float64
        x = x.astype(dtype)
        k = s.shape[-1]
        si = s[i].astype(np.float64)
        if not np.isfinite(si).all() or (u is not None and
                                         (not np.isfinite(u[i]).all() or not np.isfinite(vh[i]).all())):
            raise ValueError("Non-finite SVD output")
        norm = np.linalg.norm(x)
        denom = norm if norm > 0 else 1.0
        top = sr[0] if sr[0] > 0 else 1.0
        floor = np.finfo(np.float64).eps * max(x.shape) * top
        resolved = sr[:k] > floor
        d = {
            "spectrum_error_over_sigma1": float(np.max(np.abs(si - sr[:k])) / top),
            "singular_values_nonnegative_sorted": bool(np.all(si >= 0) and np.all(np.diff(si) <= 0)),
            "resolved_spectrum_max_relative_error": float(np.max(np.abs(si[resolved] - sr[:k][resolved]) / sr[:k][resolved])) if resolved.any() else None,
            "reference_tail_relative_fro": float(np.linalg.norm(sr[k:]) / denom),
        }
        if u is not None:
            ui, vi = u[i].astype(dtype), vh[i].astype(dtype)
            uk, vk = ui[:, :k], vi[:k, :]
            residual = np.linalg.norm(x - (uk * si) @ vk) / denom
            d.update({
                "reconstruction_relative_fro": float(residual),
                "orthogonality_u_fro_over_sqrt_cols": float(np.linalg.norm(ui.conj().T @ ui - np.eye(ui.shape[1])) / np.sqrt(ui.shape[1])),
                "orthogonality_v_fro_over_sqrt_rows": float(np.linalg.norm(vi @ vi.conj().T - np.eye(vi.shape[0])) / np.sqrt(vi.shape[0])),
            })
        rows.append(d)
    worst = {}
    for key in rows[0]:
        values = [r[key] for r in rows if r[key] is not None]
        worst[key] = (all(values) if isinstance(values[0], bool) else max(values)) if values else None
    return {"worst": worst, "per_matrix": rows}


def jacobi_eigh(H, tol=None, max_sweeps=30):
    """Two-sided cyclic Jacobi of Hermitian H (b, n, n), real or complex: w
    ascending (real), V, sweeps.  Restates primitives.py:370-427 in the
    input's dtype, batched in lock-step: zero-padding to even n (:384-386), tol =
    10 eps (:388), per round the scale max|G| (:395), active pairs
    |g_pq| > tol scale (:396), off = max |g_pq| / scale (:397), the rotation
    (:398-405), G <- G J then G <- J^T G (:407-414), V <- V J (:410-411),
    convergence after the sweep when off <= tol (:415-416)."""
    H = np.asarray(H)
    b, n, _ = H.shape
    padded = n % 2 == 1
    G = H.copy()
    if padded:
        Z = np.zeros((b, n + 1, n + 1), H.dtype)
        Z[:, :n, :n] = G
        G = Z
        n += 1
    V = np.broadcast_to(np.eye(n, dtype=G.dtype), (b, n, n)).copy()
    tol = tol or 10 * eps(H.dtype)
    bi = np.arange(b)[:, None]
    sched = [(np.array([p for p, _ in prs]), np.array([q for _, q in prs])) for prs in round_robin(n)]
    off = np.inf
    sweeps = 0
    for sweeps in range(1, max_sweeps + 1):
        off = 0.0
        for P, Q in sched:
            gpp, gqq, gpq = G[bi, P, P].real, G[bi, Q, Q].real, G[bi, P, Q]
            a = np.abs(gpq)
            scale = np.broadcast_to(np.abs(G).max(axis=(-2, -1))[:, None], a.shape)
            active = a > tol * scale
            off = max(off, float((a / np.maximum(scale, np.finfo(scale.dtype).tiny)).max()))
            a_safe = np.where(active, a, 1)
            tau = (gqq - gpp) / (2 * a_safe)
            t = np.sign(tau) / (np.abs(tau) + np.hypot(tau, 1))
            t = np.where(tau == 0, 1, t)
            c = 1 / np.sqrt(1 + t * t)
            s = t * c * (gpq / a_safe)
            c = np.where(active, c, 1).astype(G.dtype)
            s = np.where(active, s, 0).astype(G.dtype)
            cc, ss = c[:, None, :], s[:, None, :]
            gp, gq = G[:, :, P].copy(), G[:, :, Q].copy()
            G[:, :, P], G[:, :, Q] = cc * gp - np.conj(ss) * gq, ss * gp + cc * gq
            vp, vq = V[:, :, P].copy(), V[:, :, Q].copy()
            V[:, :, P], V[:, :, Q] = cc * vp - np.conj(ss) * vq, ss * vp + cc * vq
            cc, ss = c[:, :, None], s[:, :, None]
            rp, rq = G[:, P, :].copy(), G[:, Q, :].copy()
            G[:, P, :], G[:, Q, :] = cc * rp - ss * rq, np.conj(ss) * rp + cc * rq
        if off <= tol:
            break
    if off > tol:
        raise RuntimeError(f"Hermitian Jacobi did not converge in {max_sweeps} sweeps")
    w = np.diagonal(G, axis1=-2, axis2=-1).real.copy()
    if padded:
        w, V = w[:, :-1], V[:, :-1, :-1]
    order = np.argsort(w, axis=-1, kind="stable")
    return np.take_along_axis(w, order, 1), np.take_along_axis(V, order[:, None, :], 2), sweeps
