"""A seeded cross-check of the drop-in over its routes: every algorithm built
here, the four dtypes, tall / wide / square shapes on both sides of the
kernels' size limits (register tiles, large tiles, QR first, TSQR, block
rounds), and the output forms (reduced, full bases, values only, a
truncated rank), against FP64 LAPACK on the same input.

Tolerances, stated once (relative to sigma_1): sigma 2e-5 for single
precision (the 'fp32' and complex64 arithmetic of the reference), 1e-11 for
double precision; orthonormal columns and reconstruction 10x those, scaled
by max(1, size / 64).  gram_jacobi squares the condition number cond: sigma
within 10 eps cond (or reported as 0 within a factor 2 of the reference's
eigenvalue cut), vectors within 10 eps cond^2 (checked where that is below
1e-2).  The projected solvers run with rank = min(m, n) and no power
iterations, where their range basis is exact."""
import importlib
import itertools
import zlib

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu
DEV = "cuda"

SHAPES = [(3, 17, 9), (2, 9, 17), (2, 40, 40), (2, 130, 60), (1, 300, 70), (2, 70, 300), (1, 600, 24)]
DTYPES = [np.float32, np.float64, np.complex64, np.complex128]
ALGS = ["jacobi", "block_jacobi", "gram_jacobi", "qr", "tsqr", "randomized", "subspace", "block_krylov"]


def _cases():
    rng = np.random.default_rng(2026)
    out = []
    for alg, dt, shape in itertools.product(ALGS, DTYPES, SHAPES):
        form = ["reduced", "full", "values", "rank"][int(rng.integers(4))]
        if alg in ("randomized", "subspace", "block_krylov") and form in ("full", "rank"):
            form = "reduced"
        out.append(pytest.param(alg, dt, shape, form, id=f"{alg}-{np.dtype(dt).name}-{'x'.join(map(str, shape))}-{form}"))
    return out


@pytest.fixture(scope="module")
def pkg():
    return importlib.import_module("pavel-s_svd_b200")


@pytest.mark.parametrize("alg,dt,shape,form", _cases())
def test_routes_against_lapack(pkg, alg, dt, shape, form):
    # a seed fixed per case (Python's hash of strings changes per process)
    rng = np.random.default_rng(zlib.crc32(f"{alg}-{np.dtype(dt).name}-{shape}".encode()))
    a = rng.standard_normal(shape)
    if np.issubdtype(dt, np.complexfloating):
        a = a + 1j * rng.standard_normal(shape)
    a = a.astype(dt)
    m, n = shape[-2:]
    k = min(m, n)
    kw = {}
    if alg == "block_jacobi":
        kw["block_size"] = 8
    if alg == "tsqr":
        kw["tile_rows"] = max(2 * k, 32)
    if alg in ("randomized", "subspace", "block_krylov"):
        kw.update(rank=k, oversample=0, iterations=0)
    if form == "rank":
        kw["rank"] = max(1, k // 2)
    t = torch.from_numpy(a).to(DEV)
    u, s, vh = pkg.svd(t, alg, full_matrices=form == "full", values_only=form == "values", **kw)
    assert torch.equal(t, torch.from_numpy(a).to(DEV))             # input untouched
    single = np.dtype(dt) in (np.float32, np.complex64)
    tol = 2e-5 if single else 1e-11
    wide = np.complex128 if np.iscomplexobj(a) else np.float64
    a64 = a.astype(wide)
    truth = np.linalg.svd(a64, compute_uv=False)
    r = kw.get("rank", k)
    eps = float(np.finfo(np.float32 if single else np.float64).eps)
    cond = float((truth[..., 0] / truth[..., -1]).max())
    sig_tol, vec_scale = tol, 1.0
    if alg == "gram_jacobi":
        sig_tol = max(tol, 10 * eps * cond)
        vec_scale = max(1.0, eps * cond ** 2 / tol)
    s = s.cpu().numpy().astype(np.float64)
    assert s.shape == (*shape[:-2], r)
    err = np.abs(s - truth[..., :r])
    allowed = sig_tol * truth.max()
    if alg == "gram_jacobi":
        # the reference reports 0 for Gram eigenvalues below eps n w_max
        # (solvers.py:_gram): values near that cut may come back as 0
        cut = truth[..., :1] * np.sqrt(2.0 * eps * n)
        allowed = np.where(truth[..., :r] < cut, np.maximum(truth[..., :r], allowed), allowed)
    assert bool((err <= allowed).all()), float((err - allowed).max())
    if form == "values":
        assert u is None and vh is None
        return
    u = u.resolve_conj().cpu().numpy().astype(wide)
    vh = vh.resolve_conj().cpu().numpy().astype(wide)
    ucols = m if form == "full" else r
    vrows = n if form == "full" else r
    assert u.shape == (*shape[:-2], m, ucols) and vh.shape == (*shape[:-2], vrows, n)
    vt = 10 * tol * vec_scale
    if vt > 1e-2:
        return
    assert float(np.abs(np.conj(np.swapaxes(u, -1, -2)) @ u - np.eye(ucols)).max()) <= vt * max(1, m / 64)
    assert float(np.abs(vh @ np.conj(np.swapaxes(vh, -1, -2)) - np.eye(vrows)).max()) <= vt * max(1, n / 64)
    rec = (u[..., :r] * s[..., None, :]) @ vh[..., :r, :]
    if r == k:
        assert float(np.abs(rec - a64).max() / np.abs(a64).max()) <= vt * max(1, max(m, n) / 64)


BOUNDARY = [(1, 128, 64), (1, 129, 64), (1, 128, 65), (1, 256, 128), (1, 257, 128), (1, 258, 129), (1, 513, 64),
            (1, 64, 129), (2, 32, 32), (2, 33, 33)]


@pytest.mark.parametrize("shape", BOUNDARY, ids=lambda s: "x".join(map(str, s)))
@pytest.mark.parametrize("dt", [np.float32, np.float64])
@pytest.mark.parametrize("variant", ["mixed-block", "fp32-round_robin"])
def test_jacobi_size_limits(pkg, shape, dt, variant):
    """'jacobi' on both sides of each kernel's size limit (register tiles
    128 x 64, large tiles 256 x 128, the QR-first rows, the narrow class
    n <= 32), both precisions of float32 input and both pair orders."""
    precision, ordering = variant.split("-")
    rng = np.random.default_rng(sum(shape))
    a = rng.standard_normal(shape).astype(dt)
    u, s, vh, info = pkg.svd(torch.from_numpy(a).to(DEV), "jacobi", precision=precision, ordering=ordering,
                             return_info=True)
    single = dt == np.float32 and precision == "fp32"
    tol = 2e-5 if single else (1e-5 if dt == np.float32 else 1e-11)
    truth = np.linalg.svd(a.astype(np.float64), compute_uv=False)
    s = s.cpu().numpy().astype(np.float64)
    assert float(np.abs(s - truth).max() / truth.max()) <= tol
    u, vh = u.cpu().numpy().astype(np.float64), vh.cpu().numpy().astype(np.float64)
    k = min(shape[-2:])
    vt = (1e-4 if dt == np.float32 else 1e-10) * max(1, max(shape) / 64)
    assert float(np.abs(np.swapaxes(u, 1, 2) @ u - np.eye(k)).max()) <= vt
    assert float(np.abs(vh @ np.swapaxes(vh, 1, 2) - np.eye(k)).max()) <= vt
    assert float(np.abs((u * s[:, None, :]) @ vh - a).max() / np.abs(a).max()) <= vt
    assert info["jacobi_sweeps"] >= 2
