"""GPU Householder QR (jb_qr_f32/_f64/_c64/_c128) and the reference's QR-based solvers
('qr', 'tsqr', 'randomized', 'subspace', 'block_krylov') through the drop-in
svd(), against the reference's own outputs (golden fixtures), the NumPy
oracle and FP64 LAPACK.

Tolerances, stated once:
  * QR factors: 50 eps * max(1, max|A|) * m elementwise in the input dtype
    (different summation order than the reference, same reflectors); on
    columns a rank-deficient input leaves to rounding noise only Q R = A
    and Q^T Q = I are checked;
  * sigma against the reference: `sigma_tol` of the dtype (relative to
    sigma_1); singular vectors up to sign (a unit phase for complex input)
    where the value is simple (1e-3 single, 1e-8 double precision), as in
    the oracle's own tests;
  * the projected solvers are approximations: against FP64 truth they must
    be as accurate as the reference (twice its error, or sigma_tol).
"""
import importlib

import numpy as np
import pytest
import torch

from conftest import QR_DETERMINED, golden_methods, golden_qr, sigma_tol
from oracle import jacobi_oracle as O
from test_oracle import _cmp_sigma, _cmp_vectors, _cmp_vectors_phase

pytestmark = pytest.mark.gpu
DEV = "cuda"


def _qr_mod():
    return importlib.import_module("pavel-s_svd_b200.qr")


def _check_factors(a, q, r, q_ref=None, r_ref=None, determined=None):
    a = np.asarray(a)
    tol = 50 * np.finfo(a.dtype).eps * max(1.0, float(np.abs(a).max())) * a.shape[-2]
    wide = np.complex128 if np.iscomplexobj(a) else np.float64
    q64, r64 = np.asarray(q, wide), np.asarray(r, wide)
    assert np.array_equal(r64, np.triu(r64))
    assert float(np.abs(q64 @ r64 - a).max()) <= tol
    assert float(np.abs(np.conj(np.swapaxes(q64, -1, -2)) @ q64 - np.eye(a.shape[-1])).max()) <= tol
    if q_ref is not None:
        k = a.shape[-1] if determined is None else determined
        assert float(np.abs(q64[..., :k] - q_ref[..., :k]).max()) <= tol
        assert float(np.abs(r64[..., :k, :] - r_ref[..., :k, :]).max()) <= tol


def test_qr_matches_reference_golden():
    Q = _qr_mod()
    for name, g in golden_qr().items():
        a = g["a"]
        q, r = Q.qr(torch.from_numpy(a).to(DEV))
        _check_factors(a, q.cpu().numpy(), r.cpu().numpy(), g["q"], g["r"], QR_DETERMINED.get(name))


@pytest.mark.parametrize("shape,dtype", [((5, 64, 64), np.float64), ((2, 300, 100), np.float64),
                                         ((3, 256, 128), np.float32), ((4, 17, 1), np.float32),
                                         ((2, 33, 33), np.float32), ((3, 1000, 24), np.float64)])
def test_qr_matches_oracle(shape, dtype):
    """Both work-area modes (shared memory; per-CTA workspace beyond it), a
    single column, square, very tall."""
    Q = _qr_mod()
    a = np.random.default_rng(hash(shape) % 2**32).standard_normal(shape).astype(dtype)
    q, r = Q.qr(torch.from_numpy(a).to(DEV))
    qo, ro = O.qr(a)
    _check_factors(a, q.cpu().numpy(), r.cpu().numpy(), qo, ro)


def test_qr_contract():
    Q = _qr_mod()
    with pytest.raises(ValueError):
        Q.qr(torch.zeros(2, 3, 5, device=DEV))                 # wide
    with pytest.raises(TypeError):
        Q.qr(torch.zeros(2, 5, 3, dtype=torch.float16, device=DEV))
    q, r = Q.qr(torch.zeros(0, 5, 3, device=DEV))
    assert q.shape == (0, 5, 3) and r.shape == (0, 3, 3)
    # a zero matrix: every reflector is trivial, Q = [I; 0], R = 0
    q, r = Q.qr(torch.zeros(1, 6, 4, dtype=torch.float64, device=DEV))
    assert torch.equal(r, torch.zeros_like(r))
    assert torch.equal(q[0, :4], torch.eye(4, dtype=torch.float64, device=DEV)) and not q[0, 4:].any()


def test_methods_match_reference_golden(pkg):
    for name, g in golden_methods().items():
        kw = dict(g["kw"])
        if "initial_basis" in g:
            kw["initial_basis"] = torch.from_numpy(g["initial_basis"]).to(DEV)
        a = g["a"]
        u, s, vh, info = pkg.svd(torch.from_numpy(a).to(DEV), g["alg"], return_info=True, **kw)
        u, s, vh = u.resolve_conj().cpu().numpy(), s.cpu().numpy(), vh.resolve_conj().cpu().numpy()
        dt = a.dtype
        _cmp_sigma(s, g["s"], dt)
        cmp = _cmp_vectors_phase if np.iscomplexobj(a) else _cmp_vectors
        cmp(u, g["u"], g["s"], dt, -1)
        cmp(vh, g["vh"], g["s"], dt, -2)
        k = s.shape[-1]
        err = float(np.abs(s - g["truth"][..., :k]).max() / g["truth"].max())
        err_ref = float(np.abs(g["s"] - g["truth"][..., :k]).max() / g["truth"].max())
        assert err <= max(2 * err_ref, 10 * sigma_tol(dt)), name
        assert info["algorithm"] == g["alg"] and info.get("jacobi_sweeps", info.get("eigen_sweeps", 0)) >= 1
        if g["alg"] == "tsqr":
            assert info["tsqr_leaves"] >= 1   # a short last tile joins the one before (13 rows, tiles of 7: 1)
        if "initial_basis" in g:
            assert info["warm_started"] and info["sketch_columns"] == kw["rank"] + kw["oversample"]


@pytest.mark.parametrize("alg", ["qr", "tsqr"])
def test_qr_methods_full_and_values(pkg, alg):
    """Full bases, values only, wide input, a batch shape, against LAPACK."""
    rng = np.random.default_rng(7)
    for shape in ((2, 3, 70, 20), (4, 15, 40)):
        a = rng.standard_normal(shape).astype(np.float64)
        t = torch.from_numpy(a).to(DEV)
        u, s, vh = pkg.svd(t, alg, full_matrices=True, tile_rows=16)
        m, n = shape[-2:]
        assert u.shape == (*shape[:-2], m, m) and vh.shape == (*shape[:-2], n, n)
        flat = a.reshape(-1, m, n)
        truth = np.stack([np.linalg.svd(x, compute_uv=False) for x in flat]).reshape(s.shape)
        assert float(np.abs(s.cpu().numpy() - truth).max() / truth.max()) <= 1e-12
        u64, vh64 = u.cpu().numpy().reshape(-1, m, m), vh.cpu().numpy().reshape(-1, n, n)
        assert float(np.abs(np.swapaxes(u64, -1, -2) @ u64 - np.eye(m)).max()) <= 1e-12
        assert float(np.abs(vh64 @ np.swapaxes(vh64, -1, -2) - np.eye(n)).max()) <= 1e-12
        k = min(m, n)
        rec = (u64[..., :k] * s.cpu().numpy().reshape(-1, k)[:, None, :]) @ vh64[..., :k, :]
        assert float(np.abs(rec - flat).max()) <= 1e-12 * np.abs(flat).max() * max(m, n)
        u2, s2, vh2 = pkg.svd(t, alg, values_only=True, rank=3)
        assert u2 is None and vh2 is None and s2.shape == (*shape[:-2], 3)


@pytest.mark.parametrize("alg", ["randomized", "subspace", "block_krylov"])
def test_projected_solvers_own_sketch(pkg, alg):
    """Without a start basis the solver draws the reference's sketch (same
    generator, seed and call); giving that sketch as initial_basis reproduces
    the result exactly.  A decaying spectrum is captured to the accuracy of
    the method."""
    Q = _qr_mod()
    rng = np.random.default_rng(3)
    m, n, k = 60, 40, 5
    uu = np.linalg.qr(rng.standard_normal((2, m, n)))[0]
    vv = np.linalg.qr(rng.standard_normal((2, n, n)))[0]
    sv = 10.0 ** -np.arange(n, dtype=np.float64) * 0.5
    a = (uu * sv) @ np.swapaxes(vv, -1, -2)
    t = torch.from_numpy(a).to(DEV)
    u, s, vh, info = pkg.svd(t, alg, rank=k, return_info=True)
    assert "warm_started" not in info and info["sketch_columns"] == k + 8
    omega = Q.sketch(t, k + 8, 20261011)
    u2, s2, vh2 = pkg.svd(t, alg, rank=k, initial_basis=omega)
    assert torch.equal(s, s2) and torch.equal(u, u2) and torch.equal(vh, vh2)
    assert float(np.abs(s.cpu().numpy() - sv[:k]).max() / sv[0]) <= 1e-12
    with pytest.raises(ValueError, match="initial_basis shape"):
        pkg.svd(t, alg, rank=k, initial_basis=omega[:, :, :3])


def test_qr_methods_errors(pkg):
    t = torch.ones(2, 8, 5, device=DEV)
    t[1, 2, 3] = float("nan")
    for alg in ("qr", "tsqr", "randomized"):
        with pytest.raises(ValueError, match="NaN or infinity"):
            pkg.svd(t, alg)
    with pytest.raises(ValueError, match="oversample"):
        pkg.svd(torch.ones(1, 8, 5, device=DEV), "randomized", oversample=-1)
