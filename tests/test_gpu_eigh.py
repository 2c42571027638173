"""jacobi_eigh on the GPU (jb_eigh_f32/_f64, _c64/_c128 for Hermitian input)
against the reference's own outputs (golden fixtures) and FP64 LAPACK.

Bounds: eigenvalues within 10 n eps(dtype) max|w| of FP64 truth (the
reference's absolute criterion delivers eps * lambda_max accuracy); columns of
V orthonormal to 100 n eps(dtype); residual ||H V - V diag(w)|| / max|w| within
100 n eps(dtype); sweep counts within 2 of the reference's (its scale max|G|
is taken per round, here per sweep; for float32 input the arithmetic here is
FP64, the reference's is FP32)."""
import importlib

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def E():
    return importlib.import_module("pavel-s_svd_b200.eigh")


def _check(h, w, v, truth):
    n = h.shape[-1]
    e = np.finfo(h.dtype).eps
    wide = np.complex128 if np.iscomplexobj(h) else np.float64
    w = w.cpu().numpy().astype(np.float64)
    v = v.resolve_conj().cpu().numpy().astype(wide)
    scale = np.abs(truth).max(axis=-1, keepdims=True)
    assert float((np.abs(w - truth) / scale).max()) <= 10 * n * e
    eye = np.eye(n)
    assert float(np.abs(np.conj(np.swapaxes(v, -1, -2)) @ v - eye).max()) <= 100 * n * e
    res = np.abs(h.astype(wide) @ v - v * w[:, None, :]).max(axis=(-2, -1)) / scale[:, 0]
    assert float(res.max()) <= 100 * n * e


def test_eigh_matches_reference_golden(E, golden_eigh):
    for name, g in golden_eigh.items():
        h = g["h"]
        w, v, sw = E.jacobi_eigh(torch.from_numpy(h).cuda())
        assert w.dtype == torch.from_numpy(h).real.dtype and v.dtype == torch.from_numpy(h).dtype
        _check(h, w, v, g["truth"])
        assert abs(sw - int(g["sweeps"])) <= 2, name


@pytest.mark.parametrize("n,batch,dtype", [(64, 5, torch.float32), (127, 2, torch.float64), (200, 2, torch.float32),
                                           (1, 3, torch.float64), (2, 4, torch.float32), (48, 3, torch.complex64),
                                           (101, 2, torch.complex128), (130, 2, torch.complex128)])
def test_eigh_sizes(E, n, batch, dtype):
    """Even, odd (padded) and large sizes; V (and G for the largest) in
    global memory above the shared-memory limit; Hermitian input."""
    g = torch.Generator().manual_seed(n)
    cdt = torch.complex128 if dtype.is_complex else torch.float64
    x = torch.randn(batch, n, n, generator=g, dtype=cdt)
    h = (x + x.mH).to(dtype)
    w, v, sw = E.jacobi_eigh(h.cuda())
    truth = np.linalg.eigvalsh(h.to(cdt).numpy())
    _check(h.numpy(), w, v, truth)
    assert sw >= 1


def test_eigh_contract(E):
    h = torch.randn(2, 9, 9, device="cuda")
    h = h + h.transpose(1, 2)
    with pytest.raises(RuntimeError, match="did not converge in 1 sweeps"):
        E.jacobi_eigh(h, max_sweeps=1)
    with pytest.raises(ValueError):
        E.jacobi_eigh(torch.randn(2, 3, 4, device="cuda"))
    with pytest.raises(E.Unsupported):
        E.jacobi_eigh(torch.randn(2, 4, 4))
    w, v, sw = E.jacobi_eigh(torch.diag(torch.tensor([3.0, -1.0, 2.0])).cuda()[None])
    assert w.cpu().tolist() == [[-1.0, 2.0, 3.0]] and sw == 1


def test_gram_jacobi_drop_in():
    """svd(a, 'gram_jacobi') (solvers.py:99-120): the Gram route's absolute
    accuracy (sigma errors ~ eps ||A||^2 / sigma), U orthonormal with null
    completion for a rank-deficient input, wide input, full_matrices and
    values_only."""
    pkg = importlib.import_module("pavel-s_svd_b200")
    rng = np.random.default_rng(17)
    for m, n, dt in ((40, 24, np.float32), (24, 40, np.float64), (64, 64, np.float64)):
        a = rng.standard_normal((3, m, n)).astype(dt)
        x = torch.from_numpy(a).cuda()
        u, s, vh, info = pkg.svd(x, 'gram_jacobi', return_info=True)
        k = min(m, n)
        sr = np.linalg.svd(a.astype(np.float64), compute_uv=False)
        e = np.finfo(dt).eps
        bound = 100 * e * sr[:, :1] ** 2 / sr
        assert bool((np.abs(s.cpu().numpy() - sr) / sr <= bound).all())
        rec = (u.double() * s.double()[:, None, :]) @ vh.double()
        assert float((rec - x.double()).norm() / x.double().norm()) <= 1e4 * e
        assert info['eigen_sweeps'] >= 1 and info['gram_discarded_values'] == 0
    # rank 3 of 10 columns: 7 values cut, their U columns completed
    b = rng.standard_normal((30, 3)) @ rng.standard_normal((3, 10))
    u, s, vh, info = pkg.svd(torch.from_numpy(b).cuda(), 'gram_jacobi', return_info=True)
    assert info['gram_discarded_values'] == 7 and float(s[3:].abs().max()) == 0.0
    uu = u.cpu().numpy()
    assert float(np.abs(uu.T @ uu - np.eye(10)).max()) <= 1e-10
    u, s, vh = pkg.svd(torch.from_numpy(b).cuda(), 'gram_jacobi', full_matrices=True)
    assert u.shape == (30, 30) and vh.shape == (10, 10)
    assert float(np.abs(u.cpu().numpy().T @ u.cpu().numpy() - np.eye(30)).max()) <= 1e-10
    u, s, vh = pkg.svd(torch.from_numpy(b).cuda(), 'gram_jacobi', values_only=True)
    assert u is None and vh is None and s.shape == (10,)
