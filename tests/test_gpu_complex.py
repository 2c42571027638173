"""'jacobi' on complex64 / complex128 (jb_svd_batched_c64/_c128 through the
drop-in svd()) against the reference's own outputs (golden fixtures, from
its complex test inputs) and FP64 LAPACK.

Tolerances, stated once:
  * sigma against the reference: `sigma_tol` (1e-5 complex64, 1e-12
    complex128, relative to sigma_1); the sweep counts within 1 (same order
    and arithmetic, different summation order);
  * singular vectors up to a unit phase where the value is simple (1e-3
    complex64, 1e-8 complex128);
  * the reference's test contract (tests/test_standalone.py:33-45):
    reconstruction, orthogonality and spectrum within 3e-4 (complex64) /
    2e-10 (complex128).
"""
import numpy as np
import pytest
import torch

from conftest import golden_complex, sigma_tol
from test_oracle import _cmp_sigma, _cmp_vectors_phase

pytestmark = pytest.mark.gpu
DEV = "cuda"


def _contract(a, u, s, vh, tol):
    a = np.asarray(a, np.complex128).reshape(-1, *np.shape(a)[-2:])
    b, m, n = a.shape
    u = np.asarray(u, np.complex128).reshape(b, m, -1)
    vh = np.asarray(vh, np.complex128).reshape(b, -1, n)
    s = np.asarray(s, np.float64).reshape(b, -1)
    k = s.shape[-1]
    if k == min(m, n):                      # a truncated rank does not reconstruct
        rec = (u[..., :k] * s[:, None, :]) @ vh[..., :k, :]
        scale = max(float(np.abs(a).max()), np.finfo(float).tiny)
        assert float(np.linalg.norm((rec - a) / scale) / max(np.linalg.norm(a / scale), np.finfo(float).tiny)) < tol
    for q in (u, np.conj(np.swapaxes(vh, -1, -2))):
        assert float(np.abs(np.conj(np.swapaxes(q, -1, -2)) @ q - np.eye(q.shape[-1])).max()) < 5 * tol
    truth = np.stack([np.linalg.svd(x, compute_uv=False) for x in a])[:, :k]
    assert float(np.abs(s - truth).max() / max(truth.max(), np.finfo(float).tiny)) < tol


def test_complex_matches_reference_golden(pkg):
    for name, g in golden_complex().items():
        a = g["a"]
        u, s, vh, info = pkg.svd(torch.from_numpy(a).to(DEV), "jacobi", return_info=True, **g["kw"])
        s = s.cpu().numpy()
        real = np.float32 if a.dtype == np.complex64 else np.float64
        assert s.dtype == real
        _cmp_sigma(s, g["s"], real)
        assert abs(info["jacobi_sweeps"] - g["sweeps"]) <= 1, name
        u, vh = u.cpu().numpy(), vh.cpu().numpy()
        assert u.shape == g["u"].shape and vh.shape == g["vh"].shape, name
        if np.asarray(g["s"]).max() > 0:
            _cmp_vectors_phase(u, g["u"], g["s"], a.dtype, -1)
            _cmp_vectors_phase(vh, g["vh"], g["s"], a.dtype, -2)
        _contract(a, u, s, vh, 3e-4 if a.dtype == np.complex64 else 2e-10)


@pytest.mark.parametrize("shape,dtype", [((3, 64, 48), np.complex128), ((2, 100, 60), np.complex64),
                                         ((1, 256, 128), np.complex128), ((2, 30, 75), np.complex64)])
def test_complex_sizes_against_lapack(pkg, shape, dtype):
    """Shared-memory and workspace work areas, tall and wide."""
    rng = np.random.default_rng(shape[-1])
    a = (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)).astype(dtype)
    u, s, vh = pkg.svd(torch.from_numpy(a).to(DEV), "jacobi")
    _contract(a, u.cpu().numpy(), s.cpu().numpy(), vh.cpu().numpy(), 3e-4 if dtype == np.complex64 else 2e-10)


def test_complex_errors(pkg):
    rng = np.random.default_rng(0)
    a = torch.from_numpy(rng.standard_normal((12, 9)) + 1j * rng.standard_normal((12, 9))).to(DEV)
    with pytest.raises(RuntimeError, match="did not converge in 1 sweeps"):
        pkg.svd(a, "jacobi", max_sweeps=1)
    b = a.clone()
    b[3, 4] = complex(float("nan"), 0.0)
    with pytest.raises(ValueError, match="NaN or infinity"):
        pkg.svd(b, "jacobi")
    with pytest.raises(RuntimeError, match="block Jacobi did not converge"):
        pkg.svd(a, "block_jacobi", block_size=1, max_sweeps=2)     # 2-column pairs converge, the blocks not
