"""svd(a, 'jacobi') on real matrices taller than the register and large-tile
kernels take: the QR-first path (solvers._tall_svd), against the NumPy
oracle of the reference's jacobi_svd on the full matrix and FP64 LAPACK.

Tolerances, stated once: sigma within `sigma_tol` of the dtype against the
oracle (relative to sigma_1); singular vectors up to sign where the value is
simple (1e-3 single, 1e-8 double precision); sweeps within 2 of the
oracle's (the same rotations in exact arithmetic, different rounding);
orthogonality of full bases 1e-5 (float32) / 1e-12 (float64)."""
import importlib

import numpy as np
import pytest
import torch

from conftest import sigma_tol
from oracle import jacobi_oracle as O
from test_oracle import _cmp_sigma, _cmp_vectors, _cmp_vectors_phase

pytestmark = pytest.mark.gpu
DEV = "cuda"


@pytest.fixture(scope="module")
def pkg():
    return importlib.import_module("pavel-s_svd_b200")


@pytest.mark.parametrize("shape,dtype,precision", [((2, 600, 40), np.float32, "mixed"),
                                                   ((2, 600, 40), np.float32, "fp32"),
                                                   ((3, 300, 20), np.float64, "mixed"),
                                                   ((1, 2048, 32), np.float64, "mixed"),
                                                   ((2, 24, 700), np.float32, "mixed")])
def test_tall_matches_oracle(pkg, shape, dtype, precision):
    rng = np.random.default_rng(shape[-1] + shape[-2])
    a = rng.standard_normal(shape).astype(dtype)
    u, s, vh, info = pkg.svd(torch.from_numpy(a).to(DEV), "jacobi", precision=precision, return_info=True)
    assert info["qr_first"] and info["jacobi_sweeps"] >= 2
    uo, so, vho, io = O.svd(a, "jacobi", return_info=True)
    s, u, vh = s.cpu().numpy(), u.cpu().numpy(), vh.cpu().numpy()
    _cmp_sigma(s, so, a.dtype)
    _cmp_vectors(u, uo, so, a.dtype, -1)
    _cmp_vectors(vh, vho, so, a.dtype, -2)
    assert abs(info["jacobi_sweeps"] - io["jacobi_sweeps"]) <= 2
    if precision == "mixed":      # the mixed bound: 1e-5 of sigma against FP64 LAPACK
        truth = np.linalg.svd(a.astype(np.float64), compute_uv=False)
        assert float(np.abs(s - truth).max() / truth.max()) <= 1e-5


@pytest.mark.parametrize("shape,dtype", [((2, 300, 20), np.complex64), ((2, 20, 400), np.complex128)])
def test_tall_complex_matches_oracle(pkg, shape, dtype):
    """Complex input through the complex QR: tall, and wide through the
    conjugate transpose; vectors up to a unit phase."""
    rng = np.random.default_rng(shape[-2])
    a = (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)).astype(dtype)
    u, s, vh, info = pkg.svd(torch.from_numpy(a).to(DEV), "jacobi", return_info=True)
    assert info["qr_first"]
    uo, so, vho, io = O.svd(a, "jacobi", return_info=True)
    s, u, vh = s.cpu().numpy(), u.resolve_conj().cpu().numpy(), vh.resolve_conj().cpu().numpy()
    _cmp_sigma(s, so, a.dtype)
    _cmp_vectors_phase(u, uo, so, a.dtype, -1)
    _cmp_vectors_phase(vh, vho, so, a.dtype, -2)
    assert abs(info["jacobi_sweeps"] - io["jacobi_sweeps"]) <= 2
    k = min(shape[-2:])
    rec = (u.astype(np.complex128) * s[:, None, :]) @ vh.astype(np.complex128)
    assert float(np.abs(rec - a).max() / np.abs(a).max()) <= (1e-5 if dtype == np.complex64 else 1e-13)
    uf, sf, vhf = pkg.svd(torch.from_numpy(a).to(DEV), "jacobi", full_matrices=True)
    q = (vhf if shape[-1] > shape[-2] else uf).cpu().numpy().astype(np.complex128)
    assert q.shape[-1] == max(shape[-2:]) and k == s.shape[-1]
    assert float(np.abs(np.conj(np.swapaxes(q, 1, 2)) @ q - np.eye(q.shape[-1])).max()) <= (
        1e-5 if dtype == np.complex64 else 1e-12)


def test_tall_rank_deficient_cut_and_full(pkg):
    """A rank-3 matrix 500 x 20: the reference's cut eps * max(m, n) * sigma_1
    zeroes the same values as the oracle, U is completed to orthonormal
    columns; full bases; values only; a truncated rank."""
    rng = np.random.default_rng(9)
    a = (rng.standard_normal((2, 500, 3)) @ rng.standard_normal((2, 3, 20))).astype(np.float64)
    t = torch.from_numpy(a).to(DEV)
    u, s, vh = pkg.svd(t, "jacobi")
    uo, so, vho = O.svd(a, "jacobi")
    assert np.array_equal(s.cpu().numpy() == 0, so == 0) and int((so == 0).sum()) == 2 * 17
    _cmp_sigma(s.cpu().numpy(), so, a.dtype)
    un = u.cpu().numpy()
    assert float(np.abs(np.swapaxes(un, 1, 2) @ un - np.eye(20)).max()) <= 1e-12
    uf, sf, vhf = pkg.svd(t, "jacobi", full_matrices=True)
    assert uf.shape == (2, 500, 500) and vhf.shape == (2, 20, 20)
    ufn = uf.cpu().numpy()
    assert float(np.abs(np.swapaxes(ufn, 1, 2) @ ufn - np.eye(500)).max()) <= 1e-12
    rec = (ufn[..., :20] * sf.cpu().numpy()[:, None, :]) @ vhf.cpu().numpy()
    assert float(np.abs(rec - a).max() / np.abs(a).max()) <= 1e-12
    u2, s2, vh2 = pkg.svd(t, "jacobi", values_only=True)
    assert u2 is None and vh2 is None and torch.equal(s2, s)
    u3, s3, vh3 = pkg.svd(t.float(), "jacobi", rank=5)
    assert u3.shape == (2, 500, 5) and s3.shape == (2, 5) and vh3.shape == (2, 5, 20)


def test_tall_large_against_lapack(pkg):
    """4096 x 128 float32 (mixed) and a float64 batch of 1024 x 64."""
    rng = np.random.default_rng(12)
    for shape, dtype, tol in (((1, 4096, 128), np.float32, 1e-5), ((4, 1024, 64), np.float64, 1e-13)):
        a = rng.standard_normal(shape).astype(dtype)
        u, s, vh = pkg.svd(torch.from_numpy(a).to(DEV), "jacobi")
        truth = np.linalg.svd(a.astype(np.float64), compute_uv=False)
        assert float(np.abs(s.cpu().numpy() - truth).max() / truth.max()) <= tol
        un, vn = u.cpu().numpy().astype(np.float64), vh.cpu().numpy().astype(np.float64)
        orth = 1e-5 if dtype == np.float32 else 1e-12
        assert float(np.abs(np.swapaxes(un, 1, 2) @ un - np.eye(shape[-1])).max()) <= orth
        rec = (un * s.cpu().numpy()[:, None, :]) @ vn
        assert float(np.abs(rec - a).max() / np.abs(a).max()) <= 10 * orth


def test_tall_errors(pkg):
    a = torch.randn(2, 400, 10, dtype=torch.float64, device=DEV)
    with pytest.raises(RuntimeError, match="did not converge in 1 sweeps"):
        pkg.svd(a, "jacobi", max_sweeps=1)
    a[1, 7, 3] = float("inf")
    with pytest.raises(ValueError, match="NaN or infinity"):
        pkg.svd(a, "jacobi")
