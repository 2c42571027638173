"""Null-space completion on the GPU (jb_complete_null) against the oracle's
restatement of the reference's complete_null_columns (primitives.py:430-455).

Bars: the pivot rows are integers and must be the oracle's; the completed
columns agree with the oracle's within 1e-12 (float64 / complex128) and
5e-5 (float32 / complex64); kept columns come back unchanged.  Cases cover
the one-CTA-per-matrix path (many matrices), the multi-CTA team path (one
tall matrix), its blocked pass (most columns missing), a full basis that
needs the second projection, the all-zero input, and the reference's
failure when the columns cannot be completed."""
import importlib

import numpy as np
import pytest
import torch

from oracle import jacobi_oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def S():
    return importlib.import_module("pavel-s_svd_b200.solvers")


def _case(rng, b, m, n, kept, dtype):
    cplx = np.dtype(dtype).kind == "c"
    g = rng.standard_normal((b, m, n)) + (1j * rng.standard_normal((b, m, n)) if cplx else 0)
    q = np.linalg.qr(g)[0][:, :, :n]
    keep = np.zeros((b, n), bool)
    for z in range(b):
        keep[z, rng.choice(n, kept, replace=False)] = True
    return q.astype(dtype), keep


def _tol(dtype):
    return 1e-12 if np.dtype(dtype) in (np.float64, np.complex128) else 5e-5


@pytest.mark.parametrize("dtype", [np.float64, np.complex128, np.float32, np.complex64])
@pytest.mark.parametrize("b,m,n,kept", [(64, 40, 12, 8), (300, 9, 9, 3), (5, 130, 64, 40)])
def test_matches_oracle(S, dtype, b, m, n, kept):
    rng = np.random.default_rng(b * 1000 + m + n)
    u, keep = _case(rng, b, m, n, kept, dtype)
    want = O.complete_null_columns(u.astype(np.complex128 if np.dtype(dtype).kind == "c" else np.float64), keep)
    got = S._complete_null_columns(torch.from_numpy(u).cuda(), torch.from_numpy(keep).cuda()).cpu().numpy()
    assert np.array_equal(got[np.broadcast_to(keep[:, None, :], got.shape)],
                          u[np.broadcast_to(keep[:, None, :], u.shape)])
    err = np.abs(got.astype(want.dtype) - want).max()
    assert err <= _tol(dtype), err
    eye = np.eye(n)
    assert np.abs(np.conj(np.swapaxes(got, 1, 2)) @ got - eye).max() <= 10 * _tol(dtype) + 1e-6


def test_zero_input_gives_coordinate_vectors(S):
    u = torch.zeros(3, 7, 5, dtype=torch.float32, device="cuda")
    keep = torch.zeros(3, 5, dtype=torch.bool, device="cuda")
    got = S._complete_null_columns(u, keep).cpu().numpy()
    want = O.complete_null_columns(np.zeros((3, 7, 5), np.float32), np.zeros((3, 5), bool))
    assert np.array_equal(got, want)


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_team_path_tall(S, dtype):
    """One 2048 x 600 matrix, 64 kept columns: the multi-CTA team path."""
    rng = np.random.default_rng(7)
    u, keep = _case(rng, 1, 2048, 600, 64, dtype)
    want = O.complete_null_columns(u.astype(np.float64), keep)
    got = S._complete_null_columns(torch.from_numpy(u).cuda(), torch.from_numpy(keep).cuda()).cpu().numpy()
    # the same pivots: every completed column has its largest entry in the oracle's row
    miss = ~keep[0]
    assert np.array_equal(np.abs(got[0][:, miss]).argmax(0), np.abs(want[0][:, miss]).argmax(0))
    err = np.abs(got.astype(np.float64) - want).max()
    assert err <= (1e-11 if dtype == np.float64 else 5e-5), err


@pytest.mark.parametrize("dtype,m,n,kept", [(np.float64, 4096, 1024, 32), (np.float32, 4096, 512, 16)])
def test_blocked_pass(S, dtype, m, n, kept):
    """A tall matrix with most columns missing: the team path completes them
    in blocks (candidate rows, pivoted Cholesky of their projector block);
    the pivots and columns must be the per-column algorithm's."""
    rng = np.random.default_rng(m + n)
    u, keep = _case(rng, 1, m, n, kept, dtype)
    want = O.complete_null_columns(u.astype(np.float64), keep)
    got = S._complete_null_columns(torch.from_numpy(u).cuda(), torch.from_numpy(keep).cuda()).cpu().numpy()
    miss = ~keep[0]
    assert np.array_equal(np.abs(got[0][:, miss]).argmax(0), np.abs(want[0][:, miss]).argmax(0))
    err = np.abs(got.astype(np.float64) - want).max()
    assert err <= (1e-11 if dtype == np.float64 else 5e-5), err
    g64 = got[0].astype(np.float64)
    assert np.abs(g64.T @ g64 - np.eye(n)).max() <= (1e-12 if dtype == np.float64 else 2e-5)


def test_team_path_full_basis(S):
    """A full 512 x 512 basis from 100 columns: late columns have leverage
    below 1/2, so the team path runs the second projection."""
    rng = np.random.default_rng(11)
    q = np.linalg.qr(rng.standard_normal((1, 512, 100)))[0]
    want = O.complete_basis(q, 512)
    got = S._complete_basis(torch.from_numpy(q).cuda(), 512).cpu().numpy()
    assert np.abs(got - want).max() <= 1e-10
    assert np.abs(got[0].T @ got[0] - np.eye(512)).max() <= 1e-12


def test_failure_is_the_references(S):
    """More columns than rows: the fifth column has nothing left to take."""
    u = torch.zeros(2, 4, 6, dtype=torch.float64, device="cuda")
    keep = torch.zeros(2, 6, dtype=torch.bool, device="cuda")
    with pytest.raises(RuntimeError, match="null-space completion failed"):
        S._complete_null_columns(u, keep)
    with pytest.raises(RuntimeError, match="null-space completion failed"):
        O.complete_null_columns(np.zeros((2, 4, 6)), np.zeros((2, 6), bool))
