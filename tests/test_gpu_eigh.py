"""jacobi_eigh on the GPU (jb_eigh_f32/_f64) against the reference's own
outputs (golden fixtures) and FP64 LAPACK.

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
    w = w.cpu().numpy().astype(np.float64)
    v = v.cpu().numpy().astype(np.float64)
    scale = np.abs(truth).max(axis=-1, keepdims=True)
    assert float((np.abs(w - truth) / scale).max()) <= 10 * n * e
    eye = np.eye(n)
    assert float(np.abs(np.swapaxes(v, -1, -2) @ v - eye).max()) <= 100 * n * e
    res = np.abs(h.astype(np.float64) @ v - v * w[:, None, :]).max(axis=(-2, -1)) / scale[:, 0]
    assert float(res.max()) <= 100 * n * e


def test_eigh_matches_reference_golden(E, golden_eigh):
    for name, g in golden_eigh.items():
        h = g["h"]
        w, v, sw = E.jacobi_eigh(torch.from_numpy(h).cuda())
        assert w.dtype == torch.from_numpy(h).dtype
        _check(h, w, v, g["truth"])
        assert abs(sw - int(g["sweeps"])) <= 2, name


@pytest.mark.parametrize("n,batch,dtype", [(64, 5, torch.float32), (127, 2, torch.float64), (200, 2, torch.float32),
                                           (1, 3, torch.float64), (2, 4, torch.float32)])
def test_eigh_sizes(E, n, batch, dtype):
    """Even, odd (padded) and large sizes; V in global memory above n = 118."""
    g = torch.Generator().manual_seed(n)
    x = torch.randn(batch, n, n, generator=g, dtype=torch.float64)
    h = (x + x.transpose(1, 2)).to(dtype)
    w, v, sw = E.jacobi_eigh(h.cuda())
    truth = np.linalg.eigvalsh(h.double().numpy())
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
