"""Blocked one-sided Jacobi on the tensor cores (BlockJacobi) against FP64
LAPACK on the same float32 input.

Stated bounds for this mixed-precision path (3xBF16 sweeps, FP64 block
eigen-solves, ~FP32-accurate 6xBF16 finish): |sigma_i - sigma_i(FP64)| <=
5e-6 sigma_1 (spectrum_error_over_sigma1), relative error <= 1e-5 for
sigma_i >= 0.1 sigma_1, reconstruction ||A - U S V^T|| / ||A|| <= 2e-5,
max |V^T V - I| <= 2e-5, max |U^T U - I| <= max(2e-5, 2e-7 cond) (the
columns of U for small sigma carry the FP32-level error eps32 * cond of the
accurate sweeps, as in the reference's FP32 solver)."""
import importlib

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def BJ():
    return importlib.import_module("pavel-s_svd_b200.blocked")


def check(a, U, S, Vh):
    a64 = a.astype(np.float64)
    sr = np.linalg.svd(a64, compute_uv=False)
    s = S.cpu().numpy().astype(np.float64)
    err1 = np.abs(s - sr).max() / sr[0]
    big = sr >= 0.1 * sr[0]
    relbig = float(np.max(np.abs(s[big] - sr[big]) / sr[big]))
    u, vh = U.cpu().numpy().astype(np.float64), Vh.cpu().numpy().astype(np.float64)
    keep = s > 0
    rec = np.linalg.norm(a64 - (u[:, keep] * s[keep]) @ vh[keep]) / np.linalg.norm(a64)
    ou = np.abs(u[:, keep].T @ u[:, keep] - np.eye(keep.sum())).max()
    ov = np.abs(vh @ vh.T - np.eye(vh.shape[0])).max()
    return err1, relbig, rec, ou, ov


@pytest.mark.parametrize("m,n,b,cond", [(512, 256, 32, 1e3), (1000, 200, 32, 1e2), (768, 384, 64, 1e4)])
def test_blocked_matches_lapack(BJ, m, n, b, cond):
    rng = np.random.default_rng(m + n)
    u, _ = np.linalg.qr(rng.standard_normal((m, n)))
    v, _ = np.linalg.qr(rng.standard_normal((n, n)))
    s = np.geomspace(1, 1 / cond, n)
    a = ((u * s) @ v.T).astype(np.float32)
    plan = BJ.BlockJacobi(m, n, b)
    U, S, Vh, info = plan.solve(torch.from_numpy(a).cuda())
    err1, relbig, rec, ou, ov = check(a, U, S, Vh)
    print(m, n, b, info["block_sweeps"], ["%.1e/%d" % x for x in info["off_per_sweep"]], err1, relbig, rec, ou, ov)
    assert err1 <= 5e-6 and relbig <= 1e-5 and rec <= 2e-5 and ou <= max(2e-5, 2e-7 * cond) and ov <= 2e-5
