"""The algorithm laboratory's jacobi on the GPU (pavel-s_svd_b200.lab, the
jb_jacobi_rounds kernel) against the reference laboratory's own run with a
recording trace (golden fixtures).

Tolerances, stated once: the per-sweep largest active ratio and W after
every round agree to 1e-10 (float64 / complex128) or 1e-4 (float32 /
complex64) relative to their scale -- same rotations, different summation
order; the sweep counts agree exactly; sigma within `sigma_tol`; singular
vectors up to a unit phase where the value is simple.
"""
import importlib
from contextlib import nullcontext

import numpy as np
import pytest
import torch

from conftest import golden_lab, sigma_tol
from test_oracle import _cmp_sigma, _cmp_vectors_phase

pytestmark = pytest.mark.gpu
DEV = "cuda"


class Recorder:
    """A trace with the laboratory's interface that keeps the per-sweep off,
    the convergence record and W after every round of sweep 1."""
    enabled = True

    def __init__(self):
        self.offs, self.rounds, self.conv, self.stages = [], [], None, []

    def wants(self, iteration=None):
        return True

    def stage(self, name, *args, **kwargs):
        self.stages.append(name)
        return nullcontext()

    def checkpoint(self, name, iteration=None, tensors=None, scalars=None, factors=None):
        if name == "sweep":
            self.offs.append(float(scalars["max_active_pair_correlation"]))
        if name.startswith("rotation_") and iteration == 1:
            self.rounds.append(tensors["W"].clone().cpu().numpy())

    def record(self, name, iteration=None, **scalars):
        self.conv = scalars


def _lab():
    return importlib.import_module("pavel-s_svd_b200.lab")


def _single(dt):
    return np.dtype(dt) in (np.float32, np.complex64)


def test_lab_jacobi_matches_reference_laboratory():
    L = _lab()
    for name, g in golden_lab().items():
        a = g["a"]
        rec = Recorder()
        u, s, vh = L.jacobi(torch.from_numpy(a).to(DEV), rec, **g["kw"])
        tol = 1e-4 if _single(a.dtype) else 1e-10
        assert rec.conv["converged"] and rec.conv["sweeps"] == g["sweeps"], name
        offs, ref = np.array(rec.offs), g["offs"]
        assert offs.shape == ref.shape, name
        assert float(np.abs(offs - ref).max()) <= tol * max(1.0, float(ref.max())), name
        real = np.float32 if _single(a.dtype) else np.float64
        _cmp_sigma(s.cpu().numpy(), g["s"], real)
        _cmp_vectors_phase(u.resolve_conj().cpu().numpy(), g["u"], g["s"], np.complex64 if _single(a.dtype)
                           else np.complex128, -1)
        _cmp_vectors_phase(vh.resolve_conj().cpu().numpy(), g["vh"], g["s"], np.complex64 if _single(a.dtype)
                           else np.complex128, -2)
        if "rounds" in g:
            got = np.stack(rec.rounds)
            assert got.shape == g["rounds"].shape, name
            assert float(np.abs(got - g["rounds"]).max()) <= tol * float(np.abs(g["rounds"]).max()), name
            assert rec.stages.count("jacobi_rotation") == g["sweeps"] * len(g["rounds"])


def test_whole_sweep_launches_equal_per_round():
    """With a trace that records nothing a sweep is one launch; the rounds
    are the same kernel work in the same order, so the results are equal.
    The last matrix is too large to stage in shared memory (the kernel then
    works on the caller's arrays): checked against LAPACK too."""
    L = _lab()
    rng = np.random.default_rng(5)
    for a in (rng.standard_normal((40, 23)), (rng.standard_normal((30, 17)) + 1j * rng.standard_normal((30, 17)))
              .astype(np.complex64), rng.standard_normal((260, 130))):
        t = torch.from_numpy(a).to(DEV)
        u1, s1, vh1 = L.jacobi(t)
        u2, s2, vh2 = L.jacobi(t, Recorder())
        assert torch.equal(s1, s2) and torch.equal(u1, u2) and torch.equal(vh1, vh2)
        truth = np.linalg.svd(a.astype(np.complex128), compute_uv=False)
        tol = 1e-5 if a.dtype == np.complex64 else 1e-12
        assert float(np.abs(s1.cpu().numpy() - truth).max() / truth[0]) <= tol


def test_lab_jacobi_errors():
    L = _lab()
    a = torch.from_numpy(np.random.default_rng(0).normal(size=(12, 9))).to(DEV)
    with pytest.raises(ValueError, match="one dense matrix"):
        L.jacobi(a[None])
    with pytest.raises(ValueError, match="one dense matrix"):
        L.jacobi(a, max_sweeps=0)
    with pytest.raises(ValueError, match="Tolerance must be positive"):
        L.jacobi(a, tol=-1.0)
    with pytest.raises(RuntimeError, match="did not converge in 1 sweeps"):
        L.jacobi(a, max_sweeps=1)
    rec = Recorder()
    u, s, vh = L.jacobi(a, rec, max_sweeps=1, require_convergence=False)
    assert rec.conv == {"converged": False, "sweeps": 1, "tolerance": 10 * np.finfo(np.float64).eps}
    u, s, vh = L.jacobi(torch.ones(5, 1, dtype=torch.float64, device=DEV))
    assert float(s[0]) == pytest.approx(5 ** 0.5)
