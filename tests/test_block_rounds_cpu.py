"""The host logic of the block_jacobi rounds engine (block_rounds.py) on CPU:
the group tournament and its bucketing by column count, the gather / solve /
scatter of a round's pair subproblems, the convergence test, the sort and
the cut.  The pair solves, which run on the GPU in the product, are done
here by the NumPy oracle's jacobi_svd (the reference's inner solver,
primitives.py:316-367) on the batched subproblems, and the null completion
by the oracle's complete_null_columns, so the engine must
reproduce the reference's own block_jacobi runs (golden fixtures): sigma
within sigma_tol, block sweeps within one.  (LAPACK is no stand-in: its V
leaves the columns correlated at ~1e-14, above the 40 eps the block
convergence test asks for; the block method needs Jacobi-accurate pair
solves.)"""
import importlib

import numpy as np
import pytest
import torch

from conftest import golden_methods, sigma_tol
from oracle import jacobi_oracle as O


def _mods():
    return importlib.import_module("pavel-s_svd_b200.block_rounds"), importlib.import_module("pavel-s_svd_b200.solvers")


def _oracle_complete(u, keep):
    """The oracle's null completion (primitives.py:430-455) on CPU tensors:
    the product's runs on the GPU (jb_complete_null)."""
    return torch.from_numpy(O.complete_null_columns(np.ascontiguousarray(u.resolve_conj().numpy()), keep.numpy()))


def _oracle_pairs(y):
    _, _, v, _ = O.jacobi_svd(y.resolve_conj().numpy())
    return None, None, torch.from_numpy(np.ascontiguousarray(v))


def test_schedule_is_the_group_tournament():
    BR, _ = _mods()
    for n, w in ((11, 3), (22, 4), (9, 2), (16, 8), (7, 5)):
        groups = BR.groups_of(n, w)
        rounds = BR.schedule(n, w, "cpu")
        ref = list(O.round_robin(len(groups)))
        assert len(rounds) == len(ref)
        for buckets, pairs in zip(rounds, ref):
            got = sorted(tuple(row) for idx in buckets for row in idx.tolist())
            want = sorted(tuple(groups[i] + groups[j]) for i, j in pairs if len(groups[i] + groups[j]) >= 2)
            assert got == want
            for idx in buckets:                    # one bucket per column count, disjoint columns
                assert len({len(r) for r in idx.tolist()}) == 1
            cols = [c for idx in buckets for c in idx.reshape(-1).tolist()]
            assert len(cols) == len(set(cols))


def test_rounds_engine_matches_reference_runs():
    BR, S = _mods()
    seen = 0
    for name, g in golden_methods().items():
        if g["alg"] != "block_jacobi":
            continue
        a = g["a"]
        x = torch.from_numpy(a.reshape(-1, *a.shape[-2:]).copy())
        stats = {}
        opts = dict(g["kw"])
        u, s, v = BR.raw(x, stats, opts, _oracle_pairs, lambda: None, _oracle_complete)
        s = s.numpy().reshape(g["s"].shape)
        dt = a.dtype
        k = s.shape[-1]
        np.testing.assert_allclose(s, g["s"], rtol=0, atol=sigma_tol(dt) * float(np.max(g["s"])) * 10)
        assert abs(stats["block_sweeps"] - g["block_sweeps"]) <= 1, name
        un, vn = u.numpy(), v.numpy()
        eye = np.eye(k)
        tol = 1e-4 if dt in (np.float32, np.complex64) else 1e-10
        assert float(np.abs(np.conj(np.swapaxes(un, -1, -2)) @ un - eye).max()) <= tol
        rec = (un * s.reshape(un.shape[0], -1)[:, None, :]) @ np.conj(np.swapaxes(vn, -1, -2))
        assert float(np.abs(rec - a.reshape(rec.shape)).max()) <= tol * max(1.0, float(np.abs(a).max())) * 10
        seen += 1
    assert seen >= 6


def test_rounds_engine_errors():
    BR, S = _mods()
    x = torch.randn(2, 20, 12, dtype=torch.float64)
    with pytest.raises(RuntimeError, match="block Jacobi did not converge"):
        BR.raw(x, {}, {"block_size": 3, "max_sweeps": 1}, _oracle_pairs, lambda: None, _oracle_complete)
    calls = []
    BR.raw(x, {}, {"block_size": 3}, _oracle_pairs, lambda: calls.append(1), _oracle_complete)
    assert len(calls) >= 2                          # status words checked once per block sweep
    u, s, v = BR.raw(torch.zeros(0, 20, 12, dtype=torch.float64), {}, {"block_size": 3}, _oracle_pairs,
                     lambda: None, _oracle_complete)
    assert u.shape == (0, 20, 12) and s.shape == (0, 12) and v.shape == (0, 12, 12)
