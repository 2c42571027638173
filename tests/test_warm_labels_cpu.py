"""The warm start's training labels (warmstart.py), checked on CPU: the target
V0 the network learns must depend only on the SET of right singular vectors
the plain solver returned, not on their order or signs, since the solver's
order (by singular value) and signs (from the rotations) are arbitrary for a
smooth family of matrices.  The start it feeds stays the reference's Jacobi
from a given V (V = I at primitives.py:324)."""
import importlib

import pytest
import torch


def _warm():
    return importlib.import_module("pavel-s_svd_b200.warmstart")


def _orthogonal(b, n, seed):
    g = torch.Generator().manual_seed(seed)
    q, _ = torch.linalg.qr(torch.randn(b, n, n, dtype=torch.float64, generator=g))
    return q.float()


def _signed_shuffle(v, seed):
    g = torch.Generator().manual_seed(seed)
    b, n, _ = v.shape
    perm = torch.stack([torch.randperm(n, generator=g) for _ in range(b)])
    sign = torch.randint(0, 2, (b, 1, n), generator=g).float() * 2 - 1
    return torch.gather(v, 2, perm[:, None, :].expand(b, n, n)) * sign


@pytest.mark.parametrize("n", (4, 16, 64))
def test_assign_order_sees_only_the_set_of_columns(n):
    W = _warm()
    v = _orthogonal(8, n, n)
    t = W.assign_order(v)
    assert torch.equal(W.assign_order(_signed_shuffle(v, 1)), t)
    assert torch.equal(W.assign_order(_signed_shuffle(v, 2)), t)
    # the result is v's columns, each once, with positive diagonal entries
    p = (t.transpose(1, 2) @ v).abs().round()
    assert torch.equal(p.sum(1), torch.ones(8, n)) and torch.equal(p.sum(2), torch.ones(8, n))
    assert bool((torch.diagonal(t, dim1=1, dim2=2) > 0).all())


def test_assign_order_of_a_signed_permutation_is_the_identity():
    W = _warm()
    eye = torch.eye(6).expand(3, 6, 6).contiguous()
    assert torch.equal(W.assign_order(_signed_shuffle(eye, 5)), eye)


def test_assign_order_takes_the_largest_entries_first():
    """Greedy: the largest |entry| claims its row as its column position."""
    W = _warm()
    v = torch.tensor([[[0.1, 0.9, 0.0],
                       [0.8, -0.2, 0.3],
                       [0.0, 0.7, -0.95]]])
    t = W.assign_order(v)
    # -0.95 (row 2, col 2) first, then 0.9 (row 0, col 1), then col 0 to row 1
    want = torch.stack([v[0, :, 1], v[0, :, 0], -v[0, :, 2]], 1)[None]
    assert torch.equal(t, want)


def test_canonical_signs():
    W = _warm()
    v = _orthogonal(4, 12, 3)
    c = W.canonical_signs(v)
    sign = torch.randint(0, 2, (4, 1, 12), generator=torch.Generator().manual_seed(9)).float() * 2 - 1
    assert torch.equal(W.canonical_signs(v * sign), c)
    top = torch.gather(c, 1, c.abs().argmax(1, keepdim=True))
    assert bool((top > 0).all())
    assert torch.equal(c.abs(), v.abs())
    z = torch.zeros(1, 3, 3)                               # all-zero columns keep their sign
    assert torch.equal(W.canonical_signs(z), z)


def test_labels():
    W = _warm()
    v = _orthogonal(5, 8, 4)
    a = W.labels(v)
    assert a.shape == (5, 64) and a.is_contiguous()
    assert torch.equal(a, W.assign_order(v).reshape(5, 64))
    assert torch.equal(W.labels(v, order="sorted"), W.canonical_signs(v).reshape(5, 64))
    for bad in ("frame", "", None):
        with pytest.raises(ValueError):
            W.labels(v, order=bad)
    t = a.reshape(5, 8, 8)
    assert torch.allclose(t.transpose(1, 2) @ t, torch.eye(8).expand(5, 8, 8), atol=1e-5)
