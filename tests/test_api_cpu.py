"""Host-side contract of the drop-in svd(): validation order, exception
types and messages of svdbench/standalone/solvers.py:264-310 -- CPU only
(every call here fails before any device work)."""
import importlib

import numpy as np
import pytest
import torch


def test_validation_matches_reference(pkg):
    svd = pkg.svd
    a = torch.from_numpy(np.random.default_rng(0).normal(size=(12, 9)))
    with pytest.raises(ValueError, match="algorithm must be one of"):
        svd(a, "nope")
    for kw in ({"rank": 0}, {"iterations": -1}, {"oversample": -1}, {"leaf_size": 0}, {"max_sweeps": 0}):
        with pytest.raises(ValueError):
            svd(a, **kw)
    with pytest.raises(TypeError):
        svd(a.to(torch.int32))
    with pytest.raises(ValueError):
        svd(torch.zeros(0, 3))
    with pytest.raises(ValueError):
        svd(a, full_matrices=True, rank=3)


def test_no_cpu_fallback(pkg):
    a = torch.randn(6, 4)
    with pytest.raises(pkg.Unsupported):
        pkg.svd(a)
    with pytest.raises(pkg.Unsupported):
        pkg.svd(a, "bidiag_qr")
    assert issubclass(pkg.Unsupported, RuntimeError)


def test_status_mapping(pkg):
    from importlib import import_module
    S = import_module("pavel-s_svd_b200.solvers")
    N = pkg.native
    S.raise_for_status(torch.tensor([0, 0]), 60)
    with pytest.raises(ValueError, match="NaN or infinity"):
        S.raise_for_status(torch.tensor([0, N.ST_NOT_CONVERGED, N.ST_NONFINITE_IN]), 60)
    with pytest.raises(RuntimeError, match="did not converge in 7 sweeps"):
        S.raise_for_status(torch.tensor([N.ST_NOT_CONVERGED]), 7)
    with pytest.raises(RuntimeError, match="null-space completion failed"):
        S.raise_for_status(torch.tensor([N.ST_NULL_FAILED]), 7)
    with pytest.raises(RuntimeError, match="nonfinite output"):
        S.raise_for_status(torch.tensor([N.ST_NONFINITE_OUT]), 7)


def test_factory_contract(pkg):
    a = torch.randn(6, 4)
    run = pkg.factory(a, {"name": "pavel_s_svd_b200:factory", "method": "jacobi", "mode": "reduced"})
    assert callable(run) and run.metadata["vendor_factorizations"] is False
    with pytest.raises(pkg.Unsupported):
        run()  # CPU tensor: unsupported, never a silent fallback
    # metadata describes the method that runs (the harness saves it)
    for method in pkg.ALGORITHMS:
        md = pkg.factory(a, {"method": method}).metadata
        assert method in md["implementation"] and md["gpu_control"]
        assert md["rng_in_solve"] == (method in ("randomized", "subspace", "block_krylov"))
    md = pkg.factory(a, {"method": "randomized", "initial_basis": torch.randn(4, 3)}).metadata
    assert md["rng_in_solve"] is False


def test_plugin_alias_importable(pkg):
    import importlib
    assert importlib.import_module("pavel_s_svd_b200") is pkg


def test_uneven_offsets_and_order():
    from importlib import import_module
    B = import_module("pavel-s_svd_b200.batch")
    m = np.array([10, 3, 40, 7]); n = np.array([4, 5, 40, 7])
    off, total = B._aligned_offsets(m * n)
    assert (off % 4 == 0).all() and total >= (m * n).sum()
    order = B.cost_order(m, n)
    assert order[0] == 2 and sorted(order.tolist()) == [0, 1, 2, 3]


def test_streamed_chunk_weights():
    """StreamedUneven's chunk costs: small first and last chunks (their input
    and output copies are the exposed transfers), doubling to at most 4."""
    B = importlib.import_module("pavel-s_svd_b200.batch")
    assert B.chunk_weights(1) == [1.0]
    assert B.chunk_weights(3) == [1.0, 2.0, 1.0]
    assert B.chunk_weights(8) == [1.0, 2.0, 4.0, 4.0, 4.0, 4.0, 2.0, 1.0]


def test_tall_routing_thresholds(pkg):
    """Which 'jacobi' inputs take the QR-first path: beyond the register /
    large-tile rows (float32 256, float64 and complex 128) and at least twice
    as tall as wide, either orientation; empty batches never."""
    from importlib import import_module
    S = import_module("pavel-s_svd_b200.solvers")
    z = lambda *s, dt=torch.float32: torch.zeros(*s, dtype=dt)
    assert not S._qr_first(z(256, 128)) and S._qr_first(z(257, 128)) and S._qr_first(z(128, 600))
    assert not S._qr_first(z(300, 200))                       # not twice as tall as wide
    assert S._qr_first(z(129, 64, dt=torch.float64)) and not S._qr_first(z(128, 64, dt=torch.float64))
    assert S._qr_first(z(2, 200, 30, dt=torch.complex64)) and not S._qr_first(z(0, 400, 30))
