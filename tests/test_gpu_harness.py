"""The drop-in the way the reference's callers use it, on the GPU:
  * the harness plug-in (svdbench/algorithms.py:90-93, cli.py:113-124):
    factory(device_tensor, spec) -> a zero-argument callable, run under
    torch.inference_mode(), its .diagnostics and .metadata saved, the input
    preserved, for every algorithm and output mode;
  * the playground / lab callers (engine.py:114-115, 153-156;
    algorithm_laboratory/algorithms.py:21-24): svd(x, 'jacobi') on a 2-D
    tensor with the options they pass along (oversample, iterations, seed,
    steps), which the Jacobi ignores.
Results must equal a direct svd() call with the same options, bit for bit."""
import importlib

import pytest
import torch

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def pkg():
    return importlib.import_module("pavel-s_svd_b200")


@pytest.mark.parametrize("method", ["jacobi", "block_jacobi", "gram_jacobi", "qr", "tsqr", "randomized", "subspace",
                                    "block_krylov"])
@pytest.mark.parametrize("mode", ["reduced", "full", "values"])
def test_factory_under_inference_mode(pkg, method, mode):
    g = torch.Generator(device="cuda").manual_seed(5)
    a = torch.randn(3, 40, 24, device="cuda", generator=g)
    keep = a.clone()
    spec = {"name": "pavel_s_svd_b200:factory", "method": method, "mode": mode, "seed_offset": 3}
    if method in ("randomized", "subspace", "block_krylov"):
        spec.update(rank=6, oversample=4)
    with torch.inference_mode():
        run = pkg.factory(a, spec)
        if "rank" in spec and mode == "full":      # a truncated rank with full bases: the reference's error
            with pytest.raises(ValueError, match="full_matrices and truncated rank"):
                run()
            return
        u, s, vh = run()
    assert torch.equal(a, keep)
    assert run.diagnostics["algorithm"] == method and run.diagnostics["vendor_factorizations"] == 0
    assert run.metadata["vendor_factorizations"] is False
    opts = {k: v for k, v in spec.items() if k not in ("name", "method", "mode", "seed_offset")}
    u2, s2, vh2 = pkg.svd(a, method, full_matrices=mode == "full", values_only=mode == "values", **opts)
    assert torch.equal(s, s2)
    if mode == "values":
        assert u is None and vh is None
    else:
        assert torch.equal(u, u2) and torch.equal(vh, vh2)
        if mode == "full":
            assert u.shape == (3, 40, 40) and vh.shape == (3, 24, 24)


def test_playground_and_lab_calls(pkg):
    x = torch.randn(30, 12, device="cuda", dtype=torch.float64)
    u, s, vh = pkg.svd(x, "jacobi", oversample=8, iterations=2, seed=7, steps=4)
    u0, s0, vh0 = pkg.svd(x, "jacobi")
    assert torch.equal(s, s0) and torch.equal(u, u0) and torch.equal(vh, vh0)
    assert u.shape == (30, 12) and s.shape == (12,) and vh.shape == (12, 12)
    rec = (u * s) @ vh
    assert float((rec - x).abs().max()) <= 1e-12 * float(x.abs().max()) * 30
