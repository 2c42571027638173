"""The reference's own drop-in contract, run through this library on CUDA.

The reference (uncle-Slava/Pavel-s_SVD) installed unchanged into
baseline/_ref (`pip install --no-index --no-deps --target baseline/_ref`)
provides its harness; its tests/test_standalone.py, placed beside the
install as baseline/_ref/ref_tests/test_standalone.py, provides its
standalone suite.  Each test skips, saying why, when its part is absent.

  * The harness plug-in route (svdbench/algorithms.py:90-93 and
    svdbench/cli.py:108-183): prepare() with a 'pavel_s_svd_b200:factory'
    spec and run_one() on a CUDA device; the row must come back "ok" with
    the reference's own validate() metrics within its bounds.
  * The reference's Standalone test case with SVD_TEST_DEVICE=cuda and
    svdbench.standalone.svd replaced by the integration shim: CUDA input
    of the families this library builds goes to pavel_s_svd_b200.svd, the
    rest to the reference's own torch code.
"""
import importlib
import importlib.util
import os
import sys
import types
import unittest
from pathlib import Path

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parent.parent
REF = ROOT / "baseline" / "_ref"


@pytest.fixture(scope="module")
def ref():
    if not (REF / "svdbench").is_dir():
        pytest.skip("the reference is not installed in baseline/_ref")
    if str(REF) not in sys.path:
        sys.path.insert(0, str(REF))
    importlib.import_module("pavel-s_svd_b200")          # registers pavel_s_svd_b200
    return importlib.import_module("svdbench")


def _args():
    return types.SimpleNamespace(warmup=1, repeat=2, end_to_end=False, result_callback=None)


@pytest.mark.parametrize("method,mode,dtype,shape,extra", [
    ("jacobi", "reduced", "float32", (96, 40), {}),
    ("jacobi", "full", "float64", (30, 50), {}),
    ("jacobi", "values", "complex64", (3, 40, 24), {}),
    ("block_jacobi", "reduced", "float32", (512, 256), {"block_size": 32}),
    ("gram_jacobi", "reduced", "float64", (64, 20), {}),
    ("qr", "reduced", "complex128", (50, 12), {}),
])
def test_harness_run_one(ref, method, mode, dtype, shape, extra):
    from svdbench.cli import run_one
    from svdbench.metrics import reference
    from svdbench.matrices import make_matrix
    m, n = shape[-2:]
    spec_m = dict(m=m, n=n, dtype=dtype, family="gaussian")
    if len(shape) == 3:
        spec_m["batch"] = shape[0]
    a = make_matrix(spec_m)
    refs = reference(a)
    spec = {"name": "pavel_s_svd_b200:factory", "method": method, "mode": mode, **extra}
    row = run_one(a, {"name": "b200", "seed": 7}, spec, torch.device("cuda:0"), _args(), refs)
    assert row["status"] == "ok", row.get("error")
    assert row["adapter"]["vendor_factorizations"] is False
    worst = row["metrics"]["worst"]                       # validate(): worst case over the batch
    tol = 1e-5 if dtype in ("float32", "complex64") else 1e-12
    assert worst["spectrum_error_over_sigma1"] <= tol, worst
    assert worst["singular_values_nonnegative_sorted"]
    if mode != "values":
        assert worst["reconstruction_relative_fro"] <= 10 * tol, worst


def test_harness_reports_unsupported_for_cpu(ref):
    """A CPU tensor is not this library's to solve: the harness records
    'unsupported' (algorithms.Unsupported), not an error."""
    from svdbench.cli import run_one
    from svdbench.metrics import reference
    a = np.random.default_rng(1).standard_normal((20, 10))
    row = run_one(a, {"name": "b200"}, {"name": "pavel_s_svd_b200:factory", "method": "jacobi"},
                  torch.device("cpu"), _args(), reference(a))
    assert row["status"] == "unsupported", row


def test_reference_standalone_suite_through_shim(ref):
    tests = REF / "ref_tests" / "test_standalone.py"
    if not tests.exists():
        pytest.skip("the reference's tests/test_standalone.py is not placed at baseline/_ref/ref_tests")
    b200 = sys.modules["pavel_s_svd_b200"]
    SS = importlib.import_module("svdbench.standalone")
    torch_svd = SS.svd

    def svd(a, algorithm='jacobi', **kw):                 # the integration shim
        if a.is_cuda and algorithm in b200.ALGORITHMS and (
                not a.is_complex() or algorithm in b200.COMPLEX_ALGORITHMS):
            return b200.svd(a, algorithm, **kw)
        return torch_svd(a, algorithm, **kw)

    old_env = os.environ.get("SVD_TEST_DEVICE")
    os.environ["SVD_TEST_DEVICE"] = "cuda"
    SS.svd = svd
    try:
        spec = importlib.util.spec_from_file_location("reference_test_standalone", tests)
        mod = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(mod)
        assert mod.svd is svd and mod.DEVICE == "cuda"
        suite = unittest.defaultTestLoader.loadTestsFromTestCase(mod.Standalone)
        result = unittest.TestResult()
        suite.run(result)
    finally:
        SS.svd = torch_svd
        if old_env is None:
            os.environ.pop("SVD_TEST_DEVICE", None)
        else:
            os.environ["SVD_TEST_DEVICE"] = old_env
        torch.set_num_threads(os.cpu_count() or 1)
    problems = [f"{t}: {msg[-600:]}" for t, msg in result.failures + result.errors]
    assert result.testsRun >= 12 and not problems, "\n".join(problems)
