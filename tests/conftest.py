"""Shared fixtures.  `-m gpu` tests need a CUDA device and the built library;
everything else runs on CPU."""
import importlib
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

GOLDEN = ROOT / "tests" / "golden" / "reference_jacobi.npz"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built sm_100a library")


@pytest.fixture(scope="session")
def pkg():
    return importlib.import_module("pavel-s_svd_b200")


@pytest.fixture(scope="session")
def golden():
    z = np.load(GOLDEN, allow_pickle=False)
    names = [str(x) for x in z["_names"]]
    cases = {}
    for n in names:
        c = {"a": z[f"{n}/a"], "s": z[f"{n}/s"], "sweeps": int(z[f"{n}/sweeps"]), "truth": z[f"{n}/truth"],
             "kw": eval(str(z[f"{n}/kw"]))}
        if f"{n}/u" in z.files:
            c["u"], c["vh"] = z[f"{n}/u"], z[f"{n}/vh"]
        cases[n] = c
    return cases


@pytest.fixture(scope="session")
def golden_eigh():
    """The reference's jacobi_eigh outputs (h, w, v, sweeps, FP64 truth) by case."""
    z = np.load(GOLDEN, allow_pickle=False)
    return {str(n): {k: z[f"eigh_{n}/{k}"] for k in ("h", "w", "v", "sweeps", "truth")} for n in z["_eigh_names"]}


def golden_qr():
    """The reference's primitives.qr outputs (a, q, r) by case."""
    z = np.load(GOLDEN, allow_pickle=False)
    return {str(n): {k: z[f"qr_{n}/{k}"] for k in ("a", "q", "r")} for n in z["_qr_names"]}


def golden_methods():
    """The reference's svd() through its QR-based methods: input, algorithm,
    options (with the stored start basis of the projected solvers), U, s, Vh,
    FP64 truth."""
    z = np.load(GOLDEN, allow_pickle=False)
    out = {}
    for n in z["_meth_names"]:
        c = {k: z[f"meth_{n}/{k}"] for k in ("a", "u", "s", "vh", "truth")}
        c["alg"] = str(z[f"meth_{n}/alg"])
        c["kw"] = eval(str(z[f"meth_{n}/kw"]))
        if f"meth_{n}/initial_basis" in z.files:
            c["initial_basis"] = z[f"meth_{n}/initial_basis"]
        if f"meth_{n}/block_sweeps" in z.files:
            c["block_sweeps"] = int(z[f"meth_{n}/block_sweeps"])
        out[str(n)] = c
    return out


def golden_complex():
    """The reference's svd(x, 'jacobi') on complex inputs: a, U, s, Vh,
    sweeps, FP64 truth, options."""
    z = np.load(GOLDEN, allow_pickle=False)
    out = {}
    for n in z["_cx_names"]:
        c = {k: z[f"cx_{n}/{k}"] for k in ("a", "u", "s", "vh", "truth")}
        c["sweeps"] = int(z[f"cx_{n}/sweeps"])
        c["kw"] = eval(str(z[f"cx_{n}/kw"]))
        out[str(n)] = c
    return out


def golden_lab():
    """The laboratory's jacobi with a recording trace: a, U, s, Vh, the
    per-sweep largest active ratio, sweeps, options, and (with
    record_rotations) W after every round of sweep 1."""
    z = np.load(GOLDEN, allow_pickle=False)
    out = {}
    for n in z["_lab_names"]:
        c = {k: z[f"lab_{n}/{k}"] for k in ("a", "u", "s", "vh", "offs")}
        c["sweeps"] = int(z[f"lab_{n}/sweeps"])
        c["kw"] = eval(str(z[f"lab_{n}/kw"]))
        if f"lab_{n}/rounds" in z.files:
            c["rounds"] = z[f"lab_{n}/rounds"]
        out[str(n)] = c
    return out


# Columns of Q (and rows of R) fixed by the input, by QR case: beyond them a
# rank-deficient input leaves Q to rounding noise.
QR_DETERMINED = {"deficient_f64": 4}


@pytest.fixture(scope="session")
def workloads():
    return importlib.import_module("pavel-s_svd_b200.workloads")


def sigma_tol(dtype):
    """Agreement bound on sigma (relative to sigma_1) between two correct
    implementations: single precision 1e-5 (the accuracy bound of the mixed path), double 1e-12."""
    return 1e-5 if np.dtype(dtype) in (np.float32, np.complex64) else 1e-12
