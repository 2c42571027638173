"""Generate the golden fixtures of the Jacobi path from the reference itself.

Run once, in a container where uncle-Slava/Pavel-s_SVD is checked out, with
the path of that checkout as the argument or in REFERENCE_ROOT:

    python tests/golden/make_golden.py <path of the reference checkout>

It imports the reference's ``svdbench.standalone.svd`` and
``svdbench.matrices.make_matrix`` unchanged, runs ``svd(x, 'jacobi', ...)``
on CPU (1 thread, as the reference's own tests do) and writes
``tests/golden/reference_jacobi.npz``: for every case the input, the
reference's U, s, Vh, jacobi_sweeps, and SciPy FP64 singular values; the
reference's jacobi_eigh, qr and QR-based solvers ('qr', 'tsqr' and the
projected ones from a stored start basis) on their own cases.  The GPU box
never runs this script; tests read only the .npz.
"""
from __future__ import annotations

import hashlib
import importlib.util
import os
import sys
from pathlib import Path

import numpy as np

REF: Path | None = None   # the reference checkout, set by main()
HERE = Path(__file__).resolve().parent
REPO = HERE.parent.parent


def _workloads():
    spec = importlib.util.spec_from_file_location("workloads", REPO / "pavel-s_svd_b200" / "workloads.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def cases(make_matrix):
    """(name, input array, svd kwargs) -- mirrors the reference's own test
    inputs (tests/test_standalone.py:47-90, 187-207) in real dtypes, the
    real-valued byte-exact corpus (corpus/standalone/*.npy) and samples of
    the benchmark workloads."""
    out = []
    for dt in ("float32", "float64"):
        for m, n in ((13, 7), (7, 13)):
            out.append((f"gauss_{dt}_{m}x{n}_b2", make_matrix(dict(m=m, n=n, batch=2, dtype=dt, family="gaussian")), {}))
    special = [np.zeros((9, 5)), np.eye(7), np.diag([0., 2., 0., 3., 1.]),
               make_matrix(dict(m=15, n=7, dtype="float64", family="low_rank", rank=3, tail=0)),
               make_matrix(dict(m=15, n=7, dtype="float64", family="clustered"))]
    base = make_matrix(dict(m=11, n=5, dtype="float64", family="gaussian"))
    special += [base * 1e-150, base * 1e150]
    for i, a in enumerate(special):
        out.append((f"special{i}", np.ascontiguousarray(a), {}))
    for shape in ((1, 1), (8, 1), (1, 8), (10, 4), (4, 10)):
        a = make_matrix(dict(m=shape[0], n=shape[1], family="gaussian", dtype="float64"))
        out.append((f"full_{shape[0]}x{shape[1]}", a, {"full_matrices": True}))
        out.append((f"values_{shape[0]}x{shape[1]}", a, {"values_only": True}))
    out.append(("geometric_24x9", make_matrix(dict(m=24, n=9, dtype="float64", family="geometric", condition=1e8)), {}))
    out.append(("multidim_2x3x9x5", np.random.default_rng(22).normal(size=(2, 3, 9, 5)), {}))
    out.append(("rank4_of_13x7", make_matrix(dict(m=13, n=7, dtype="float32", family="gaussian")), {"rank": 4}))
    out.append(("full_f32_12x5", make_matrix(dict(m=12, n=5, dtype="float32", family="low_rank", rank=2, tail=0)),
                {"full_matrices": True}))
    corpus = REF / "corpus" / "standalone"
    for name in ("square32", "tall256x16", "batch8x16", "condition1e8", "condition1e12", "rank_deficient", "zero",
                 "square64", "tall2048x32"):
        p = corpus / f"{name}.npy"
        if p.exists():
            out.append((f"corpus_{name}", np.load(p, allow_pickle=False), {}))
    wl = _workloads()
    out.append(("plain_single_256x128", wl.plain_single(), {"tol": 1e-6, "max_sweeps": 30}))
    for i, a in enumerate(wl.uneven_batch(48)):
        out.append((f"uneven_{i:02d}", a, {}))
    return out


def eigh_cases(make_matrix):
    """(name, batch of symmetric matrices): Grams of the reference's matrix
    families (what gram_jacobi feeds jacobi_eigh, solvers.py:99-120), an odd
    size (padding), an indefinite matrix and a diagonal one."""
    out = []
    for dt in ("float32", "float64"):
        a = make_matrix(dict(m=24, n=10, batch=3, dtype=dt, family="gaussian"))
        out.append((f"gram_gauss_{dt}_10", np.ascontiguousarray(np.swapaxes(a, -1, -2) @ a)))
        a = make_matrix(dict(m=20, n=7, batch=2, dtype=dt, family="gaussian"))
        out.append((f"gram_gauss_{dt}_7", np.ascontiguousarray(np.swapaxes(a, -1, -2) @ a)))
    a = make_matrix(dict(m=40, n=16, dtype="float64", family="geometric", condition=1e4))
    out.append(("gram_geometric_16", np.ascontiguousarray((a.T @ a)[None])))
    rng = np.random.default_rng(31)
    x = rng.standard_normal((2, 12, 12))
    out.append(("indefinite_12", np.ascontiguousarray(x + np.swapaxes(x, -1, -2))))
    out.append(("diagonal_6", np.diag([3.0, -1.0, 2.0, 0.0, 5.0, 1.0])[None].copy()))
    for dt in ("complex64", "complex128"):     # Hermitian Grams (gram_jacobi on complex input)
        a = make_matrix(dict(m=20, n=9, batch=2, dtype=dt, family="gaussian"))
        g = np.conj(np.swapaxes(a, -1, -2)) @ a
        out.append((f"gram_gauss_{dt}_9", np.ascontiguousarray((g + np.conj(np.swapaxes(g, -1, -2))) / 2)))
    return out


def qr_cases(make_matrix):
    """(name, batch of tall matrices) for primitives.qr (primitives.py:74-89):
    Gaussian in both dtypes, square, a zero column and a repeated column (the
    reflector's trivial and rank-deficient branches), a tall f32 batch."""
    out = []
    for dt in ("float32", "float64"):
        out.append((f"gauss_{dt}", make_matrix(dict(m=20, n=7, batch=3, dtype=dt, family="gaussian"))))
    out.append(("square_f64", make_matrix(dict(m=16, n=16, batch=2, dtype="float64", family="gaussian"))))
    a = make_matrix(dict(m=18, n=6, batch=2, dtype="float64", family="gaussian")).copy()
    a[:, :, 2] = 0.0
    a[:, :, 4] = a[:, :, 1]
    a[1, 3:, 5] = 0.0
    out.append(("deficient_f64", a))
    out.append(("tall_f32", make_matrix(dict(m=130, n=33, batch=2, dtype="float32", family="gaussian"))))
    for dt in ("complex64", "complex128"):
        out.append((f"gauss_{dt}", make_matrix(dict(m=21, n=8, batch=2, dtype=dt, family="gaussian"))))
    return out


def method_cases(make_matrix):
    """(name, input, algorithm, kwargs) for the Jacobi-based methods built on
    QR: 'qr' and 'tsqr' (solvers.py:71-96, 245-248), tall and wide, with
    tiles that force several leaves and a merged short last leaf; the
    projected solvers (solvers.py:185-220) from a stored start basis
    (initial_basis), since their own sketch comes from torch's generator."""
    rng = np.random.default_rng(41)
    out = []
    for dt in ("float32", "float64"):
        out.append((f"qr_{dt}", make_matrix(dict(m=40, n=12, batch=3, dtype=dt, family="gaussian")), "qr", {}))
        out.append((f"qr_wide_{dt}", make_matrix(dict(m=9, n=20, batch=2, dtype=dt, family="gaussian")), "qr", {}))
        out.append((f"tsqr_{dt}", make_matrix(dict(m=53, n=8, batch=2, dtype=dt, family="gaussian")), "tsqr",
                    {"tile_rows": 10}))
        a = make_matrix(dict(m=30, n=12, batch=2, dtype=dt, family="geometric", condition=1e3))
        for alg, rank, over, it in (("randomized", 4, 3, 2), ("subspace", 5, 2, 3), ("block_krylov", 3, 2, 2)):
            om = rng.standard_normal((2, 12, rank + over)).astype(dt)
            out.append((f"{alg}_{dt}", a, alg, {"rank": rank, "oversample": over, "iterations": it,
                                                "initial_basis": om}))
    a = make_matrix(dict(m=10, n=26, batch=2, dtype="float64", family="gaussian"))
    out.append(("randomized_wide_float64", a, "randomized",
                {"rank": 4, "oversample": 4, "initial_basis": rng.standard_normal((2, 26, 8))}))
    # complex inputs (tests/test_standalone.py:47-54 runs every family on them)
    for dt in ("complex64", "complex128"):
        out.append((f"qr_{dt}", make_matrix(dict(m=13, n=7, batch=2, dtype=dt, family="gaussian")), "qr", {}))
        out.append((f"tsqr_wide_{dt}", make_matrix(dict(m=7, n=13, batch=2, dtype=dt, family="gaussian")), "tsqr",
                    {"tile_rows": 7}))
        a = make_matrix(dict(m=24, n=10, batch=2, dtype=dt, family="geometric", condition=1e3))
        om = (rng.standard_normal((2, 10, 6)) + 1j * rng.standard_normal((2, 10, 6))).astype(dt)
        out.append((f"subspace_{dt}", a, "subspace", {"rank": 3, "oversample": 3, "iterations": 2,
                                                      "initial_basis": om}))
        out.append((f"gram_{dt}", make_matrix(dict(m=15, n=8, batch=2, dtype=dt, family="gaussian")), "gram_jacobi",
                    {}))
        out.append((f"gram_wide_{dt}", make_matrix(dict(m=6, n=11, batch=2, dtype=dt, family="gaussian")),
                    "gram_jacobi", {}))
    # block_jacobi (solvers.py:30-68): ragged last group, an odd group count
    # (padded with an empty group), wide input, a rank-deficient matrix
    # (cut columns completed), both real and both complex dtypes
    out.append(("block_float64", make_matrix(dict(m=20, n=11, batch=2, dtype="float64", family="gaussian")),
                "block_jacobi", {"block_size": 3}))
    out.append(("block_wide_float64", make_matrix(dict(m=9, n=22, batch=2, dtype="float64", family="gaussian")),
                "block_jacobi", {}))
    out.append(("block_float32", make_matrix(dict(m=24, n=10, batch=2, dtype="float32", family="gaussian")),
                "block_jacobi", {}))
    out.append(("block_lowrank_float64", make_matrix(dict(m=18, n=8, dtype="float64", family="low_rank", rank=3,
                                                          tail=0)), "block_jacobi", {"block_size": 2}))
    out.append(("block_complex64", make_matrix(dict(m=15, n=9, batch=2, dtype="complex64", family="gaussian")),
                "block_jacobi", {}))
    out.append(("block_wide_complex128", make_matrix(dict(m=8, n=14, batch=2, dtype="complex128",
                                                          family="gaussian")), "block_jacobi", {"block_size": 3}))
    return out


def complex_cases(make_matrix):
    """(name, input, svd kwargs) for 'jacobi' on complex dtypes: the
    reference's own complex test inputs (tests/test_standalone.py:47-54,
    68-80, 92-98, 187-194) -- Gaussian tall and wide batches in both
    precisions, full bases of small shapes, a rank-4 matrix (cut values and
    null completion), a multi-dimensional batch -- plus a zero matrix and a
    truncated rank."""
    out = []
    for dt in ("complex64", "complex128"):
        for m, n in ((13, 7), (7, 13)):
            out.append((f"gauss_{dt}_{m}x{n}_b2", make_matrix(dict(m=m, n=n, batch=2, dtype=dt, family="gaussian")),
                        {}))
    for shape in ((1, 1), (8, 1), (1, 8), (10, 4), (4, 10)):
        a = make_matrix(dict(m=shape[0], n=shape[1], family="gaussian", dtype="complex128"))
        out.append((f"full_{shape[0]}x{shape[1]}", a, {"full_matrices": True}))
    out.append(("rank4_40x25", make_matrix(dict(m=40, n=25, dtype="complex128", family="low_rank", rank=4, tail=0)),
                {}))
    rng = np.random.default_rng(23)
    out.append(("multidim_2x3x9x5", rng.normal(size=(2, 3, 9, 5)) + 1j * rng.normal(size=(2, 3, 9, 5)), {}))
    out.append(("zero_9x5", np.zeros((9, 5), np.complex128), {}))
    out.append(("rank3_of_c64_13x7", make_matrix(dict(m=13, n=7, dtype="complex64", family="gaussian")),
                {"rank": 3}))
    return out


class _Recorder:
    """A laboratory trace (svdbench/laboratory/trace.py interface) that keeps
    the per-sweep off, the convergence record and W after every round of
    sweep 1."""
    enabled = True

    def __init__(self):
        self.offs, self.rounds, self.conv = [], [], None

    def wants(self, iteration=None):
        return True

    def stage(self, *args, **kwargs):
        from contextlib import nullcontext
        return nullcontext()

    def checkpoint(self, name, iteration=None, tensors=None, scalars=None, factors=None):
        if name == "sweep":
            self.offs.append(float(scalars["max_active_pair_correlation"]))
        if name.startswith("rotation_") and iteration == 1:
            self.rounds.append(tensors["W"].clone().resolve_conj().numpy())

    def record(self, name, iteration=None, **scalars):
        self.conv = scalars


def lab_cases():
    """(name, matrix, kwargs) for the laboratory's jacobi
    (algorithm_laboratory/algorithms.py:105-157): odd and even widths, both
    real precisions, a wide complex matrix, a rank-deficient one."""
    rng = np.random.default_rng(51)
    out = [("odd_f64_12x7", rng.standard_normal((12, 7)), {"record_rotations": True}),
           ("even_f32_16x10", rng.standard_normal((16, 10)).astype(np.float32), {}),
           ("wide_c128_6x11", rng.standard_normal((6, 11)) + 1j * rng.standard_normal((6, 11)),
            {"record_rotations": True}),
           ("c64_9x5", (rng.standard_normal((9, 5)) + 1j * rng.standard_normal((9, 5))).astype(np.complex64), {})]
    b = rng.standard_normal((10, 3)) @ rng.standard_normal((3, 6))
    out.append(("rank3_f64_10x6", b, {}))
    return out


def main():
    global REF
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("REFERENCE_ROOT")
    if not root:
        sys.exit("usage: make_golden.py <reference checkout> (or set REFERENCE_ROOT)")
    REF = Path(root)
    sys.path.insert(0, str(REF))
    import torch
    import scipy.linalg
    from svdbench.standalone import svd
    from svdbench.matrices import make_matrix
    torch.set_num_threads(1)
    blob = {}
    names = []
    for name, a, kw in cases(make_matrix):
        a = np.ascontiguousarray(a)
        u, s, vh, info = svd(torch.from_numpy(a.copy()), "jacobi", return_info=True, **kw)
        flat = a.reshape(-1, *a.shape[-2:]).astype(np.float64)
        truth = np.stack([scipy.linalg.svd(x, compute_uv=False, lapack_driver="gesvd") for x in flat])
        blob[f"{name}/a"] = a
        blob[f"{name}/s"] = s.numpy()
        if u is not None and a.size <= 20000:
            blob[f"{name}/u"] = u.numpy()
            blob[f"{name}/vh"] = vh.numpy()
        blob[f"{name}/sweeps"] = np.array(info["jacobi_sweeps"])
        blob[f"{name}/truth"] = truth
        blob[f"{name}/kw"] = np.array(repr(kw))
        blob[f"{name}/sha256"] = np.array(hashlib.sha256(a.tobytes(order="C")).hexdigest())
        names.append(name)
        print(f"{name:28s} {str(a.shape):18s} {a.dtype}  sweeps={info['jacobi_sweeps']}")
    blob["_names"] = np.array(names)
    # jacobi_eigh (primitives.py:370-427): symmetric inputs, the reference's
    # w (ascending), V and sweeps
    from svdbench.standalone import primitives as P
    enames = []
    for name, h in eigh_cases(make_matrix):
        w, v, sw = P.jacobi_eigh(torch.from_numpy(h.copy()))
        blob[f"eigh_{name}/h"] = h
        blob[f"eigh_{name}/w"] = w.numpy()
        blob[f"eigh_{name}/v"] = v.resolve_conj().numpy()
        blob[f"eigh_{name}/sweeps"] = np.array(sw)
        blob[f"eigh_{name}/truth"] = np.stack([np.linalg.eigvalsh(x.astype(np.complex128 if np.iscomplexobj(x)
                                                                           else np.float64)) for x in h])
        enames.append(name)
        print(f"eigh {name:22s} {str(h.shape):14s} {h.dtype}  sweeps={sw}")
    blob["_eigh_names"] = np.array(enames)
    # primitives.qr: the reference's Q and R
    qnames = []
    for name, a in qr_cases(make_matrix):
        a = np.ascontiguousarray(a)
        q, r = P.qr(torch.from_numpy(a.copy()))
        blob[f"qr_{name}/a"], blob[f"qr_{name}/q"], blob[f"qr_{name}/r"] = a, q.resolve_conj().numpy(), r.resolve_conj().numpy()
        qnames.append(name)
        print(f"qr {name:24s} {str(a.shape):14s} {a.dtype}")
    blob["_qr_names"] = np.array(qnames)
    # the QR-based solvers through the public svd()
    mnames = []
    for name, a, alg, kw in method_cases(make_matrix):
        a = np.ascontiguousarray(a)
        tkw = {k: (torch.from_numpy(np.ascontiguousarray(v)) if isinstance(v, np.ndarray) else v) for k, v in kw.items()}
        u, s, vh, info = svd(torch.from_numpy(a.copy()), alg, return_info=True, **tkw)
        flat = a.reshape(-1, *a.shape[-2:]).astype(np.complex128 if np.iscomplexobj(a) else np.float64)
        blob[f"meth_{name}/a"] = a
        blob[f"meth_{name}/u"] = u.resolve_conj().numpy()
        blob[f"meth_{name}/s"] = s.numpy()
        blob[f"meth_{name}/vh"] = vh.resolve_conj().numpy()
        blob[f"meth_{name}/truth"] = np.stack([scipy.linalg.svd(x, compute_uv=False, lapack_driver="gesvd")
                                               for x in flat])
        blob[f"meth_{name}/alg"] = np.array(alg)
        if "block_sweeps" in info:
            blob[f"meth_{name}/block_sweeps"] = np.array(info["block_sweeps"])
        blob[f"meth_{name}/kw"] = np.array(repr({k: v for k, v in kw.items() if k != "initial_basis"}))
        if "initial_basis" in kw:
            blob[f"meth_{name}/initial_basis"] = np.ascontiguousarray(kw["initial_basis"])
        mnames.append(name)
        print(f"{alg} {name:24s} {str(a.shape):14s} {a.dtype}  sweeps={info.get('jacobi_sweeps')}")
    blob["_meth_names"] = np.array(mnames)
    # 'jacobi' on complex inputs
    cnames = []
    for name, a, kw in complex_cases(make_matrix):
        a = np.ascontiguousarray(a)
        u, s, vh, info = svd(torch.from_numpy(a.copy()), "jacobi", return_info=True, **kw)
        flat = a.reshape(-1, *a.shape[-2:]).astype(np.complex128)
        blob[f"cx_{name}/a"] = a
        blob[f"cx_{name}/u"] = u.resolve_conj().numpy()
        blob[f"cx_{name}/s"] = s.numpy()
        blob[f"cx_{name}/vh"] = vh.resolve_conj().numpy()
        blob[f"cx_{name}/sweeps"] = np.array(info["jacobi_sweeps"])
        blob[f"cx_{name}/truth"] = np.stack([scipy.linalg.svd(x, compute_uv=False, lapack_driver="gesvd")
                                             for x in flat])
        blob[f"cx_{name}/kw"] = np.array(repr(kw))
        cnames.append(name)
        print(f"complex {name:24s} {str(a.shape):14s} {a.dtype}  sweeps={info['jacobi_sweeps']}")
    blob["_cx_names"] = np.array(cnames)
    # the laboratory's jacobi with a recording trace
    from algorithm_laboratory import algorithms as L
    lnames = []
    for name, a, kw in lab_cases():
        a = np.ascontiguousarray(a)
        rec = _Recorder()
        u, s, vh = L.jacobi(torch.from_numpy(a.copy()), rec, **kw)
        blob[f"lab_{name}/a"] = a
        blob[f"lab_{name}/u"] = u.resolve_conj().numpy()
        blob[f"lab_{name}/s"] = s.numpy()
        blob[f"lab_{name}/vh"] = vh.resolve_conj().numpy()
        blob[f"lab_{name}/offs"] = np.array(rec.offs)
        blob[f"lab_{name}/sweeps"] = np.array(rec.conv["sweeps"])
        blob[f"lab_{name}/kw"] = np.array(repr(kw))
        if rec.rounds:
            blob[f"lab_{name}/rounds"] = np.stack(rec.rounds)
        lnames.append(name)
        print(f"lab {name:20s} {str(a.shape):10s} {a.dtype}  sweeps={rec.conv['sweeps']} rounds={len(rec.rounds)}")
    blob["_lab_names"] = np.array(lnames)
    np.savez_compressed(HERE / "reference_jacobi.npz", **blob)
    print("wrote", HERE / "reference_jacobi.npz")


if __name__ == "__main__":
    main()
