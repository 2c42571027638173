"""The oracle against the reference's own outputs (golden fixtures made by
tests/golden/make_golden.py from uncle-Slava/Pavel-s_SVD) -- CPU only."""
import numpy as np
import pytest

from oracle import jacobi_oracle as O
from oracle import c_oracle as C
from conftest import QR_DETERMINED, golden_complex, golden_methods, golden_qr, sigma_tol


def _cmp_sigma(s, ref, dtype, factor=1.0):
    s = np.asarray(s, np.float64).reshape(ref.shape)
    top = max(float(np.abs(ref).max()), np.finfo(np.float64).tiny)
    err = float(np.abs(s - ref).max()) / top
    assert err <= factor * sigma_tol(dtype), err
    return err


def _cmp_vectors(u, ref, s, dtype, axis):
    """Columns (axis=-1) or rows (axis=-2) agree up to sign where the singular
    value is simple (gap > 1e-3 relative); returns max deviation."""
    ref = np.asarray(ref, np.float64)
    ref = ref.reshape(-1, *ref.shape[-2:])
    u = np.asarray(u, np.float64).reshape(ref.shape)
    tol = 1e-3 if np.dtype(dtype) == np.float32 else 1e-8
    s = np.asarray(s, np.float64).reshape(ref.shape[0], -1)
    worst = 0.0
    for b in range(u.shape[0]):
        sb = s[b]
        ncols = ref.shape[-1] if axis == -1 else ref.shape[-2]
        for j in range(min(len(sb), ncols)):
            gap = min([abs(sb[j] - sb[i]) for i in range(len(sb)) if i != j] or [np.inf])
            if sb[j] == 0 or gap <= 1e-3 * sb[0]:
                continue
            x = u[b][:, j] if axis == -1 else u[b][j, :]
            y = ref[b][:, j] if axis == -1 else ref[b][j, :]
            d = min(np.abs(x - y).max(), np.abs(x + y).max())
            worst = max(worst, d)
    assert worst <= tol, worst
    return worst


def test_numpy_oracle_matches_reference(golden):
    for name, c in golden.items():
        a = c["a"]
        u, s, vh, info = O.svd(a, "jacobi", return_info=True, **c["kw"])
        _cmp_sigma(s, c["s"], a.dtype)
        if a.dtype == np.float64:
            assert info["jacobi_sweeps"] == c["sweeps"], name
        else:
            assert abs(info["jacobi_sweeps"] - c["sweeps"]) <= 1, name
        if "u" in c and u is not None:
            _cmp_vectors(u, c["u"], c["s"], a.dtype, -1)
            _cmp_vectors(vh, c["vh"], c["s"], a.dtype, -2)


def _c_oracle(a, kw):
    x = a.reshape(-1, *a.shape[-2:])
    rank = kw.get("rank")
    u, s, vh, sweeps, status = C.svd_batched(x, rank=rank, full_matrices=kw.get("full_matrices", False),
                                             values_only=kw.get("values_only", False), tol=kw.get("tol"),
                                             max_sweeps=kw.get("max_sweeps", 60))
    return u, s, vh, sweeps, status


def test_c_oracle_matches_reference(golden):
    for name, c in golden.items():
        a = c["a"]
        u, s, vh, sweeps, status = _c_oracle(a, c["kw"])
        assert (status == 0).all(), name
        _cmp_sigma(s, c["s"], a.dtype)
        if a.dtype == np.float64:
            assert int(sweeps.max()) == c["sweeps"], name
        else:
            assert abs(int(sweeps.max()) - c["sweeps"]) <= 1, name
        if "u" in c and u is not None:
            _cmp_vectors(u.reshape(c["u"].shape), c["u"], c["s"], a.dtype, -1)
            _cmp_vectors(vh.reshape(c["vh"].shape), c["vh"], c["s"], a.dtype, -2)


def test_oracle_pins_reference_sweeps_of_corpus(golden):
    """Sweep counts the reference recorded for the byte-exact corpus
    (results/standalone-hetzner.jsonl lines 5, 23, 59, 77, 95, 131, 149)."""
    recorded = {"corpus_square32": 8, "corpus_tall256x16": 6, "corpus_batch8x16": 7, "corpus_condition1e8": 12,
                "corpus_condition1e12": 14, "corpus_rank_deficient": 5, "corpus_zero": 1}
    for name, sw in recorded.items():
        assert golden[name]["sweeps"] == sw, name
        _, _, _, sweeps, _ = _c_oracle(golden[name]["a"], {})
        assert int(sweeps.max()) == sw, name


def test_corpus_inputs_are_the_reference_bytes(golden):
    """SHA-256 prefixes recorded by the reference (results/standalone-hetzner.jsonl)."""
    import hashlib
    recorded = {"corpus_square32": "52d63f80514ec9f0", "corpus_tall256x16": "d6e0fa184b2d7ebd",
                "corpus_batch8x16": "64f1e958765e61c4", "corpus_condition1e8": "f4e8c3c129a2e86f",
                "corpus_condition1e12": "d3e0049c7534acfe", "corpus_rank_deficient": "d929a6987cec069d",
                "corpus_zero": "a1a4f5721c1c4610", "corpus_tall2048x32": "d9e8b9afed4d1eb6"}
    for name, h in recorded.items():
        assert hashlib.sha256(golden[name]["a"].tobytes()).hexdigest().startswith(h), name


def test_oracle_errors_follow_reference():
    a = np.random.default_rng(0).normal(size=(12, 9))
    with pytest.raises(RuntimeError):
        O.svd(a, "jacobi", max_sweeps=1)
    with pytest.raises(ValueError):
        O.svd(a * np.nan)
    with pytest.raises(ValueError):
        O.svd(a, rank=0)
    with pytest.raises(TypeError):
        O.svd(a.astype(np.int32))
    _, _, _, _, status = C.svd_batched(a[None], max_sweeps=1)
    assert status[0] == 1
    _, _, _, _, status = C.svd_batched((a * np.nan)[None])
    assert status[0] == 2


def test_c_oracle_uneven_matches_batched(workloads):
    import importlib
    B = importlib.import_module("pavel-s_svd_b200.batch")
    mats = workloads.uneven_batch(24)
    flat, m, n, a_off = B.pack(mats)
    k = np.minimum(m, n)
    desc = np.zeros(len(mats), B.DESC_DTYPE)
    desc["m"], desc["n"], desc["rank"] = m, n, k
    desc["a_off"] = a_off
    desc["u_off"], _ = B._aligned_offsets(m * k)
    desc["s_off"], _ = B._aligned_offsets(k)
    desc["v_off"], _ = B._aligned_offsets(k * n)
    u, s, vh, sweeps, status = C.svd_uneven(flat.numpy(), desc)
    assert (status == 0).all()
    for i, a in enumerate(mats):
        _, s1, _, sw1, _ = C.svd_batched(a[None])
        so = desc["s_off"][i]
        np.testing.assert_array_equal(s[so:so + k[i]], s1[0])
        assert sweeps[i] == sw1[0]


def test_oracle_threads_do_not_change_results(workloads):
    x = np.stack(workloads.uneven_batch(1) * 6)
    r1 = C.svd_batched(x, threads=1)
    r4 = C.svd_batched(x, threads=4)
    for p, q in zip(r1, r4):
        np.testing.assert_array_equal(p, q)


def test_eigh_oracle_matches_reference(golden_eigh):
    """The NumPy restatement of jacobi_eigh (primitives.py:370-427) against
    the reference's own w, V and sweeps: same arithmetic dtype, so the sweep
    counts agree and w to rounding; V column by column up to sign."""
    for name, g in golden_eigh.items():
        h = g["h"]
        w, v, sw = O.jacobi_eigh(h)
        wr, vr = g["w"], g["v"]
        scale = float(np.abs(wr).max())
        tol = 50 * np.finfo(h.dtype).eps
        assert float(np.abs(w - wr).max()) <= tol * scale, name
        assert abs(int(sw) - int(g["sweeps"])) <= 1, name
        for b in range(h.shape[0]):
            for j in range(h.shape[-1]):
                gap = min([abs(wr[b, j] - wr[b, i]) for i in range(h.shape[-1]) if i != j] or [np.inf])
                if gap <= 1e-3 * scale:
                    continue
                x, y = v[b][:, j], vr[b][:, j]
                ph = np.vdot(x, y)                        # a unit phase (a sign for real input)
                ph = ph / abs(ph) if abs(ph) > 0 else 1.0
                assert np.abs(x * ph - y).max() <= 1e3 * np.finfo(h.dtype).eps, name
        # and against FP64 truth
        truth = g["truth"]
        assert float(np.abs(w - truth).max()) <= 10 * np.finfo(h.dtype).eps * scale * h.shape[-1], name


def test_eigh_oracle_raises_like_reference():
    h = np.random.default_rng(3).standard_normal((1, 9, 9))
    h = h + h.transpose(0, 2, 1)
    with pytest.raises(RuntimeError, match="did not converge in 1 sweeps"):
        O.jacobi_eigh(h, max_sweeps=1)


def test_qr_oracle_matches_reference():
    """The NumPy restatement of primitives.qr (primitives.py:41-89) against
    the reference's own Q and R: the same reflectors in the same dtype agree
    to rounding.  Where a rank-deficient input leaves columns of Q to
    rounding noise, those are checked by Q R = A and Q^T Q = I only."""
    for name, g in golden_qr().items():
        a, qr_, rr = g["a"], g["q"], g["r"]
        q, r = O.qr(a)
        k = QR_DETERMINED.get(name, a.shape[-1])
        tol = 50 * np.finfo(a.dtype).eps * max(1.0, float(np.abs(a).max()))
        assert float(np.abs(q[..., :k] - qr_[..., :k]).max()) <= tol, name
        assert float(np.abs(r[..., :k, :] - rr[..., :k, :]).max()) <= tol * a.shape[-2], name
        assert float(np.abs(q @ r - a).max()) <= tol * a.shape[-2], name
        eye = np.eye(a.shape[-1])
        assert float(np.abs(np.conj(np.swapaxes(q, -1, -2)) @ q - eye).max()) <= tol * a.shape[-2], name
        assert np.array_equal(r, np.triu(r)), name


def test_qr_methods_oracle_matches_reference():
    """svd() through 'qr', 'tsqr', the projected solvers and 'block_jacobi'
    (solvers.py:30-68, 71-96, 185-220, 245-248), restated in NumPy, against
    the reference's U, s, Vh (and block sweeps) on the same inputs and start
    bases."""
    for name, g in golden_methods().items():
        if g["alg"] == "gram_jacobi":      # restated through jacobi_eigh (test_eigh_oracle_matches_reference)
            continue
        kw = dict(g["kw"])
        if "initial_basis" in g:
            kw["initial_basis"] = g["initial_basis"]
        u, s, vh, info = O.svd(g["a"], g["alg"], return_info=True, **kw)
        dt = g["a"].dtype
        if "block_sweeps" in g:
            assert info["block_sweeps"] == g["block_sweeps"], name
        _cmp_sigma(s, g["s"], dt)
        cmp = _cmp_vectors_phase if np.iscomplexobj(g["a"]) else _cmp_vectors
        cmp(u, g["u"], g["s"], dt, -1)
        cmp(vh, g["vh"], g["s"], dt, -2)
        # as accurate against FP64 truth as the reference (the projected
        # solvers are approximations: their own error is the bar)
        k = s.shape[-1]
        err = float(np.abs(s - g["truth"][..., :k]).max() / g["truth"].max())
        err_ref = float(np.abs(g["s"] - g["truth"][..., :k]).max() / g["truth"].max())
        assert err <= max(2 * err_ref, 10 * sigma_tol(dt)), name


def _cmp_vectors_phase(u, ref, s, dtype, axis):
    """Complex columns (axis=-1) or rows (axis=-2) agree up to a unit phase
    where the singular value is simple (gap > 1e-3 relative)."""
    ref = np.asarray(ref, np.complex128).reshape(-1, *np.shape(ref)[-2:])
    u = np.asarray(u, np.complex128).reshape(ref.shape)
    s = np.asarray(s, np.float64).reshape(ref.shape[0], -1)
    tol = 1e-3 if np.dtype(dtype) == np.complex64 else 1e-8
    worst = 0.0
    for b in range(u.shape[0]):
        sb = s[b]
        ncols = ref.shape[-1] if axis == -1 else ref.shape[-2]
        for j in range(min(len(sb), ncols)):
            gap = min([abs(sb[j] - sb[i]) for i in range(len(sb)) if i != j] or [np.inf])
            if sb[j] == 0 or gap <= 1e-3 * sb[0]:
                continue
            x = u[b][:, j] if axis == -1 else u[b][j, :]
            y = ref[b][:, j] if axis == -1 else ref[b][j, :]
            ph = np.vdot(x, y)
            ph = ph / abs(ph) if abs(ph) > 0 else 1.0
            worst = max(worst, float(np.abs(x * ph - y).max()))
    assert worst <= tol, worst
    return worst


def test_complex_oracle_matches_reference():
    """The NumPy restatement of jacobi_svd on complex inputs against the
    reference's U, s, Vh and sweep counts (same arithmetic and order)."""
    for name, g in golden_complex().items():
        a = g["a"]
        u, s, vh, info = O.svd(a, "jacobi", return_info=True, **g["kw"])
        real = np.float32 if a.dtype == np.complex64 else np.float64
        _cmp_sigma(s, g["s"], real)
        assert abs(info["jacobi_sweeps"] - g["sweeps"]) <= 1, name
        if s.ndim and np.asarray(g["s"]).max() > 0:
            _cmp_vectors_phase(u, g["u"], g["s"], a.dtype, -1)
            _cmp_vectors_phase(vh, g["vh"], g["s"], a.dtype, -2)
