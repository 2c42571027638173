"""Parity of the sm_100a path (called through the C ABI via svd()/UnevenBatch)
with the reference's outputs (golden fixtures), the C oracle and FP64 LAPACK.

Tolerances, stated once:
  * sigma agreement with the reference / oracle: 1e-5 * sigma_1 in single
    precision, 1e-12 * sigma_1 in double (`sigma_tol`);
  * mixed precision ('mixed', float32 input) against FP64 LAPACK: every
    singular value above twice the reference cut eps32*max(m,n)*sigma_1 within
    1e-5 RELATIVE (the accuracy bound of the mixed path);
  * the reference's own test contract (tests/test_standalone.py:33-45):
    reconstruction < tol, max|Q^T Q - I| < 5 tol, spectrum < tol with
    tol = 3e-4 (single) / 2e-10 (double).
"""
import numpy as np
import pytest
import torch

from conftest import sigma_tol
from oracle import c_oracle as C

pytestmark = pytest.mark.gpu
DEV = "cuda"


def _err(a, b):
    a = np.asarray(a, np.float64); b = np.asarray(b, np.float64)
    scale = np.abs(a).max()
    if scale == 0:
        return float(np.abs(b).max())
    return float(np.linalg.norm((a - b) / scale) / np.linalg.norm(a / scale))


def reference_check(a, u, s, vh, tol):
    """tests/test_standalone.py:33-45 of the reference, in NumPy FP64."""
    a = np.asarray(a, np.float64)
    u = np.asarray(u, np.float64); s = np.asarray(s, np.float64); vh = np.asarray(vh, np.float64)
    r = s.shape[-1]
    recon = (u[..., :r] * s[..., None, :]) @ vh[..., :r, :]
    assert _err(a, recon) < tol
    for q in (u, np.swapaxes(vh, -1, -2)):
        eye = np.eye(q.shape[-1])
        assert np.abs(np.swapaxes(q, -1, -2) @ q - eye).max() < 5 * tol
    flat = a.reshape(-1, *a.shape[-2:])
    expected = np.stack([np.linalg.svd(x, compute_uv=False) for x in flat])
    actual = s.reshape(expected.shape)
    assert np.abs(actual - expected).max() / max(expected.max(), np.finfo(float).tiny) < tol


def mixed_bound(a, s):
    """Max relative sigma error vs FP64 LAPACK over values above 2x the cut."""
    flat = np.asarray(a, np.float64).reshape(-1, *a.shape[-2:])
    s = np.asarray(s, np.float64).reshape(flat.shape[0], -1)
    worst = 0.0
    for x, si in zip(flat, s):
        sr = np.linalg.svd(x, compute_uv=False)[:len(si)]
        cut = 2 * np.finfo(np.float32).eps * max(x.shape) * sr[0]
        sel = sr > cut
        if sel.any():
            worst = max(worst, float(np.max(np.abs(si[sel] - sr[sel]) / sr[sel])))
    return worst


@pytest.mark.parametrize("ordering", ["round_robin", "block"])
def test_golden_cases_native_precision(pkg, golden, ordering):
    """Plain path (reference arithmetic: fp32 for float32, fp64 for float64)
    against the reference's own outputs; with the reference's round-robin
    order the sweep counts agree too."""
    for name, c in golden.items():
        a = c["a"]
        t = torch.from_numpy(a.copy()).to(DEV)
        saved = t.clone()
        u, s, vh, info = pkg.svd(t, "jacobi", return_info=True, precision="fp32", ordering=ordering, **c["kw"])
        assert torch.equal(t, saved), name
        s_np = s.cpu().numpy()
        top = max(float(np.abs(c["s"]).max()), np.finfo(np.float64).tiny)
        assert np.abs(s_np.astype(np.float64) - c["s"]).max() / top <= sigma_tol(a.dtype), name
        assert abs(info["jacobi_sweeps"] - c["sweeps"]) <= (1 if ordering == "round_robin" else 2), name
        if u is not None:
            tol = 3e-4 if a.dtype == np.float32 else 2e-10
            k = s.shape[-1]
            if not c["kw"].get("rank"):
                reference_check(a, u.cpu().numpy(), s_np, vh.cpu().numpy(), tol)
            assert u.shape == torch.Size(c["u"].shape if "u" in c else u.shape), name


def test_golden_cases_mixed_meet_fp64_bound(pkg, golden):
    for name, c in golden.items():
        a = c["a"]
        if a.dtype != np.float32:
            continue
        t = torch.from_numpy(a.copy()).to(DEV)
        u, s, vh = pkg.svd(t, "jacobi", **c["kw"])
        assert mixed_bound(a, s.cpu().numpy()) <= 1e-5, name
        top = max(float(np.abs(c["s"]).max()), np.finfo(np.float64).tiny)
        # The reference's own fp32 error bounds the distance to it.
        assert np.abs(s.cpu().numpy().astype(np.float64) - c["s"]).max() / top <= 1e-4, name


def test_reference_contract_edge_cases(pkg):
    """Zero, identity, rank-deficient, extreme scales, singletons, full bases,
    values only, multi-dimensional batches (tests/test_standalone.py:56-77, 187-192)."""
    rng = np.random.default_rng(3)
    mats = [np.zeros((9, 5)), np.eye(7), np.diag([0., 2., 0., 3., 1.]), rng.normal(size=(11, 5)) * 1e-150,
            rng.normal(size=(11, 5)) * 1e150, rng.normal(size=(15, 3)) @ rng.normal(size=(3, 7))]
    for a in mats:
        u, s, vh = pkg.svd(torch.from_numpy(a).to(DEV))
        reference_check(a, u.cpu().numpy(), s.cpu().numpy(), vh.cpu().numpy(), 2e-9)
    for shape in ((1, 1), (8, 1), (1, 8), (10, 4), (4, 10), (5, 5), (7, 7)):
        a = rng.normal(size=shape)
        for dt, tol in ((np.float64, 2e-10), (np.float32, 3e-4)):
            t = torch.from_numpy(a.astype(dt)).to(DEV)
            u, s, vh = pkg.svd(t, full_matrices=True)
            assert u.shape == (shape[0], shape[0]) and vh.shape == (shape[1], shape[1])
            reference_check(a.astype(dt), u.cpu().numpy(), s.cpu().numpy(), vh.cpu().numpy(), tol)
            none, ss, none2 = pkg.svd(t, values_only=True)
            assert none is None and none2 is None
            assert float((s - ss).abs().max()) <= (1e-12 if dt == np.float64 else 1e-6)
    a = rng.normal(size=(2, 3, 9, 5))
    u, s, vh = pkg.svd(torch.from_numpy(a).to(DEV))
    assert s.shape == (2, 3, 5)
    assert _err(a, (u.cpu().numpy() * s.cpu().numpy()[..., None, :]) @ vh.cpu().numpy()) < 1e-10


def test_rank_truncation_and_wide(pkg):
    rng = np.random.default_rng(4)
    for shape in ((13, 7), (7, 13), (40, 25), (25, 40)):
        a = rng.normal(size=shape)
        full = pkg.svd(torch.from_numpy(a).to(DEV))
        u, s, vh = pkg.svd(torch.from_numpy(a).to(DEV), rank=4)
        assert u.shape == (shape[0], 4) and s.shape == (4,) and vh.shape == (4, shape[1])
        torch.testing.assert_close(s, full[1][:4], rtol=0, atol=0)


def test_errors_like_reference(pkg):
    a = torch.from_numpy(np.random.default_rng(0).normal(size=(12, 9))).to(DEV)
    with pytest.raises(RuntimeError):
        pkg.svd(a, "jacobi", max_sweeps=1)
    with pytest.raises(ValueError):
        pkg.svd(a * float("nan"))
    b = a.clone()
    b[3, 4] = float("inf")
    with pytest.raises(ValueError):
        pkg.svd(b.float())
    with pytest.raises(TypeError):
        pkg.svd(a.to(torch.int32))
    # the context stays usable after every error
    u, s, vh = pkg.svd(a)
    assert torch.isfinite(s).all()


def test_plain_single_workload(pkg, golden, workloads):
    """256x128 f32, s_i = 10^(-4i/127), tol 1e-6, <= 30 sweeps."""
    c = golden["plain_single_256x128"]
    a = workloads.plain_single()
    np.testing.assert_array_equal(a, c["a"])
    t = torch.from_numpy(a).to(DEV)
    u, s, vh, info = pkg.svd(t, tol=1e-6, max_sweeps=30, precision="fp32", return_info=True)
    assert abs(info["jacobi_sweeps"] - c["sweeps"]) <= 2
    top = float(c["s"].max())
    assert np.abs(s.cpu().numpy() - c["s"]).max() / top <= 1e-5
    u, s, vh, info = pkg.svd(t, tol=1e-6, max_sweeps=30, return_info=True)
    assert mixed_bound(a, s.cpu().numpy()) <= 1e-5
    reference_check(a, u.cpu().numpy(), s.cpu().numpy(), vh.cpu().numpy(), 3e-4)


def _plan(pkg, mats, precision):
    from importlib import import_module
    B = import_module("pavel-s_svd_b200.batch")
    flat, m, n, a_off = B.pack(mats, DEV)
    plan = B.UnevenBatch(m, n, DEV, a_off=a_off, precision=precision)
    return B, flat, m, n, plan


@pytest.mark.parametrize("precision", ["fp32", "mixed"])
def test_orderings_and_precisions_agree(pkg, workloads, precision):
    """Block order vs the reference's round-robin order on the same inputs."""
    rng = np.random.default_rng(11)
    for shape in ((64, 64), (128, 64), (37, 29), (29, 37), (200, 40), (9, 1), (256, 128)):
        a = torch.from_numpy(rng.normal(size=(3, *shape)).astype(np.float32)).to(DEV)
        _, s1, _ = pkg.svd(a, precision=precision, ordering="block")
        _, s2, _ = pkg.svd(a, precision=precision, ordering="round_robin")
        assert float((s1 - s2).abs().max() / s2.max()) <= 1e-5, shape


def test_uneven_batch_matches_oracle(pkg, workloads):
    mats = workloads.uneven_batch(512)
    B, flat, m, n, plan = _plan(pkg, mats, "fp32")
    plan.launch(flat)
    sweeps = plan.check()
    desc = np.frombuffer(plan.desc.cpu().numpy().tobytes(), B.DESC_DTYPE)
    u_o, s_o, vh_o, sw_o, st_o = C.svd_uneven(flat.cpu().numpy(), desc)
    assert (st_o == 0).all()
    S = plan.S.cpu().numpy()
    for i in range(len(mats)):
        k = min(m[i], n[i])
        so = desc["s_off"][i]
        ref = s_o[so:so + k].astype(np.float64)
        assert np.abs(S[so:so + k] - ref).max() / ref[0] <= sigma_tol(np.float32), i
    # block order vs the oracle's round-robin order: same work, sweeps within 2
    assert np.abs(sweeps - sw_o).max() <= 2 and abs(float(np.mean(sweeps - sw_o))) < 0.5
    for i in range(0, len(mats), 37):
        u, s, vh = plan.result(i)
        reference_check(mats[i], u.cpu().numpy(), s.cpu().numpy(), vh.cpu().numpy(), 3e-4)


def test_uneven_batch_mixed_meets_bound_and_graph_replay(pkg, workloads):
    mats = workloads.uneven_batch(1024)
    B, flat, m, n, plan = _plan(pkg, mats, "mixed")
    plan.launch(flat)
    plan.check()
    S1 = plan.S.clone()
    worst = 0.0
    for i in range(len(mats)):
        _, s, _ = plan.result(i)
        worst = max(worst, mixed_bound(mats[i], s.cpu().numpy()))
    assert worst <= 1e-5, worst
    g = plan.capture(flat)
    plan.S.zero_()
    g.replay()
    torch.cuda.synchronize()
    plan.check()
    assert torch.equal(plan.S, S1)
    del g


def test_uneven_batch_full_workload(pkg, workloads):
    """All 8192 matrices of the uneven-batch benchmark workload (n ~ U[8, 64],
    m ~ U[n, 2n], seed 1): the mixed solve meets sigma-rel-err <= 1e-5 against
    FP64 LAPACK on every matrix, with reconstruction <= 1e-6; the fp32 solve
    (the reference's arithmetic) agrees with the C oracle of the reference's
    FP32 Jacobi within sigma_tol on every matrix."""
    mats = workloads.uneven_batch(8192)
    B, flat, m, n, plan = _plan(pkg, mats, "mixed")
    plan.launch(flat)
    plan.check()
    S, U, Vh = plan.S.cpu().numpy(), plan.U.cpu().numpy(), plan.Vh.cpu().numpy()
    worst, worst_rec = 0.0, 0.0
    for i in range(len(mats)):
        k = min(m[i], n[i])
        s = S[plan.s_off[i]:plan.s_off[i] + k]
        worst = max(worst, mixed_bound(mats[i], s))
        u = U[plan.u_off[i]:plan.u_off[i] + m[i] * k].reshape(m[i], k).astype(np.float64)
        vh = Vh[plan.v_off[i]:plan.v_off[i] + k * n[i]].reshape(k, n[i]).astype(np.float64)
        a = mats[i].astype(np.float64)
        worst_rec = max(worst_rec, float(np.linalg.norm(a - (u * s) @ vh) / np.linalg.norm(a)))
    assert worst <= 1e-5, worst
    assert worst_rec <= 1e-6, worst_rec
    B, flat, m, n, plan32 = _plan(pkg, mats, "fp32")
    plan32.launch(flat)
    plan32.check()
    desc = np.frombuffer(plan32.desc.cpu().numpy().tobytes(), B.DESC_DTYPE)
    _, s_o, _, _, st_o = C.svd_uneven(flat.cpu().numpy(), desc)
    assert (st_o == 0).all()
    S32 = plan32.S.cpu().numpy()
    for i in range(len(mats)):
        k = min(m[i], n[i])
        so = desc["s_off"][i]
        ref = s_o[so:so + k].astype(np.float64)
        assert np.abs(S32[so:so + k] - ref).max() / ref[0] <= sigma_tol(np.float32), i


def test_svd_uneven_list_api(pkg, workloads):
    """The list API, with matrices beyond the register kernels mixed in (a
    300 x 20, a 20 x 300, a 100 x 100): those go through svd() one by one,
    the rest in one launch; every result in input order."""
    mats = list(workloads.uneven_batch(16))
    rng = np.random.default_rng(3)
    mats[3:3] = [rng.standard_normal((300, 20)).astype(np.float32), rng.standard_normal((20, 300)).astype(np.float32)]
    mats.append(rng.standard_normal((100, 100)).astype(np.float32))
    for precision in ("fp32", "mixed"):
        res = pkg.svd_uneven([torch.from_numpy(a).to(DEV) for a in mats], precision=precision)
        assert len(res) == len(mats)
        for a, (u, s, vh) in zip(mats, res):
            u2, s2, vh2 = pkg.svd(torch.from_numpy(a).to(DEV), precision=precision)
            assert u.shape == u2.shape and vh.shape == vh2.shape
            # different launch shapes sum in a different order: agree to fp32 accuracy
            torch.testing.assert_close(s, s2, rtol=0, atol=1e-5 * float(s2[0]))


@pytest.mark.parametrize("precision", ["mixed", "fp32"])
def test_uneven_size_classes_each_solved_once(pkg, precision):
    """An uneven batch wider than 32 columns runs in two launches per phase
    (widths <= 32 in CTAs of half the size).  Interleaved narrow and wide
    matrices, in a shuffled order: every matrix is solved (status OK, at
    least one sweep) and agrees with its own single-matrix solve, which runs
    in one launch, with U and Vh meeting the reference's test contract."""
    import importlib
    B = importlib.import_module("pavel-s_svd_b200.batch")
    rng = np.random.default_rng(21)
    shapes = [(40, 33), (20, 9), (64, 64), (33, 32), (96, 40), (31, 31), (128, 64), (12, 30), (70, 35), (1, 1)]
    mats = [rng.normal(size=s).astype(np.float32) for s in shapes]
    m = np.array([a.shape[0] for a in mats]); n = np.array([a.shape[1] for a in mats])
    plan = B.UnevenBatch(m, n, DEV, precision=precision, order="input")
    assert plan.kernels_per_solve == (4 if precision == "mixed" else 2)
    flat = torch.zeros(int(plan.a_off[-1] + m[-1] * n[-1] + 4), dtype=torch.float32, device=DEV)
    for a, o in zip(mats, plan.a_off):
        flat[int(o):int(o) + a.size] = torch.from_numpy(a.reshape(-1)).to(DEV)
    plan.launch(flat)
    sweeps = plan.check()
    assert (sweeps >= 1).all()
    for i, a in enumerate(mats):
        u, s, vh = plan.result(i)
        u2, s2, vh2 = pkg.svd(torch.from_numpy(a).to(DEV), precision=precision)
        torch.testing.assert_close(s, s2, rtol=0, atol=1e-6 * float(s2[0]))
        reference_check(a, u.cpu().numpy(), s.cpu().numpy(), vh.cpu().numpy(), 3e-4)


def test_sharded_uneven_equals_single_plan(pkg, workloads):
    """batch.ShardedUneven splits one uneven batch by cost into one share per
    device (shard_by_cost) and solves every share with no exchange.  With
    two shares on the one device of this run, every matrix's singular values
    and sweeps equal those of the single-plan solve (the same kernels per
    matrix), and every matrix is solved exactly once."""
    from importlib import import_module
    B = import_module("pavel-s_svd_b200.batch")
    mats = workloads.uneven_batch(512)
    B_, flat, m, n, plan = _plan(pkg, mats, "mixed")
    plan.launch(flat)
    sweeps = plan.check()
    sh = B.ShardedUneven(m, n, [DEV, DEV], precision="mixed")
    assert sorted(np.concatenate(sh.shards).tolist()) == list(range(len(mats)))
    sh.launch(sh.pack(mats))
    sw2 = sh.check()
    assert np.array_equal(sw2, sweeps)
    for i in range(len(mats)):
        _, s1, _ = plan.result(i)
        _, s2, _ = sh.result(i)
        assert torch.equal(s1, s2), i
