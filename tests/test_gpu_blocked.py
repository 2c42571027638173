"""Blocked one-sided Jacobi on the tensor cores (BlockJacobi) against FP64
LAPACK on the same float32 input.

Stated bounds for this mixed-precision path (3xBF16 sweeps, FP64 block
eigen-solves, ~FP32-accurate 6xBF16 finish): |sigma_i - sigma_i(FP64)| <=
5e-6 sigma_1 (spectrum_error_over_sigma1), relative error <= 1e-5 for
sigma_i >= 0.1 sigma_1, reconstruction ||A - U S V^T|| / ||A|| <= 2e-5,
max |V^T V - I| <= 2e-5, max |U^T U - I| <= 2e-5 (U = A V / sigma carries
eps32 * cond into the small columns' directions; the finish re-orthogonalises
the kept columns against the larger ones)."""
import importlib

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def BJ():
    return importlib.import_module("pavel-s_svd_b200.blocked")


def check(a, U, S, Vh):
    a64 = a.astype(np.float64)
    sr = np.linalg.svd(a64, compute_uv=False)
    s = S.cpu().numpy().astype(np.float64)
    err1 = np.abs(s - sr).max() / sr[0]
    big = sr >= 0.1 * sr[0]
    relbig = float(np.max(np.abs(s[big] - sr[big]) / sr[big]))
    u, vh = U.cpu().numpy().astype(np.float64), Vh.cpu().numpy().astype(np.float64)
    keep = s > 0
    rec = np.linalg.norm(a64 - (u[:, keep] * s[keep]) @ vh[keep]) / np.linalg.norm(a64)
    ou = np.abs(u[:, keep].T @ u[:, keep] - np.eye(keep.sum())).max()
    ov = np.abs(vh @ vh.T - np.eye(vh.shape[0])).max()
    return err1, relbig, rec, ou, ov


@pytest.mark.parametrize("m,n,b,cond", [(512, 256, 32, 1e3), (1000, 200, 32, 1e2), (768, 384, 64, 1e4)])
def test_blocked_matches_lapack(BJ, m, n, b, cond):
    rng = np.random.default_rng(m + n)
    u, _ = np.linalg.qr(rng.standard_normal((m, n)))
    v, _ = np.linalg.qr(rng.standard_normal((n, n)))
    s = np.geomspace(1, 1 / cond, n)
    a = ((u * s) @ v.T).astype(np.float32)
    plan = BJ.BlockJacobi(m, n, b)
    U, S, Vh, info = plan.solve(torch.from_numpy(a).cuda())
    err1, relbig, rec, ou, ov = check(a, U, S, Vh)
    print(m, n, b, info["block_sweeps"], ["%.1e/%d" % x for x in info["off_per_sweep"]], err1, relbig, rec, ou, ov)
    assert err1 <= 5e-6 and relbig <= 1e-5 and rec <= 2e-5 and ou <= 2e-5 and ov <= 2e-5


@pytest.mark.parametrize("M,N,K,lda", [(300, 520, 1000, 1000), (256, 384, 1004, 1012), (129, 77, 37, 37),
                                        (130, 200, 64, 66)])
def test_gemm_f64acc_against_fp64(M, N, K, lda):
    """jb_gemm_f64acc (C = A B^T, exact float products summed in FP64):
    equal to the FP64 product rounded once to float, on the float4 path
    (16-byte rows: K, lda multiples of 4, ragged K slices and tiles) and on
    the scalar path (odd lda or K).  The inputs cancel heavily, so an
    FP32-accumulated product misses this bound by orders of magnitude."""
    N_ = importlib.import_module("pavel-s_svd_b200.native")
    g = torch.Generator().manual_seed(M + N + K)
    a_full = torch.randn(M, lda, generator=g)
    b_full = torch.randn(N, lda, generator=g)
    # cancellation: columns h..2h-1 of A are minus columns 0..h-1 (scaled by
    # 1e3) plus O(1), and the same columns of B repeat columns 0..h-1, so
    # every entry of C is O(1) made from terms of size 1e3
    h = K // 2
    a_full[:, :h] *= 1e3
    a_full[:, h:2 * h] = -a_full[:, :h] + a_full[:, h:2 * h]
    b_full[:, h:2 * h] = b_full[:, :h]
    a = a_full[:, :K]
    b = b_full[:, :K]
    A = a_full.cuda()
    B = b_full.cuda()
    C = torch.empty(M, N, device="cuda")
    N_.check(N_.lib().jb_gemm_f64acc(A.data_ptr(), B.data_ptr(), C.data_ptr(), M, N, K, lda, lda, N,
                                     torch.cuda.current_stream().cuda_stream), "jb_gemm_f64acc")
    torch.cuda.synchronize()
    ref = (a.double() @ b.double().T)
    scale = a.double().abs() @ b.double().abs().T
    err = (C.cpu().double() - ref).abs()
    bound = 2.5e-7 * ref.abs() + 1e-14 * scale
    assert bool((err <= bound).all()), float((err / bound).max())
    f32 = (a @ b.T).double()                               # FP32 accumulation, for contrast
    assert float((f32 - ref).abs().max()) > 10 * float(bound.max())


def test_w_from_v_tensor_matches_fp64(BJ):
    """W^T = V^T A^T of the blocked solver's stage switch and finish: the
    six-term BF16 tensor-core product (taken when every kept column is within
    TENSOR_W_COND of sigma_1) agrees with the FP64-accumulated one to ~2^-24
    of the largest column norm in every entry, and the cond_kept measure
    picks the path as stated."""
    m, n, b = 600, 256, 32
    plan = BJ.BlockJacobi(m, n, b)
    g = torch.Generator(device="cuda").manual_seed(5)
    ap = torch.zeros(plan.mpad, plan.npad, device="cuda")
    ap[:m, :n] = torch.randn(m, n, device="cuda", generator=g)
    vt = torch.linalg.qr(torch.randn(plan.npad, plan.npad, device="cuda", generator=g, dtype=torch.float64))[0]
    vt = vt.float().contiguous()
    w64 = plan._w_from_v(vt, ap)
    wtc = plan._w_from_v(vt, ap, cond_kept=1.0)
    scale = float(ap.norm(dim=0).max())
    assert float((wtc - w64).abs().max()) <= 2e-6 * scale
    assert float((wtc - w64).abs().max()) > 0.0             # a different product was taken
    assert BJ.TENSOR_W_COND == 32.0


@pytest.mark.parametrize("n", [64, 128, 48])
def test_block_eig_f64(n):
    """jb_block_eig_f64 alone: Qt (hi + lo + lo2) orthogonal, Qt G Qt^T
    diagonal with a descending diagonal, for slot widths served by the
    register-resident odd-even kernel (64, 128) and by the shared-memory
    round-robin kernel (48)."""
    N = importlib.import_module("pavel-s_svd_b200.native")
    g = torch.Generator(device="cuda").manual_seed(n)
    P = 5
    x = torch.randn(P, n, 3 * n, device="cuda", generator=g, dtype=torch.float64)
    x = x * torch.logspace(0, -3, n, device="cuda", dtype=torch.float64)[:, None]
    G64 = x @ x.transpose(1, 2)
    G = G64.float().contiguous()
    qt = [torch.empty(P, n, n, dtype=torch.bfloat16, device="cuda") for _ in range(3)]
    off = torch.zeros(P, device="cuda")
    dmax = torch.zeros(P, device="cuda")
    sweeps = torch.zeros(P, dtype=torch.int32, device="cuda")
    st = torch.cuda.current_stream().cuda_stream
    N.check(N.lib().jb_block_eig_f64(G.data_ptr(), qt[0].data_ptr(), qt[1].data_ptr(), qt[2].data_ptr(),
                                     off.data_ptr(), dmax.data_ptr(), sweeps.data_ptr(), P, n, 12, 1e-12, None, st),
            "jb_block_eig_f64")
    torch.cuda.synchronize()
    Q = (qt[0].double() + qt[1].double() + qt[2].double())
    eye = torch.eye(n, device="cuda", dtype=torch.float64)
    # Q accumulates its rotations in FP32: ~eps32 * sqrt(rotations per column)
    assert float((Q @ Q.transpose(1, 2) - eye).abs().max()) <= 1e-5
    D = Q @ G.double() @ Q.transpose(1, 2)
    diag = D.diagonal(dim1=1, dim2=2)
    offd = (D - torch.diag_embed(diag)).abs() / (diag.abs().sqrt()[:, :, None] * diag.abs().sqrt()[:, None, :])
    assert float(offd.max()) <= 1e-5
    assert bool((diag[:, :-1] >= diag[:, 1:] * (1 - 1e-6)).all())
    ref = torch.linalg.eigvalsh(G.double()).flip(-1)
    # eigenvalues to ~2x the FP32 non-orthogonality of Q, relative to the largest
    assert float(((diag - ref).abs() / ref.abs().max(dim=1, keepdim=True).values).max()) <= 1e-5
    assert float(dmax.max()) > 0 and int(sweeps.min()) >= 2
    assert 0.0 < float(off.min())


@pytest.mark.parametrize("n", [64, 128])
def test_block_eig_variants_agree(n):
    """The register-resident odd-even kernel at 4, 8 and 16 columns per warp
    and the shared-memory round-robin kernel (jb_block_eig_f64_ex variants 4,
    8, 16 and 1) diagonalise the same graded Grams: the register layouts run
    the same rotations (each build may contract multiply-adds differently,
    so Q^T agrees to FP32 rounding); the round robin (a different pair order)
    gives the same eigenvectors up to sign within the FP32 accumulation of Q."""
    N = importlib.import_module("pavel-s_svd_b200.native")
    g = torch.Generator(device="cuda").manual_seed(n)
    P = 8
    x = torch.randn(P, n, 2 * n, device="cuda", generator=g, dtype=torch.float64)
    x = x * torch.logspace(0, -4, n, device="cuda", dtype=torch.float64)[:, None]
    G = (x @ x.transpose(1, 2)).float().contiguous()
    st = torch.cuda.current_stream().cuda_stream
    outs = []
    for variant in (8, 1, 4, 16):
        qt = [torch.empty(P, n, n, dtype=torch.bfloat16, device="cuda") for _ in range(3)]
        off = torch.zeros(P, device="cuda")
        dmax = torch.zeros(P, device="cuda")
        sw = torch.zeros(P, dtype=torch.int32, device="cuda")
        N.check(N.lib().jb_block_eig_f64_ex(G.data_ptr(), qt[0].data_ptr(), qt[1].data_ptr(), qt[2].data_ptr(),
                                            off.data_ptr(), dmax.data_ptr(), sw.data_ptr(), P, n, 12, 1e-12, None,
                                            variant, st), "jb_block_eig_f64_ex")
        torch.cuda.synchronize()
        outs.append(sum(q.double() for q in qt))
    dots = (outs[0] * outs[1]).sum(-1).abs()                  # |<row of Q1^T, row of Q2^T>|
    assert float((dots - 1).abs().max()) <= 1e-5
    for other in outs[2:]:
        torch.testing.assert_close(other, outs[0], rtol=0, atol=2e-6)


@pytest.mark.parametrize("m,n,b", [(1024, 512, 32), (1536, 768, 64)])
def test_dataflow_schedule_matches_batched(BJ, m, n, b):
    """The per-slot dataflow schedule (per-slot streams, only the true
    dependencies, replayed as a CUDA graph) runs the batched schedule's
    kernels per slot: the same block sweeps and singular values to the
    rounding of split-K accumulation order, both within the LAPACK bound."""
    rng = np.random.default_rng(m)
    u, _ = np.linalg.qr(rng.standard_normal((m, n)))
    v, _ = np.linalg.qr(rng.standard_normal((n, n)))
    a = ((u * np.geomspace(1, 1e-3, n)) @ v.T).astype(np.float32)
    x = torch.from_numpy(a).cuda()
    out = {}
    for sched in ("batched", "dataflow"):
        plan = BJ.BlockJacobi(m, n, b)
        plan.schedule = sched
        for _ in range(2):                         # eager sweeps, then graph replays
            U, S, Vh, info = plan.solve(x)
        out[sched] = (S.double().cpu().numpy(), info["block_sweeps"])
        err1, relbig, rec, ou, ov = check(a, U, S, Vh)
        assert err1 <= 5e-6 and relbig <= 1e-5 and rec <= 2e-5 and ov <= 2e-5, (sched, err1, relbig, rec, ov)
    sb, nb_ = out["batched"]
    sd, nd = out["dataflow"]
    assert abs(nb_ - nd) <= 1
    assert float(np.abs(sb - sd).max() / sb[0]) <= 2e-6


@pytest.mark.parametrize("n", [64, 128])
@pytest.mark.parametrize("layout,fp32", [(4, False), (8, False), (16, False), (8, True)])
@pytest.mark.parametrize("sweeps", [1, 2])
def test_block_eig_deferred_q_matches(n, layout, fp32, sweeps):
    """JB_EIG_DEFER_Q: the register eigen-solve records its rotations and
    q_apply_kernel forms Q^T from them.  The same Q^T as the eigen-solve that
    accumulates Q itself (the same FP32 updates; to rounding), the same off,
    dmax and sweep counts."""
    N = importlib.import_module("pavel-s_svd_b200.native")
    lib = N.lib()
    g = torch.Generator(device="cuda").manual_seed(3 * n + layout)
    P = 6
    x = torch.randn(P, n, 2 * n, device="cuda", generator=g, dtype=torch.float64)
    x = x * torch.logspace(0, -3, n, device="cuda", dtype=torch.float64)[:, None]
    G = (x @ x.transpose(1, 2)).float().contiguous()
    st = torch.cuda.current_stream().cuda_stream
    ws = torch.empty(int(lib.jb_block_eig_workspace_bytes(P, n, sweeps)), dtype=torch.uint8, device="cuda")
    outs = []
    for dq in (False, True):
        variant = layout | (N.EIG_FP32 if fp32 else 0) | (N.EIG_DEFER_Q if dq else 0)
        qt = [torch.full((P, n, n), 3.0, dtype=torch.bfloat16, device="cuda") for _ in range(3)]
        off = torch.zeros(P, device="cuda")
        dmax = torch.zeros(P, device="cuda")
        sw = torch.zeros(P, dtype=torch.int32, device="cuda")
        N.check(lib.jb_block_eig_ws(G.data_ptr(), qt[0].data_ptr(), qt[1].data_ptr(), qt[2].data_ptr(),
                                    off.data_ptr(), dmax.data_ptr(), sw.data_ptr(), P, n, sweeps, 1e-9, None, variant,
                                    ws.data_ptr(), ws.numel(), st), "jb_block_eig_ws")
        torch.cuda.synchronize()
        outs.append((sum(q.double() for q in qt), off, dmax, sw))
    (qa, offa, da, swa), (qb, offb, db, swb) = outs
    torch.testing.assert_close(qb, qa, rtol=0, atol=2e-6)
    assert torch.equal(offa, offb) and torch.equal(da, db) and torch.equal(swa, swb)
    with pytest.raises(RuntimeError):                       # the deferred form needs its workspace
        N.check(lib.jb_block_eig_ws(G.data_ptr(), qt[0].data_ptr(), qt[1].data_ptr(), None, off.data_ptr(),
                                    dmax.data_ptr(), sw.data_ptr(), P, n, sweeps, 1e-9, None,
                                    layout | N.EIG_DEFER_Q, None, 0, st), "jb_block_eig_ws")


def test_block_jacobi_drop_in():
    """svd(a, 'block_jacobi', ...) through the drop-in API: tall and wide
    inputs, the reference's defaults (block_size 4 -> width 32 here), the
    one-block case routed to the plain Jacobi, values_only and rank."""
    pkg = importlib.import_module("pavel-s_svd_b200")
    rng = np.random.default_rng(11)
    for m, n, bs in ((512, 256, 32), (256, 384, 4)):
        a = rng.standard_normal((m, n)).astype(np.float32)
        x = torch.from_numpy(a).cuda()
        u, s, vh, info = pkg.svd(x, 'block_jacobi', block_size=bs, return_info=True)
        assert info['block_size_used'] == 32 and info['block_sweeps'] >= 2
        assert torch.equal(x, torch.from_numpy(a).cuda())          # input untouched
        sr = np.linalg.svd(a.astype(np.float64), compute_uv=False)
        k = min(m, n)
        assert u.shape == (m, k) and s.shape == (k,) and vh.shape == (k, n)
        assert float(np.abs(s.cpu().numpy() - sr).max() / sr[0]) <= 5e-6
        rec = (u.double() * s.double()) @ vh.double()
        assert float((rec - x.double()).norm() / x.double().norm()) <= 2e-5
    u, s, vh = pkg.svd(x, 'block_jacobi', block_size=32, values_only=True)
    assert u is None and vh is None and s.shape == (256,)
    u, s, vh = pkg.svd(x, 'block_jacobi', block_size=32, rank=10)
    assert u.shape == (256, 10) and vh.shape == (10, 384)
    small = torch.randn(3, 40, 24, device="cuda")
    u, s, vh, info = pkg.svd(small, 'block_jacobi', block_size=32, return_info=True)
    assert info['algorithm'] == 'jacobi' and s.shape == (3, 24)
    with pytest.raises(ValueError):
        pkg.svd(x, 'block_jacobi', block_size=0)
    # full bases on the tensor-core path: the reference's null completion
    u, s, vh = pkg.svd(x, 'block_jacobi', block_size=32, full_matrices=True)
    assert u.shape == (256, 256) and vh.shape == (384, 384)
    for q in (u.double(), vh.double()):
        assert float((q.mT @ q - torch.eye(q.shape[0], dtype=torch.float64, device="cuda")).abs().max()) <= 1e-4


def _lapack_check(a, u, s, vh, tol):
    a64 = a.astype(np.complex128 if np.iscomplexobj(a) else np.float64).reshape(-1, *a.shape[-2:])
    truth = np.stack([np.linalg.svd(x, compute_uv=False) for x in a64])
    k = min(a.shape[-2:])
    assert float(np.abs(s.reshape(-1, s.shape[-1])[:, :k] - truth).max() / truth.max()) <= tol
    u = u.reshape(-1, *u.shape[-2:]).astype(a64.dtype)
    vh = vh.reshape(-1, *vh.shape[-2:]).astype(a64.dtype)
    rec = (u[..., :k] * s.reshape(-1, s.shape[-1])[:, None, :k]) @ vh[..., :k, :]
    assert float(np.abs(rec - a64).max() / np.abs(a64).max()) <= 10 * tol
    for q, eye in ((np.conj(np.swapaxes(u, -1, -2)) @ u, u.shape[-1]), (vh @ np.conj(np.swapaxes(vh, -1, -2)),
                                                                        vh.shape[-2])):
        assert float(np.abs(q - np.eye(eye)).max()) <= 10 * tol


def test_block_jacobi_rounds_golden(pkg):
    """The rounds path against the reference's own block_jacobi runs: block
    sweeps within one of the reference's (the pair solves are this library's
    Jacobi, whose rounding differs), sigma and vectors as in the reference."""
    from conftest import golden_methods, sigma_tol
    from test_oracle import _cmp_sigma, _cmp_vectors, _cmp_vectors_phase
    seen = 0
    for name, g in golden_methods().items():
        if g["alg"] != "block_jacobi":
            continue
        seen += 1
        a = g["a"]
        u, s, vh, info = pkg.svd(torch.from_numpy(a).cuda(), "block_jacobi", return_info=True, **g["kw"])
        assert abs(info["block_sweeps"] - g["block_sweeps"]) <= 1, name
        assert info["jacobi_sweeps"] >= 1 and "block_size_used" not in info
        u, s, vh = u.resolve_conj().cpu().numpy(), s.cpu().numpy(), vh.resolve_conj().cpu().numpy()
        _cmp_sigma(s, g["s"], a.dtype)
        cmp = _cmp_vectors_phase if np.iscomplexobj(a) else _cmp_vectors
        cmp(u, g["u"], g["s"], a.dtype, -1)
        cmp(vh, g["vh"], g["s"], a.dtype, -2)
        err = float(np.abs(s - g["truth"]).max() / g["truth"].max())
        assert err <= max(2 * float(np.abs(g["s"] - g["truth"]).max() / g["truth"].max()), 10 * sigma_tol(a.dtype))
    assert seen >= 6


@pytest.mark.parametrize("shape,dtype,bs", [((3, 200, 120), np.float64, 16), ((2, 90, 140), np.complex128, 8),
                                            ((4, 64, 40), np.complex64, 5), ((8, 48, 33), np.float32, 4),
                                            ((6, 200, 100), np.float32, 16)])
def test_block_jacobi_rounds_against_lapack(pkg, shape, dtype, bs):
    """Larger batches through the rounds path (float64, complex, float32 below
    the tensor-core size), tall and wide, ragged groups."""
    rng = np.random.default_rng(shape[-1])
    a = rng.standard_normal(shape)
    if np.issubdtype(dtype, np.complexfloating):
        a = a + 1j * rng.standard_normal(shape)
    a = a.astype(dtype)
    u, s, vh, info = pkg.svd(torch.from_numpy(a).cuda(), "block_jacobi", block_size=bs, return_info=True)
    assert info["block_sweeps"] >= 2 and "block_size_used" not in info     # the rounds engine
    tol = 1e-12 if dtype in (np.float64, np.complex128) else 2e-5
    _lapack_check(a, u.resolve_conj().cpu().numpy(), s.cpu().numpy(), vh.resolve_conj().cpu().numpy(), tol)


def test_block_jacobi_rounds_contract(pkg):
    """Full bases (wide, complex), values only, a truncated rank, the
    reference's non-convergence error."""
    rng = np.random.default_rng(5)
    a = (rng.standard_normal((2, 12, 30)) + 1j * rng.standard_normal((2, 12, 30))).astype(np.complex128)
    x = torch.from_numpy(a).cuda()
    u, s, vh = pkg.svd(x, "block_jacobi", full_matrices=True, block_size=4)
    assert u.shape == (2, 12, 12) and vh.shape == (2, 30, 30)
    _lapack_check(a, u.cpu().numpy(), s.cpu().numpy(), vh.cpu().numpy(), 1e-12)
    u, s2, vh = pkg.svd(x, "block_jacobi", values_only=True, block_size=4)
    assert u is None and vh is None and torch.allclose(s2, s, rtol=0, atol=1e-12)
    u, s3, vh = pkg.svd(x.real.contiguous(), "block_jacobi", rank=5, block_size=4)
    assert u.shape == (2, 12, 5) and s3.shape == (2, 5) and vh.shape == (2, 5, 30)
    with pytest.raises(RuntimeError, match="block Jacobi did not converge"):
        pkg.svd(x.real.contiguous(), "block_jacobi", block_size=1, max_sweeps=2)
    for dt, shape in ((torch.float64, (0, 12, 30)), (torch.float32, (2, 0, 80, 70))):   # empty batches
        u, s, vh = pkg.svd(torch.zeros(shape, dtype=dt, device="cuda"), "block_jacobi", block_size=4)
        k = min(shape[-2:])
        assert u.shape == (*shape[:-2], shape[-2], k) and s.shape == (*shape[:-2], k)
        assert vh.shape == (*shape[:-2], k, shape[-1])


def _replay_completion(sub, keep, pivots, delta=1e-6):
    """The reference's completion of the columns keep == False
    (primitives.py:437-454: largest leftover leverage picks the coordinate,
    two projections, normalise), in FP64, with each column's pivot row taken
    from `pivots` and checked to be the largest leverage up to `delta`.  Two
    rows whose leverages differ by less than the FP32 rounding of the kept
    columns are a tie that the reference's own arithmetic breaks either way,
    so the GPU may pick either of them."""
    u = np.where(keep[None, :], sub, 0.0)
    k = 0
    for j in range(u.shape[1]):
        if keep[j]:
            continue
        lev = 1.0 - (u ** 2).sum(1)
        p = int(pivots[k])
        k += 1
        assert lev[p] >= lev.max() - delta, (j, p, float(lev[p]), float(lev.max()))
        v = np.zeros(u.shape[0])
        v[p] = 1.0
        for _ in range(2):
            v = v - u @ (u.T @ v)
        u[:, j] = v / np.linalg.norm(v)
    return u


@pytest.mark.parametrize("name,b", [("clustered_large", 32), ("tall_lowrank", 64)])
def test_configured_sizes_against_lapack(pkg, name, b):
    """The two blocked configurations at their full sizes through the drop-in
    svd(a, 'block_jacobi', block_size=b): 4096 x 1024 with 64 clusters of 16
    values (cond 1e6), and 8192 x 2048 rank 64 plus N(0, 1e-6) noise.

    The reference zeroes sigma <= cut = eps32 * max(m, n) * sigma_1 and
    completes those U columns (solvers.py:18-21).  Bounds, against SciPy
    FP64 gesdd of the same float32 input:
      * resolved values (sigma > 2 cut): relative error <= 1e-5;
      * values below cut / 2 are reported as 0, every reported value is
        within 1e-5 sigma_1 of the truth;
      * |V^T V - I| <= 2e-5;
      * U (kept and completed columns): |U^T U - I| <= 2e-5 (the kept
        columns re-orthogonalised at the finish);
      * ||A - U S V^T|| / ||A|| within 2e-5 of the cut values' own share;
      * the completed columns are the oracle's completion of the kept ones
        (first 40 missing columns, FP64 oracle: same pivots, 1e-5)."""
    import scipy.linalg
    wl = importlib.import_module("pavel-s_svd_b200.workloads")
    a_np = getattr(wl, name)()
    m, n = a_np.shape
    a = torch.from_numpy(a_np).cuda()
    u, s, vh, info = pkg.svd(a, 'block_jacobi', block_size=b, return_info=True)
    assert info['block_size_used'] == b and info['converged']
    sr = scipy.linalg.svd(a_np.astype(np.float64), compute_uv=False, lapack_driver="gesdd")
    s_np = s.cpu().numpy().astype(np.float64)
    cut = np.finfo(np.float32).eps * max(m, n) * sr[0]
    res = sr > 2 * cut
    assert res.sum() >= 64
    rel = np.abs(s_np[res] - sr[res]) / sr[res]
    assert float(rel.max()) <= 1e-5, float(rel.max())
    assert bool((s_np[sr < cut / 2] == 0).all())
    rep = s_np > 0
    assert float(np.abs(s_np[rep] - sr[rep]).max()) <= 1e-5 * sr[0]
    u64, vh64, a64 = u.double(), vh.double(), a.double()
    eye = torch.eye(n, dtype=torch.float64, device="cuda")
    assert float((vh64 @ vh64.T - eye).abs().max()) <= 2e-5
    ou = float((u64.T @ u64 - eye).abs().max())
    assert ou <= 2e-5, ou
    s64 = torch.from_numpy(s_np).cuda()
    rec = float((a64 - (u64 * s64) @ vh64).norm() / a64.norm())
    cut_share = float(np.sqrt((sr[~rep] ** 2).sum()) / np.sqrt((sr ** 2).sum()))
    assert rec <= cut_share + 2e-5, (rec, cut_share)
    # completion parity: the oracle's completion of the kept columns
    miss = np.flatnonzero(~rep)
    assert len(miss) > 0
    cols = np.concatenate([np.flatnonzero(rep), miss[:40]])
    cols.sort()
    sub = u.cpu().numpy().astype(np.float64)[:, cols]
    keep_sub = rep[cols]
    got = sub
    want = _replay_completion(sub, keep_sub, np.abs(got[:, ~keep_sub]).argmax(0))
    assert float(np.abs(got[:, ~keep_sub] - want[:, ~keep_sub]).max()) <= 1e-5
