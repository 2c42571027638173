"""Learned warm start: the network's hand-written backward pass against a CPU
FP64 reference, the warm-start solve against the plain solve, the identity
fallback, and the sweeps a trained network saves on held-out matrices.

Tolerances: gradients agree with the FP64 reference of the same BF16-rounded
forward pass to 3e-2 relative Frobenius error (BF16 gradients feed the
tensor-core products); singular values of warm and plain solves (both mixed
precision) agree to 1e-5 relative to sigma_1 and meet the 1e-5 relative
bound against FP64 LAPACK."""
import importlib

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def W():
    return importlib.import_module("pavel-s_svd_b200.warmstart")


def bf16(x):
    return torch.from_numpy(np.asarray(x, np.float32)).bfloat16().float().double().numpy()


def test_backward_matches_cpu_fp64(W):
    torch.manual_seed(0)
    net = W.WarmStartMLP(dims=(64, 32, 32, 48), seed=3)
    for b in net.b:
        b.normal_(0, 0.1)
    B = 16
    x = torch.randn(B, 64, device="cuda").bfloat16()
    t = torch.randn(B, 48, device="cuda")
    loss, gw, gb = net.gradients(x, t)
    torch.cuda.synchronize()
    # CPU FP64 reference of the same forward (bf16 weights and activations).
    ws = [bf16(w.cpu().numpy()) for w in net.w]
    bs = [b.cpu().double().numpy() for b in net.b]
    hs = [x.float().cpu().double().numpy()]
    h = hs[0]
    for l in range(3):
        z = h @ ws[l].T + bs[l]
        if l < 2:
            h = bf16(np.maximum(z, 0))
            hs.append(h)
        else:
            y = z
    tt = t.cpu().double().numpy()
    g = 2 * (y - tt) / y.size
    ref_loss = ((y - tt) ** 2).mean()
    assert abs(float(loss) - ref_loss) <= 1e-3 * ref_loss
    for l in range(2, -1, -1):
        ref_w = g.T @ hs[l]
        ref_b = g.sum(0)
        e_w = np.linalg.norm(gw[l].cpu().double().numpy() - ref_w) / np.linalg.norm(ref_w)
        e_b = np.linalg.norm(gb[l].cpu().double().numpy() - ref_b) / np.linalg.norm(ref_b)
        assert e_w <= 3e-2 and e_b <= 3e-2, (l, e_w, e_b)
        if l:
            g = (g @ ws[l]) * (hs[l] > 0)


def _family(workloads, count, seed=4):
    a, theta = workloads.warm_family(count=count, seed=seed, chunk=512)
    return torch.from_numpy(a).cuda()


def test_exact_and_garbage_starts(W, workloads):
    a = _family(workloads, 256)
    v, info = W.plain_v(a)
    solver = W.WarmSolver(net=None, m=128, n=64, batch=256)
    # exact start: the plain solver's own V
    solver.launch(a, v0=v.contiguous())
    sweeps_exact, used = solver.check()
    assert used.mean() > 0.95
    _, s_ref, _ = importlib.import_module("pavel-s_svd_b200").svd(a)
    assert float(((solver.S - s_ref).abs() / s_ref[:, :1]).max()) <= 1e-5
    assert sweeps_exact.mean() < info["jacobi_sweeps"] / 2
    # garbage start: random V0 (may be kept only if it lowers the off-norm)
    g = torch.Generator(device="cuda").manual_seed(1)
    solver.launch(a, v0=torch.randn(256, 64, 64, device="cuda", generator=g))
    sweeps_g, used_g = solver.check()
    assert float(((solver.S - s_ref).abs() / s_ref[:, :1]).max()) <= 1e-5


def test_trained_network_saves_sweeps(W, workloads):
    """The configured split: train on 60000 matrices of the family with labels
    taken only from the plain solver's V (columns in the label-only canonical
    order of assign_order), evaluate 4096 held-out matrices.  The trained
    start must lower the Gram off-norm, be kept for most matrices and save
    sweeps, with the same singular values; the ideal start (the generator's
    own V(theta), used here only as a bound) shows what a perfect network
    could save.  The gain in matrices/s is measured and printed, not
    asserted: on this family the saved sweeps (~4 %) pay neither for the
    network nor for the start's preparation (the in-kernel QR of V0 and the
    fallback test take about as long as the Jacobi itself), so the warm path
    is about 2x slower than the plain Jacobi from V = I alone.  What is
    bounded here is the network's own cost: the warm path against the
    identity start through the same preparation."""
    a_np, theta = workloads.warm_family(count=65536, device="cuda")
    a = torch.from_numpy(a_np).cuda()
    tr, te = a[:60000].contiguous(), a[60000:64096].contiguous()
    v_tr, _ = W.plain_v(tr)
    net = W.WarmStartMLP(seed=0)
    hist = W.train(net, tr, v_tr, epochs=15, batch=512, lr=1e-3, order="assign")
    assert hist[-1] < 0.5 * hist[0]
    solver = W.WarmSolver(net, m=128, n=64, batch=4096)
    eye = torch.eye(64, device="cuda").expand(4096, 64, 64).contiguous()

    def timed(v0):
        solver.launch(te, v0=v0)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(3):
            solver.launch(te, v0=v0)
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / 3

    ms_pipe_identity = timed(eye)                    # V0 = I through the same QR preparation
    n_plain, used0 = solver.check()
    s_plain = solver.S.clone()
    assert used0.sum() == 0
    ms_warm = timed(None)
    sweeps, used = solver.check()
    off0, off1 = float(solver.off[0].mean()), float(solver.off[1].mean())
    s_warm = solver.S.clone()
    solver.launch(te, v0=workloads.family_v(theta[60000:64096], device="cuda").contiguous())
    ideal, _ = solver.check()
    solver.solve_from(te, eye)                     # the plain Jacobi alone, for the printout
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(3):
        solver.solve_from(te, eye)
    e1.record()
    torch.cuda.synchronize()
    ms_plain_alone = e0.elapsed_time(e1) / 3
    print(f"held-out sweeps: plain {n_plain.mean():.2f} ({ms_plain_alone:.2f} ms alone, {ms_pipe_identity:.2f} ms "
          f"through the preparation), trained {sweeps.mean():.2f} ({ms_warm:.2f} ms, kept {used.mean():.2f}, "
          f"off-norm {off0:.3f} -> {off1:.3f}), ideal start {ideal.mean():.2f}")
    assert float(((s_warm - s_plain).abs() / s_plain[:, :1]).max()) <= 1e-5
    assert used.mean() > 0.5
    assert off1 < off0
    assert sweeps.mean() < n_plain.mean()
    assert ms_warm <= 1.15 * ms_pipe_identity
