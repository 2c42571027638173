"""Learned warm start for one-sided Jacobi.

A small BF16 MLP maps the normalised Gram sketch of a tall matrix (upper
triangle of A^T A / ||A||_F^2, n(n+1)/2 features) to a start V0 (n x n).
The start is orthonormalised by an in-kernel Householder QR and kept only
when it lowers the Gram off-norm of A V0 below that of A (else V = I: the
plain solver); Jacobi then finishes from W = A V0.  The network is trained
on the V's that the plain Jacobi solver itself produced (sign-canonicalised
columns, MSE loss).

Every product runs on jb_gemm_bf16 (tcgen05 tensor cores) and every other
step on this library's element-wise kernels: the network's forward and
backward passes and the Adam step are hand-written, not torch autograd.
There is no counterpart in the reference project, whose Jacobi always starts
from the identity (svdbench/standalone/primitives.py:324).
"""
from __future__ import annotations

import numpy as np
import torch

from . import native as N
from .solvers import Workspace, raise_for_status
from .tensor import gemm


def _st(dev):
    return torch.cuda.current_stream(dev).cuda_stream


def sketch(a: torch.Tensor) -> torch.Tensor:
    """(B, m, n) float32 CUDA -> (B, n(n+1)/2) bf16 features."""
    a = a.contiguous()
    b, m, n = a.shape
    x = torch.empty(b, n * (n + 1) // 2, dtype=torch.bfloat16, device=a.device)
    N.check(N.lib().jb_gram_sketch(a.data_ptr(), x.data_ptr(), b, m, n, _st(a.device)), "jb_gram_sketch")
    return x


def canonical_signs(v: torch.Tensor) -> torch.Tensor:
    """Flip each column of v (..., n, n) so that its largest-magnitude entry is
    positive: the Jacobi V is defined up to column signs."""
    idx = v.abs().argmax(-2, keepdim=True)
    sign = torch.sign(torch.gather(v, -2, idx))
    sign[sign == 0] = 1
    return v * sign


def transpose_bf16(x: torch.Tensor) -> torch.Tensor:
    """(rows, cols) f32 or bf16 -> (cols, rows) bf16 on the library's kernel."""
    rows, cols = x.shape
    out = torch.empty(cols, rows, dtype=torch.bfloat16, device=x.device)
    N.check(N.lib().jb_transpose_bf16(x.data_ptr(), int(x.dtype == torch.float32), out.data_ptr(), rows, cols, 1,
                                      _st(x.device)), "jb_transpose_bf16")
    return out


class WarmStartMLP:
    """dims[0] -> dims[1] -> ... -> dims[-1]; ReLU on hidden layers, linear
    output.  FP32 master weights with Adam state; BF16 copies (out x in) and
    transposes (in x out) feed the tensor cores."""

    def __init__(self, dims=(2080, 1024, 1024, 1024, 4096), device="cuda", seed=0):
        self.dims = tuple(int(d) for d in dims)
        self.device = torch.device(device)
        rng = np.random.default_rng(seed)
        self.w, self.b = [], []
        for din, dout in zip(self.dims[:-1], self.dims[1:]):
            bound = np.sqrt(6.0 / din) if dout != self.dims[-1] else np.sqrt(1.0 / din)
            self.w.append(torch.from_numpy(rng.uniform(-bound, bound, (dout, din)).astype(np.float32)).to(self.device))
            self.b.append(torch.zeros(dout, dtype=torch.float32, device=self.device))
        self.mw = [torch.zeros_like(w) for w in self.w]
        self.vw = [torch.zeros_like(w) for w in self.w]
        self.mb = [torch.zeros_like(b) for b in self.b]
        self.vb = [torch.zeros_like(b) for b in self.b]
        self.step = 0
        self.refresh()

    def refresh(self):
        """BF16 copies of the master weights (after loading or initialising)."""
        self.wb = [w.bfloat16() for w in self.w]
        self.wt = [transpose_bf16(w) for w in self.w]

    def state(self):
        return {f"w{i}": w.cpu().numpy() for i, w in enumerate(self.w)} | \
               {f"b{i}": b.cpu().numpy() for i, b in enumerate(self.b)} | {"dims": np.array(self.dims)}

    def load(self, state):
        for i in range(len(self.w)):
            self.w[i].copy_(torch.from_numpy(state[f"w{i}"]))
            self.b[i].copy_(torch.from_numpy(state[f"b{i}"]))
        self.refresh()

    def forward(self, x: torch.Tensor, keep=False):
        """x: (B, dims[0]) bf16 -> (B, dims[-1]) float32 (and the hidden
        activations when keep)."""
        lib = N.lib()
        st = _st(self.device)
        hs = [x]
        h = x
        L = len(self.w)
        for l in range(L):
            z = gemm(h, self.wb[l])                                  # (B, out) fp32
            last = l == L - 1
            out = torch.empty(z.shape, dtype=torch.float32 if last else torch.bfloat16, device=self.device)
            N.check(lib.jb_bias_act(z.data_ptr(), self.b[l].data_ptr(), out.data_ptr(), z.shape[0], z.shape[1],
                                    0 if last else 1, 0 if last else 1, st), "jb_bias_act")
            h = out
            if not last:
                hs.append(h)
        return (h, hs) if keep else h

    def gradients(self, x, target):
        """Loss sum((y - t)^2) / numel and the gradients of every parameter."""
        lib = N.lib()
        st = _st(self.device)
        y, hs = self.forward(x, keep=True)
        B = y.shape[0]
        dy = torch.empty_like(y)
        loss = torch.zeros(1, dtype=torch.float32, device=self.device)
        N.check(lib.jb_mse_grad(y.data_ptr(), target.data_ptr(), dy.data_ptr(), loss.data_ptr(), y.numel(),
                                2.0 / y.numel(), st), "jb_mse_grad")
        gw, gb = [None] * len(self.w), [None] * len(self.w)
        g = dy                                                       # (B, out) fp32
        for l in range(len(self.w) - 1, -1, -1):
            gb[l] = torch.empty(g.shape[1], dtype=torch.float32, device=self.device)
            N.check(lib.jb_col_sum(g.data_ptr(), gb[l].data_ptr(), g.shape[0], g.shape[1], st), "jb_col_sum")
            gT = transpose_bf16(g)                                   # (out, B)
            hT = transpose_bf16(hs[l])                               # (in, B)
            gw[l] = gemm(gT, hT)                                     # (out, in) = g^T h
            if l > 0:
                dh = gemm(g.bfloat16() if g.dtype == torch.float32 else g, self.wt[l])   # (B, in)
                gn = torch.empty(dh.shape, dtype=torch.float32, device=self.device)
                N.check(lib.jb_relu_backward(dh.data_ptr(), hs[l].data_ptr(), gn.data_ptr(), 0, dh.numel(), st),
                        "jb_relu_backward")
                g = gn
        return loss / y.numel(), gw, gb

    def train_step(self, x, target, lr=1e-3, beta1=0.9, beta2=0.999, eps=1e-8):
        lib = N.lib()
        st = _st(self.device)
        loss, gw, gb = self.gradients(x, target)
        self.step += 1
        for l in range(len(self.w)):
            out, inn = self.w[l].shape
            N.check(lib.jb_adam(self.w[l].data_ptr(), gw[l].data_ptr(), self.mw[l].data_ptr(), self.vw[l].data_ptr(),
                                self.wb[l].data_ptr(), self.wt[l].data_ptr(), out, inn, lr, beta1, beta2, eps,
                                self.step, st), "jb_adam")
            N.check(lib.jb_adam(self.b[l].data_ptr(), gb[l].data_ptr(), self.mb[l].data_ptr(), self.vb[l].data_ptr(),
                                None, None, 1, out, lr, beta1, beta2, eps, self.step, st), "jb_adam")
        return loss

    def predict_v0(self, a: torch.Tensor) -> torch.Tensor:
        """(B, m, n) -> start vectors (B, n, n), row-major, columns = vectors."""
        b, m, n = a.shape
        return self.forward(sketch(a)).view(b, n, n)


def assign_order(v: torch.Tensor) -> torch.Tensor:
    """Reorder and re-sign the columns of V (B, n, n) by a rule that sees only
    the SET of columns: greedily give the largest remaining |entry| of V its
    row as column position, then make every diagonal entry positive.  The
    solver returns columns sorted by singular value, which for a parameterised
    family is a random permutation of a smooth basis; this order is not."""
    b, n, _ = v.shape
    a = v.abs().clone()
    out = torch.empty_like(v)
    bi = torch.arange(b, device=v.device)
    for _ in range(n):
        flat = a.reshape(b, -1).argmax(-1)
        i, j = flat // n, flat % n
        col = v[bi, :, j]
        sign = torch.sign(v[bi, i, j])
        sign[sign == 0] = 1
        out[bi, :, i] = col * sign[:, None]
        a[bi, i, :] = -1
        a[bi, :, j] = -1
    return out


def labels(v: torch.Tensor, order="assign") -> torch.Tensor:
    """Training targets from the plain solver's V (B, n, n) alone, flattened
    row-major: 'assign' (assign_order, default) or 'sorted' (the solver's
    singular-value order with canonical signs)."""
    if order not in ("assign", "sorted"):
        raise ValueError("order must be 'assign' or 'sorted'")
    t = assign_order(v) if order == "assign" else canonical_signs(v)
    return t.reshape(v.shape[0], -1).contiguous()


def plain_v(a: torch.Tensor, precision="mixed"):
    """V and sweeps of the plain solver (V = I start) for a batch."""
    from .solvers import svd
    u, s, vh, info = svd(a, precision=precision, return_info=True)
    return vh.transpose(-1, -2).contiguous(), info


def train(net: WarmStartMLP, a_train: torch.Tensor, v_train: torch.Tensor, epochs=10, batch=1024, lr=1e-3,
          seed=0, log=None, order="assign"):
    """Minibatch Adam on (sketch(a), canonical V) pairs; returns per-epoch mean loss."""
    x_all = sketch(a_train)
    t_all = labels(v_train, order)
    g = torch.Generator(device="cpu").manual_seed(seed)
    hist = []
    n = x_all.shape[0]
    for ep in range(epochs):
        perm = torch.randperm(n, generator=g).to(a_train.device)
        tot = torch.zeros((), device=a_train.device)
        steps = 0
        for lo in range(0, n - batch + 1, batch):
            idx = perm[lo:lo + batch]
            tot += net.train_step(x_all[idx].contiguous(), t_all[idx].contiguous(), lr=lr)[0]
            steps += 1
        hist.append(float(tot) / max(steps, 1))
        if log:
            log(f"epoch {ep}: loss {hist[-1]:.5f}")
    return hist


class WarmSolver:
    """svd of a fixed-shape batch from the network's warm start."""

    def __init__(self, net: WarmStartMLP, m: int, n: int, batch: int, device="cuda", precision="mixed",
                 tol=None, max_sweeps=60):
        self.net, self.m, self.n, self.batch = net, m, n, batch
        self.device = torch.device(device)
        self.prec = N.PREC_MIXED if precision == "mixed" else N.PREC_NATIVE
        self.tol, self.max_sweeps = float(tol or 0.0), max_sweeps
        k = min(m, n)
        dev = self.device
        self.vstart = torch.empty(batch, n, n, dtype=torch.float32, device=dev)
        self.used = torch.zeros(batch, dtype=torch.int32, device=dev)
        self.off = torch.zeros(2, batch, dtype=torch.float32, device=dev)
        self.U = torch.empty(batch, m, k, dtype=torch.float32, device=dev)
        self.S = torch.empty(batch, k, dtype=torch.float32, device=dev)
        self.Vh = torch.empty(batch, k, n, dtype=torch.float32, device=dev)
        self.info = torch.zeros(2, batch, dtype=torch.int32, device=dev)
        lib = N.lib()
        self.ws = torch.empty(max(int(lib.jb_workspace_bytes(m, n, batch, 4, self.prec, 0)), 256), dtype=torch.uint8,
                              device=dev)

    def launch(self, a: torch.Tensor, v0: torch.Tensor | None = None):
        """Sketch -> network -> QR prep -> warm Jacobi, all enqueued on the stream."""
        lib = N.lib()
        st = _st(self.device)
        if v0 is None:
            v0 = self.net.predict_v0(a)
        N.check(lib.jb_warm_prep_f32(a.data_ptr(), v0.contiguous().data_ptr(), self.vstart.data_ptr(),
                                     self.used.data_ptr(), self.off[0].data_ptr(), self.off[1].data_ptr(), self.batch,
                                     self.m, self.n, st), "jb_warm_prep_f32")
        k = min(self.m, self.n)
        N.check(lib.jb_svd_warm_f32(a.data_ptr(), self.vstart.data_ptr(), self.U.data_ptr(), self.S.data_ptr(),
                                    self.Vh.data_ptr(), self.batch, self.m, self.n, k, 0, self.tol, self.max_sweeps,
                                    self.prec, self.info[0].data_ptr(), self.info[1].data_ptr(), self.ws.data_ptr(),
                                    self.ws.numel(), st), "jb_svd_warm_f32")

    def solve_from(self, a: torch.Tensor, vstart: torch.Tensor):
        """The Jacobi alone from a given orthonormal start V (B, n, n),
        row-major with the vectors as columns like launch's v0 (no network,
        no QR preparation, no fallback test): with the identity, the plain
        solver; with the generator's own frame, the ceiling of a perfect
        network."""
        lib = N.lib()
        self.vstart.copy_(vstart.transpose(-1, -2))       # the solver reads the columns contiguously
        k = min(self.m, self.n)
        N.check(lib.jb_svd_warm_f32(a.data_ptr(), self.vstart.data_ptr(), self.U.data_ptr(), self.S.data_ptr(),
                                    self.Vh.data_ptr(), self.batch, self.m, self.n, k, 0, self.tol, self.max_sweeps,
                                    self.prec, self.info[0].data_ptr(), self.info[1].data_ptr(), self.ws.data_ptr(),
                                    self.ws.numel(), _st(self.device)), "jb_svd_warm_f32")

    def check(self):
        host = self.info.cpu()
        raise_for_status(host[1], self.max_sweeps)
        return host[0].numpy(), self.used.cpu().numpy()
