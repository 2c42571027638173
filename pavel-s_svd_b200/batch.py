"""Uneven batches: thousands of matrices of different shapes in ONE launch.

The reference can only batch equal shapes (svdbench/standalone/solvers.py:
289-290); a harness solving matrices of different sizes loops over
``svd(x, 'jacobi')`` one call per matrix.  ``UnevenBatch`` replaces that loop:
shapes are fixed when the plan is built (descriptors, output offsets, a
largest-first processing order and the workspace are made once), and every
solve is one persistent-kernel launch (``jb_svd_uneven_f32``) that can be
captured in a CUDA graph and replayed.
"""
from __future__ import annotations

import numpy as np
import torch

from . import native as N
from .solvers import raise_for_status

DESC_DTYPE = np.dtype([("m", "<i4"), ("n", "<i4"), ("rank", "<i4"), ("flags", "<i4"),
                       ("a_off", "<i8"), ("u_off", "<i8"), ("s_off", "<i8"), ("v_off", "<i8"),
                       ("x_off", "<i8")])
assert DESC_DTYPE.itemsize == N.DESC_BYTES


def _aligned_offsets(sizes, align=4):
    sizes = (np.asarray(sizes, np.int64) + align - 1) // align * align
    off = np.zeros(len(sizes), np.int64)
    if len(sizes) > 1:
        off[1:] = np.cumsum(sizes)[:-1]
    return off, int(sizes.sum())


def pack(mats, device=None, dtype=np.float32):
    """Pack row-major matrices into one flat buffer with 4-element aligned
    offsets.  Returns (flat, m, n, a_off); flat is a torch tensor."""
    m = np.array([a.shape[0] for a in mats], np.int64)
    n = np.array([a.shape[1] for a in mats], np.int64)
    a_off, total = _aligned_offsets(m * n)
    flat = np.zeros(max(total, 1), dtype)
    for a, o in zip(mats, a_off):
        flat[o:o + a.size] = np.asarray(a, dtype).ravel()
    t = torch.from_numpy(flat)
    return (t.to(device) if device is not None else t), m, n, a_off


def cost_order(m, n):
    """Processing order, largest estimated cost first (LPT on the persistent
    grid): one sweep of one-sided Jacobi on the tall view costs ~ nt^2 (7 mt + 4 nt)."""
    mt, nt = np.maximum(m, n), np.minimum(m, n)
    cost = nt.astype(np.float64) ** 2 * (7 * mt + 4 * nt)
    return np.argsort(-cost, kind="stable").astype(np.int32)


class UnevenBatch:
    """Plan and buffers for solving a fixed list of shapes repeatedly.

    ``m``, ``n``: per-matrix shapes.  ``a_off``: element offsets of each
    matrix in the flat input (default: ``pack``'s layout).  Outputs are flat
    buffers ``U``, ``S``, ``Vh`` (reduced SVD, rank = min(m, n)) addressed by
    the per-matrix offsets; ``result(i)`` returns views."""

    def __init__(self, m, n, device, *, a_off=None, tol=None, max_sweeps=60, precision="mixed",
                 values_only=False, order="cost"):
        self.m = np.asarray(m, np.int64)
        self.n = np.asarray(n, np.int64)
        self.count = len(self.m)
        dev = torch.device(device)
        if dev.type == "cuda" and dev.index is None:
            dev = torch.device("cuda", torch.cuda.current_device())
        self.device = dev
        self.tol = float(tol or 0.0)
        self.max_sweeps = int(max_sweeps)
        if precision not in ("mixed", "fp32"):
            raise ValueError("precision must be 'mixed' or 'fp32'")
        self.precision = N.PREC_MIXED if precision == "mixed" else N.PREC_NATIVE
        k = np.minimum(self.m, self.n)
        if a_off is None:
            a_off, _ = _aligned_offsets(self.m * self.n)
        self.a_off = np.asarray(a_off, np.int64)
        self.u_off, ut = _aligned_offsets(self.m * k)
        self.s_off, st = _aligned_offsets(k)
        self.v_off, vt = _aligned_offsets(k * self.n)
        self.x_off, xt = _aligned_offsets(k * k)
        self.values_only = values_only
        desc = np.zeros(self.count, DESC_DTYPE)
        desc["m"], desc["n"], desc["rank"] = self.m, self.n, k
        desc["flags"] = N.VALUES_ONLY if values_only else 0
        desc["a_off"], desc["u_off"], desc["s_off"], desc["v_off"] = self.a_off, self.u_off, self.s_off, self.v_off
        desc["x_off"] = self.x_off
        dev = self.device
        self.desc = torch.from_numpy(desc.view(np.uint8).copy()).to(dev)
        self.order_host = cost_order(self.m, self.n) if order == "cost" else np.arange(self.count, dtype=np.int32)
        self.order = torch.from_numpy(self.order_host).to(dev)
        self.max_m = int(max(self.m.max(), self.n.max())) if self.count else 1
        self.max_n = int(np.minimum(self.m, self.n).max()) if self.count else 1
        self.U = None if values_only else torch.zeros(max(ut, 1), dtype=torch.float32, device=dev)
        self.S = torch.zeros(max(st, 1), dtype=torch.float32, device=dev)
        self.Vh = None if values_only else torch.zeros(max(vt, 1), dtype=torch.float32, device=dev)
        self.info = torch.zeros(2, max(self.count, 1), dtype=torch.int32, device=dev)
        lib = N.lib()
        # Workspace: the base area (ticket counters, per-CTA areas of the
        # round-robin kernels) followed, in mixed precision, by the scratch
        # floats the descriptors' x_off address.
        ws = lib.jb_uneven_workspace_bytes(self.max_m, self.max_n, self.count, self.precision, int(xt))
        self.workspace = torch.empty(max(int(ws), 256), dtype=torch.uint8, device=dev)
        # memset of the work tickets + one persistent kernel per precision phase
        self.kernels_per_solve = 2 if self.precision == N.PREC_MIXED else 1

    # -- solving ----------------------------------------------------------------
    def launch(self, a_flat: torch.Tensor, stream=None):
        """Enqueue one solve of all matrices of a_flat (float32, device)."""
        if a_flat.dtype != torch.float32 or a_flat.device != self.device:
            raise TypeError("a_flat must be a float32 tensor on the plan's device")
        lib = N.lib()
        st = stream.cuda_stream if stream is not None else torch.cuda.current_stream(self.device).cuda_stream
        ptr = lambda t: None if t is None else t.data_ptr()
        rc = lib.jb_svd_uneven_f32(a_flat.data_ptr(), ptr(self.U), self.S.data_ptr(), ptr(self.Vh),
                                   self.desc.data_ptr(), self.order.data_ptr(), self.count, self.max_m,
                                   self.max_n, self.tol, self.max_sweeps, self.precision,
                                   self.info[0].data_ptr(), self.info[1].data_ptr(), self.workspace.data_ptr(),
                                   self.workspace.numel(), st)
        N.check(rc, "jb_svd_uneven_f32")

    def capture(self, a_flat: torch.Tensor) -> torch.cuda.CUDAGraph:
        """Capture one solve over the fixed buffer a_flat into a CUDA graph."""
        self.launch(a_flat)  # first call sets kernel attributes outside capture
        torch.cuda.synchronize(self.device)
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            self.launch(a_flat)
        return g

    def check(self):
        """Synchronise, raise the reference's exception for any failed matrix,
        return the per-matrix sweep counts (numpy)."""
        host = self.info[:, :self.count].cpu().numpy()
        raise_for_status(torch.from_numpy(host[1]), self.max_sweeps)
        return host[0]

    def result(self, i):
        m, n = int(self.m[i]), int(self.n[i])
        k = min(m, n)
        s = self.S[self.s_off[i]:self.s_off[i] + k]
        if self.values_only:
            return None, s, None
        u = self.U[self.u_off[i]:self.u_off[i] + m * k].view(m, k)
        vh = self.Vh[self.v_off[i]:self.v_off[i] + k * n].view(k, n)
        return u, s, vh


def svd_uneven(mats, *, tol=None, max_sweeps=60, precision="mixed", values_only=False):
    """Solve a list of float32 CUDA matrices of different shapes in one launch.
    Returns a list of (U, s, Vh) like svd() of each matrix would."""
    if not mats:
        return []
    dev = mats[0].device
    for a in mats:
        if a.dtype != torch.float32 or a.ndim != 2 or a.device != dev:
            raise TypeError("svd_uneven takes 2-D float32 tensors on one CUDA device")
    m = np.array([a.shape[0] for a in mats], np.int64)
    n = np.array([a.shape[1] for a in mats], np.int64)
    plan = UnevenBatch(m, n, dev, tol=tol, max_sweeps=max_sweeps, precision=precision, values_only=values_only)
    flat = torch.zeros(int(plan.a_off[-1] + m[-1] * n[-1] + 4), dtype=torch.float32, device=dev)
    for a, o in zip(mats, plan.a_off):
        flat[int(o):int(o) + a.numel()] = a.reshape(-1)
    plan.launch(flat)
    plan.check()
    return [plan.result(i) for i in range(len(mats))]
