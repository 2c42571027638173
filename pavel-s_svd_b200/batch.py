"""Uneven batches: thousands of matrices of different shapes in ONE call.

The reference can only batch equal shapes (svdbench/standalone/solvers.py:
289-290); a harness solving matrices of different sizes loops over
``svd(x, 'jacobi')`` one call per matrix.  ``UnevenBatch`` replaces that loop:
shapes are fixed when the plan is built (descriptors, output offsets, a
largest-first processing order and the workspace are made once), and every
solve is one call of ``jb_svd_uneven_f32`` -- one persistent kernel per
precision phase and size class -- that can be captured in a CUDA graph and
replayed.
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
    return np.argsort(-matrix_cost(np.asarray(m), np.asarray(n)), kind="stable").astype(np.int32)


def matrix_cost(m, n):
    """Estimated cost of one matrix: one sweep of one-sided Jacobi on the tall
    view costs ~ nt^2 (7 mt + 4 nt) (the sweep count varies little)."""
    mt, nt = np.maximum(m, n), np.minimum(m, n)
    return nt.astype(np.float64) ** 2 * (7 * mt + 4 * nt)


def shard_by_cost(m, n, parts):
    """Split one uneven batch into `parts` shards of about equal cost, for
    solving it on several devices with no exchange between them: the
    cost-ordered work list (cost_order, largest first) is dealt greedily,
    every matrix to the shard with the least cost so far (LPT, within one
    matrix's cost of the best split).  Returns `parts` sorted index arrays;
    every matrix is in exactly one shard."""
    import heapq
    parts = int(parts)
    if parts < 1:
        raise ValueError("parts must be >= 1")
    m = np.asarray(m, np.int64)
    n = np.asarray(n, np.int64)
    cost = matrix_cost(m, n)
    heap = [(0.0, p) for p in range(parts)]
    owner = np.empty(len(m), np.int64)
    for i in cost_order(m, n):
        load, p = heapq.heappop(heap)
        owner[i] = p
        heapq.heappush(heap, (load + float(cost[i]), p))
    return [np.flatnonzero(owner == p) for p in range(parts)]


class Launch:
    """Launch choices of an uneven solve: ``flags`` (ROUND_ROBIN pair order,
    BLOCK_WIDTH_8 register blocks, ONE_SIZE_CLASS: no separate half-size
    launch for matrices of at most 32 columns) and ``exit_ratio`` (the FP32 phase of a
    mixed solve hands over once no pair ratio of a sweep exceeds it; 0 = the
    library default 1e-2, < 0 = the FP32 phase runs to tol).  Every choice
    converges to the same tolerance; they differ only in speed."""

    def __init__(self, flags=0, exit_ratio=0.0):
        self.flags, self.exit_ratio = int(flags), float(exit_ratio)

    def __repr__(self):
        names = [n for n, b in (("round_robin", N.ROUND_ROBIN), ("block_width_8", N.BLOCK_WIDTH_8),
                                ("one_size_class", N.ONE_SIZE_CLASS)) if self.flags & b]
        return f"Launch({'|'.join(names) or 'default'}, exit_ratio={self.exit_ratio:g})"

    def key(self):
        return (self.flags, self.exit_ratio)


# Candidates the autotuner times (the first is the library default).
TUNE_CANDIDATES = (Launch(), Launch(exit_ratio=3e-3), Launch(exit_ratio=-1.0), Launch(N.BLOCK_WIDTH_8),
                   Launch(N.ONE_SIZE_CLASS), Launch(N.ROUND_ROBIN))
_tune_cache = {}


def tune(m, n, a_flat, *, precision="mixed", tol=None, max_sweeps=60, candidates=TUNE_CANDIDATES, repeats=3):
    """Autotuner: time every launch choice on this batch (CUDA events, graph
    replays after one warm-up) and return the fastest as a Launch, with the
    timings.  The result is cached per shape multiset, precision and
    tolerance, so a harness pays for it once, in preparation."""
    m = np.asarray(m, np.int64)
    n = np.asarray(n, np.int64)
    key = (hash(m.tobytes()), hash(n.tobytes()), precision, tol, max_sweeps)
    if key in _tune_cache:
        return _tune_cache[key]
    dev = a_flat.device
    times = {}
    for cand in candidates:
        plan = UnevenBatch(m, n, dev, tol=tol, max_sweeps=max_sweeps, precision=precision, launch=cand)
        g = plan.capture(a_flat)
        g.replay()
        plan.check()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(repeats):
            g.replay()
        e1.record()
        torch.cuda.synchronize(dev)
        plan.check()
        times[repr(cand)] = e0.elapsed_time(e1) / repeats
        del g, plan
    best = min(candidates, key=lambda c: times[repr(c)])
    _tune_cache[key] = (best, times)
    return best, times


class UnevenBatch:
    """Plan and buffers for solving a fixed list of shapes repeatedly.

    ``m``, ``n``: per-matrix shapes.  ``a_off``: element offsets of each
    matrix in the flat input (default: ``pack``'s layout).  Outputs are flat
    buffers ``U``, ``S``, ``Vh`` (reduced SVD, rank = min(m, n)) addressed by
    the per-matrix offsets; ``result(i)`` returns views.  The plan owns its
    workspace (ticket counters, the FP32 V hand-off) and output buffers, so
    one plan serves one stream at a time; solves on several streams at once
    take one plan each."""

    def __init__(self, m, n, device, *, a_off=None, tol=None, max_sweeps=60, precision="mixed",
                 values_only=False, order="cost", launch=None):
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
        # launch choices (see Launch / tune): flags JB_ROUND_ROBIN | JB_BLOCK_WIDTH_8 and the
        # FP32-phase exit ratio of the mixed solve
        self.launch_choice = launch or Launch()
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
        ws = lib.jb_uneven_workspace_bytes(self.max_m, self.max_n, self.count, self.precision,
                                           self.launch_choice.flags, int(xt))
        self.workspace = torch.empty(max(int(ws), 256), dtype=torch.uint8, device=dev)
        # Persistent kernels per solve (after a memset of the work tickets): one
        # per precision phase, two when the register path splits the batch
        # into size classes (widths above and up to 32 columns run in CTAs of
        # different sizes; the library does this for batches wider than 32
        # that fit the register tiles: max(m, n) <= 128, min(m, n) <= 64).
        phases = 2 if self.precision == N.PREC_MIXED else 1
        split = (not self.launch_choice.flags & (N.ROUND_ROBIN | N.BLOCK_WIDTH_8) and self.max_m <= 128
                 and 32 < self.max_n <= 64)
        self.kernels_per_solve = phases * (2 if split else 1)

    # -- solving ----------------------------------------------------------------
    def launch(self, a_flat: torch.Tensor, stream=None):
        """Enqueue one solve of all matrices of a_flat (float32, device)."""
        if a_flat.dtype != torch.float32 or a_flat.device != self.device:
            raise TypeError("a_flat must be a float32 tensor on the plan's device")
        lib = N.lib()
        st = stream.cuda_stream if stream is not None else torch.cuda.current_stream(self.device).cuda_stream
        ptr = lambda t: None if t is None else t.data_ptr()
        lc = self.launch_choice
        rc = lib.jb_svd_uneven_f32_ex(a_flat.data_ptr(), ptr(self.U), self.S.data_ptr(), ptr(self.Vh),
                                      self.desc.data_ptr(), self.order.data_ptr(), self.count, self.max_m,
                                      self.max_n, self.tol, self.max_sweeps, self.precision, lc.flags,
                                      lc.exit_ratio, self.info[0].data_ptr(), self.info[1].data_ptr(),
                                      self.workspace.data_ptr(), self.workspace.numel(), st)
        N.check(rc, "jb_svd_uneven_f32_ex")

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


def chunk_weights(chunks):
    """Relative cost of the chunks of a StreamedUneven: doubling from the
    first and towards the last chunk, at most 4 (8 chunks: 1 2 4 4 4 4 2 1).
    The first chunk's input copy and the last chunk's output copy are the
    only transfers left exposed, so those two chunks are the smallest."""
    return [float(min(2 ** i, 2 ** (chunks - 1 - i), 4)) for i in range(chunks)]


class StreamedUneven:
    """Host-to-host solve of an uneven batch with the transfers overlapped
    with the compute.

    The matrices (in ``pack`` order) are split into ``chunks`` contiguous
    groups with costs in the proportions of ``chunk_weights`` (small first and
    last chunks), each with its own UnevenBatch.  Per chunk: the host->device
    copy of its inputs on one copy stream, its solve once that copy has landed,
    the device->host copy of its U, S, Vh and status on another copy stream
    once the solve is done.  Chunks alternate between two compute streams, so
    the first CTAs of chunk i+1 start on the SMs that chunk i's last matrices
    leave idle.  The input copy of chunk i+1 and the output copy of chunk i-1
    overlap chunk i's solve, so a step costs about the compute plus the first
    chunk's input copy and the last chunk's output copy.  Host buffers are the
    flat ``pack`` layouts of the whole batch (pinned for asynchronous
    copies)."""

    def __init__(self, m, n, device, *, chunks=8, tol=None, max_sweeps=60, precision="mixed", launch=None):
        m = np.asarray(m, np.int64)
        n = np.asarray(n, np.int64)
        count = len(m)
        dev = torch.device(device)
        if dev.type == "cuda" and dev.index is None:
            dev = torch.device("cuda", torch.cuda.current_device())
        self.device, self.count, self.max_sweeps = dev, count, int(max_sweeps)
        k = np.minimum(m, n)
        self.a_off, self.a_total = _aligned_offsets(m * n)
        self.u_off, self.u_total = _aligned_offsets(m * k)
        self.s_off, self.s_total = _aligned_offsets(k)
        self.v_off, self.v_total = _aligned_offsets(k * n)
        mt, nt = np.maximum(m, n), np.minimum(m, n)
        cost = np.cumsum(nt.astype(np.float64) ** 2 * (7 * mt + 4 * nt))
        chunks = max(1, min(int(chunks), count))
        frac = np.cumsum(chunk_weights(chunks)) / np.sum(chunk_weights(chunks))
        cuts = [0] + [int(np.searchsorted(cost, cost[-1] * f)) + 1 for f in frac[:-1]] + [count]
        cuts = sorted(set(min(max(x, 0), count) for x in cuts))
        self.ranges = [(lo, hi) for lo, hi in zip(cuts[:-1], cuts[1:]) if hi > lo]

        def span(off, total, lo, hi):
            return int(off[lo]), int(off[hi]) if hi < count else total

        self.plans, self.dev_in, self.spans = [], [], []
        for lo, hi in self.ranges:
            plan = UnevenBatch(m[lo:hi], n[lo:hi], dev, tol=tol, max_sweeps=max_sweeps, precision=precision,
                               launch=launch)
            a0, a1 = span(self.a_off, self.a_total, lo, hi)
            self.plans.append(plan)
            self.dev_in.append(torch.empty(max(a1 - a0, 1), dtype=torch.float32, device=dev))
            self.spans.append((span(self.a_off, self.a_total, lo, hi), span(self.u_off, self.u_total, lo, hi),
                               span(self.s_off, self.s_total, lo, hi), span(self.v_off, self.v_total, lo, hi)))
        self.s_in = torch.cuda.Stream(dev)
        self.s_comp = [torch.cuda.Stream(dev), torch.cuda.Stream(dev)]
        self.s_out = torch.cuda.Stream(dev)
        self.host_info = [torch.empty(2, max(hi - lo, 1), dtype=torch.int32).pin_memory() for lo, hi in self.ranges]

    def host_buffers(self):
        """Pinned host buffers of the whole batch: (input, U, S, Vh)."""
        mk = lambda size: torch.empty(max(size, 1), dtype=torch.float32).pin_memory()
        return mk(self.a_total), mk(self.u_total), mk(self.s_total), mk(self.v_total)

    def run(self, host_in, host_u, host_s, host_vh):
        """Enqueue the overlapped copy-in / solve / copy-out of every chunk;
        the caller's current stream waits for all of it.  Call check() to
        synchronise and raise the reference's errors."""
        main = torch.cuda.current_stream(self.device)
        for s in (self.s_in, *self.s_comp, self.s_out):
            s.wait_stream(main)
        solved = []
        # each chunk's solve is enqueued right after its input copy, so the
        # first solve starts as soon as the (small) first chunk has landed
        for i, ((a, _, _, _), d, plan) in enumerate(zip(self.spans, self.dev_in, self.plans)):
            with torch.cuda.stream(self.s_in):
                d[:a[1] - a[0]].copy_(host_in[a[0]:a[1]], non_blocking=True)
                landed = torch.cuda.Event()
                landed.record(self.s_in)
            comp = self.s_comp[i % 2]
            comp.wait_event(landed)
            plan.launch(d, stream=comp)
            done = torch.cuda.Event()
            done.record(comp)
            solved.append(done)
        for plan, (_, u, s_, v), ev, info in zip(self.plans, self.spans, solved, self.host_info):
            self.s_out.wait_event(ev)
            with torch.cuda.stream(self.s_out):
                host_u[u[0]:u[1]].copy_(plan.U[:u[1] - u[0]], non_blocking=True)
                host_s[s_[0]:s_[1]].copy_(plan.S[:s_[1] - s_[0]], non_blocking=True)
                host_vh[v[0]:v[1]].copy_(plan.Vh[:v[1] - v[0]], non_blocking=True)
                info[:, :plan.count].copy_(plan.info[:, :plan.count], non_blocking=True)
        main.wait_stream(self.s_out)

    def check(self):
        """Synchronise; raise for any failed matrix; return the sweep counts."""
        self.s_out.synchronize()
        if not self.plans:
            return np.zeros(0, np.int32)
        info = np.concatenate([h[:, :p.count].numpy() for p, h in zip(self.plans, self.host_info)], axis=1)
        if info[1].any():
            raise_for_status(torch.from_numpy(info[1]), self.max_sweeps)
        return info[0].copy()

    def device_bytes_per_run(self):
        """Bytes copied host->device and device->host by one run."""
        return 4 * self.a_total, 4 * (self.u_total + self.s_total + self.v_total) + 8 * self.count


class ShardedUneven:
    """One uneven batch solved on several devices at once.

    The batch is split by shard_by_cost into one share per device; each
    device gets an UnevenBatch over its share and solves it on its own
    current stream.  Nothing is exchanged between devices: every device reads
    its own inputs and writes its own outputs, and the host only gathers
    them.  One host thread enqueues every device's launch (they are
    asynchronous), so the devices run concurrently."""

    def __init__(self, m, n, devices, *, tol=None, max_sweeps=60, precision="mixed", values_only=False,
                 launch=None):
        self.m = np.asarray(m, np.int64)
        self.n = np.asarray(n, np.int64)
        self.count = len(self.m)
        self.devices = [torch.device(d) for d in devices]
        if not self.devices:
            raise ValueError("at least one device")
        self.shards = shard_by_cost(self.m, self.n, len(self.devices))
        self.max_sweeps = int(max_sweeps)
        self.plans = [UnevenBatch(self.m[idx], self.n[idx], dev, tol=tol, max_sweeps=max_sweeps,
                                  precision=precision, values_only=values_only, launch=launch)
                      if len(idx) else None for idx, dev in zip(self.shards, self.devices)]
        self.where = np.empty((self.count, 2), np.int64)      # matrix -> (shard, index in shard)
        for p, idx in enumerate(self.shards):
            self.where[idx, 0] = p
            self.where[idx, 1] = np.arange(len(idx))

    def pack(self, mats):
        """Per-device flat inputs (float32) of a list of host matrices."""
        flats = []
        for idx, dev, plan in zip(self.shards, self.devices, self.plans):
            if plan is None:
                flats.append(None)
                continue
            flat, _, _, _ = pack([mats[i] for i in idx])
            flats.append(flat.pin_memory().to(dev, non_blocking=True))
        return flats

    def launch(self, flats):
        """Enqueue every device's solve on that device's current stream."""
        for plan, flat, dev in zip(self.plans, flats, self.devices):
            if plan is not None:
                with torch.cuda.device(dev):
                    plan.launch(flat)

    def check(self):
        """Synchronise every device; raise for any failed matrix; return the
        sweep counts in the batch's order."""
        sweeps = np.zeros(self.count, np.int32)
        for idx, plan in zip(self.shards, self.plans):
            if plan is not None:
                sweeps[idx] = plan.check()
        return sweeps

    def result(self, i):
        p, j = self.where[i]
        return self.plans[p].result(int(j))


REGISTER_ROWS, REGISTER_COLS = 128, 64   # tall-view limits of the register kernels


def svd_uneven(mats, *, tol=None, max_sweeps=60, precision="mixed", values_only=False):
    """Solve a list of float32 CUDA matrices of different shapes in one call.
    Returns a list of (U, s, Vh) like svd() of each matrix would.  The
    matrices the register kernels take (tall view up to REGISTER_ROWS x
    REGISTER_COLS) are one persistent launch; larger ones, which would move
    the whole launch to the general kernels, go through svd() one by one
    (large tiles, QR first)."""
    if not mats:
        return []
    dev = mats[0].device
    for a in mats:
        if a.dtype != torch.float32 or a.ndim != 2 or a.device != dev:
            raise TypeError("svd_uneven takes 2-D float32 tensors on one CUDA device")
    fits = [max(a.shape) <= REGISTER_ROWS and min(a.shape) <= REGISTER_COLS for a in mats]
    out = [None] * len(mats)
    idx = [i for i, f in enumerate(fits) if f]
    if idx:
        m = np.array([mats[i].shape[0] for i in idx], np.int64)
        n = np.array([mats[i].shape[1] for i in idx], np.int64)
        plan = UnevenBatch(m, n, dev, tol=tol, max_sweeps=max_sweeps, precision=precision, values_only=values_only)
        flat = torch.zeros(int(plan.a_off[-1] + m[-1] * n[-1] + 4), dtype=torch.float32, device=dev)
        for i, o in zip(idx, plan.a_off):
            flat[int(o):int(o) + mats[i].numel()] = mats[i].reshape(-1)
        plan.launch(flat)
        plan.check()
        for j, i in enumerate(idx):
            out[i] = plan.result(j)
    if len(idx) < len(mats):
        from .solvers import svd
        for i, f in enumerate(fits):
            if not f:
                out[i] = svd(mats[i], "jacobi", tol=tol, max_sweeps=max_sweeps, precision=precision,
                             values_only=values_only)
    return out
