"""Blocked one-sided Jacobi SVD of one large matrix on the tensor cores.

Counterpart of block_jacobi (svdbench/standalone/solvers.py:30-68): column
blocks of width b, a round-robin tournament over blocks (primitives.py:309-313),
and per block pair the rotation vv of the pair's own SVD applied to W and V.
B200 form, per round, all block pairs ("slots") at once:

    G_k  = X_k X_k^T        jb_gemm_bf16x, SYRK + CHAIN128: one TMA stream of
                            the slot's 2b rows of W^T read as both operands,
                            accumulation chains of <= 128 along K in separate
                            tensor-memory accumulators summed in FP32
    vv_k = eig(G_k)         jb_block_eig_f64: FP64 Jacobi on the 2b x 2b Gram,
                            eigenvectors sorted by descending eigenvalue (the
                            reference's inner SVD sorts, primitives.py:357-358)
    X_k <- vv_k^T X_k       jb_gemm_bf16x_rows: the update for W^T and V^T,
                            each rotated row written as BF16 parts straight
                            into its slot of the next round

Precision stages.  The first sweeps run on two-part operands (compensated
3xBF16 products, FP32 accumulation): their off value counts only columns of
norm >= 1e-2 sigma_1, for which the ~2^-16 sigma_1 storage error of a part
pair is harmless, and they end when it is <= `switch`.  Then V is made
orthogonal (Newton-Schulz, 6xBF16 products), W = A V is recomputed from the
exact input with FP64 accumulation (jb_gemm_f64acc), and the sweeps continue
on three-part operands (6xBF16, ~FP32) over the reference's live set until
off <= tol_phase1 (the reference's 40 eps32, solvers.py:41,55-57).

Finish: V orthogonalised again, W = A V with FP64 accumulation, sigma =
column norms in FP64, sorted descending, values below eps32 * max(m, n) *
sigma_1 reported as 0 and their U columns replaced by the reference's null
completion (solvers.py:18-21, 61-66; jb_complete_null).  With V orthogonal to ~1e-6
and W's columns orthogonal to ~tol_phase1, every sigma above the cut keeps a
relative error of a few 1e-6.
"""
from __future__ import annotations

import math

import numpy as np
import torch

from . import native as N
from .tensor import gemm_parts, gemm_parts_rows, gemm_parts_rows2, split3_bf16


def _st(dev):
    return torch.cuda.current_stream(dev).cuda_stream


def circ(pos, r, n):
    return 0 if pos == 0 else 1 + (pos - 1 - r) % (n - 1)


def schedule(nb):
    """slot[r][k] = (i, j), i < j: the blocks of pair slot k in round r
    (circle method, primitives.py:309-313)."""
    out = []
    for r in range(nb - 1):
        row = []
        for k in range(nb // 2):
            a, b = circ(k, r, nb), circ(nb - 1 - k, r, nb)
            row.append((min(a, b), max(a, b)))
        out.append(row)
    return out


# W = A V at the stage switch and the finish runs on the tensor cores when the
# columns the reference's cut keeps span at most this ratio (else FP64 sums)
TENSOR_W_COND = 32.0


class BlockJacobi:
    """Plan + buffers for one m x n (m >= n) float32 matrix, block width b."""

    def __init__(self, m, n, block_size, device="cuda"):
        self.m, self.n, self.b = int(m), int(n), int(block_size)
        if self.m < self.n:
            raise ValueError("BlockJacobi takes tall matrices (m >= n)")
        b = self.b
        if b < 8 or b % 8 or 2 * b > 128:
            raise ValueError("block_size must be a multiple of 8 in [8, 64]")
        nb = -(-self.n // b)
        nb += nb % 2
        self.nb, self.npad, self.P = nb, nb * b, nb // 2
        self.mpad = -(-self.m // 8) * 8
        dev = torch.device(device)
        if dev.type == "cuda" and dev.index is None:
            dev = torch.device("cuda", torch.cuda.current_device())
        self.device = dev
        self.sched = schedule(nb)
        R = nb - 1
        # slot position of every block in every round: pos[r][blk] = (k, h)
        pos = np.zeros((R, nb, 2), np.int64)
        for r, row in enumerate(self.sched):
            for k, (i, j) in enumerate(row):
                pos[r, i] = (k, 0)
                pos[r, j] = (k, 1)
        self.pos = pos
        # update output row (k, t) of round r -> row in round r+1's layout
        maps = np.zeros((R, self.P * 2 * b), np.int32)
        for r in range(R):
            nr = (r + 1) % R
            for k, (i, j) in enumerate(self.sched[r]):
                for t in range(2 * b):
                    blk = i if t < b else j
                    k2, h2 = pos[nr, blk]
                    maps[r, k * 2 * b + t] = k2 * 2 * b + h2 * b + (t % b)
        self.maps = torch.from_numpy(maps).to(dev)
        # column c -> row of round 0's layout; and the inverse for every round
        init = np.zeros(self.npad, np.int32)
        for c in range(self.npad):
            k, h = pos[0, c // b]
            init[c] = k * 2 * b + h * b + c % b
        self.init_map = torch.from_numpy(init).to(dev)
        back = np.zeros((R, self.npad), np.int32)
        for r in range(R):
            for c in range(self.npad):
                k, h = pos[r, c // b]
                back[r, k * 2 * b + h * b + c % b] = c
        self.back_maps = torch.from_numpy(back).to(dev)
        bf = dict(dtype=torch.bfloat16, device=dev)
        rows = self.P * 2 * b
        # [buffer][part]: hi, mid (lo of the two-part split), lo (three-part split)
        self.W = [[torch.zeros(rows, self.mpad, **bf) for _ in range(3)] for _ in range(2)]
        self.V = [[torch.zeros(rows, self.npad, **bf) for _ in range(3)] for _ in range(2)]
        f32 = dict(dtype=torch.float32, device=dev)
        self.G = torch.empty(self.P, 2 * b, 2 * b, **f32)
        self.Qt = [torch.empty(self.P, 2 * b, 2 * b, **bf) for _ in range(3)]
        self.off = torch.zeros(R, self.P, **f32)
        self.dmax = torch.zeros(R, self.P, **f32)
        self.Gfull = torch.empty(self.npad, self.npad, **f32)      # post-sweep Gram of the whole W
        self.post_off = torch.zeros(1, **f32)
        self.isweeps = torch.zeros(self.P, dtype=torch.int32, device=dev)
        self.live = torch.zeros(1, dtype=torch.float64, device=dev)   # live-column floor of the sweep
        # CTAs along K of the Gram products: about one wave over the SMs
        self.gram_split = max(1, torch.cuda.get_device_properties(dev).multi_processor_count // self.P)
        # layout of the register eigen-solve: columns of G per warp (4, 8 or 16)
        self.eig_variant = 8
        # the two-part sweeps' Grams carry ~16-bit accuracy: their eigen-solves
        # rotate G in FP32 (jb_block_eig_f64_ex with JB_EIG_FP32; measured on
        # the 4096 x 1024 and 8192 x 2048 configurations: 1.3x faster per call,
        # the same block sweeps and sigma errors); the three-part sweeps in FP64
        self.eig_fp32_two_part = True
        # the three-part sweeps' eigen-solves in FP32 too when every column the
        # cut keeps is within TENSOR_W_COND of sigma_1 (set at the stage switch)
        self._eig_fp32_three_part = False
        # "batched": every round's products as one launch per kind; "dataflow":
        # per-slot launches on per-slot streams with only the true dependencies
        # (_sweep_dataflow), so products overlap other slots' eigen-solves
        self.schedule = "batched"
        self.slot_split = 1            # K split of a per-slot Gram (1: the fewest CTAs TMEM allows)
        # Q of the register eigen-solve formed by a separate all-GPU kernel from
        # the recorded rotations (JB_EIG_DEFER_Q), with a workspace per slot
        self.eig_defer_q = False
        self._eig_ws, self._eig_ws_slot = None, 0
        self.tuned = None
        self._graphs, self._seen, self._pool = {}, set(), None

    def _combine_v(self, cur):
        """V^T (npad x npad, FP32) from the slots of buffer `cur` (round 0 layout)."""
        vt = torch.empty(self.npad, self.npad, dtype=torch.float32, device=self.device)
        N.check(N.lib().jb_rows_combine(self.V[cur][0].data_ptr(), self.V[cur][1].data_ptr(),
                                        self.V[cur][2].data_ptr(), self.back_maps[0].data_ptr(), vt.data_ptr(),
                                        self.P * 2 * self.b, self.npad, _st(self.device)), "combine V")
        return vt

    def _polar(self, vt, steps):
        """Newton-Schulz: V <- V (3I - V^T V) / 2 on V^T rows (G = Vt Vt^T,
        Vt <- H Vt), SPLIT6 products with 128-long accumulation chains."""
        eye = torch.eye(self.npad, dtype=torch.float32, device=self.device)
        for _ in range(steps):
            vp = split3_bf16(vt)
            g = gemm_parts(vp, vp, chain128=True)[0]
            h = (3.0 * eye - g) * 0.5
            vt = gemm_parts(split3_bf16(h), vp, b_mn=True, chain128=True)[0]
        return vt

    def _polish_kept(self, U, r):
        """Re-orthogonalise the r kept columns of U (mpad x n, in place,
        columns in descending sigma) by one first-order Gram-Schmidt step
        against the larger columns: u_j <- u_j - sum_{k<j} (u_k . u_j) u_k,
        then unit length (SPLIT6 products).  U = A V / sigma carries V's
        FP32-level error times sigma_1 / sigma_j into a small column's
        direction (eps32 * cond from orthogonal); the step leaves the square
        of that.  Only the smaller column of each pair moves, by about its
        own error, so A - U S V^T changes by about eps32 sigma_1 (a symmetric
        polar step would move the large columns as much and cost sigma_1
        times the error)."""
        if r < 2:
            return
        r8 = -(-r // 8) * 8                                   # 16-byte rows for the products
        ut = torch.zeros(r8, self.mpad, dtype=torch.float32, device=self.device)
        ut[:r] = U[:, :r].T
        up = split3_bf16(ut)
        g = gemm_parts(list(up), list(up), chain128=True)[0]  # U^T U
        h = -torch.tril(g, diagonal=-1)                        # row j: -(u_k . u_j), k < j
        h.diagonal().fill_(1.0)
        h[r:], h[:, r:] = 0.0, 0.0
        ut = gemm_parts(list(split3_bf16(h.contiguous())), list(up), b_mn=True, chain128=True)[0][:r]
        U[:, :r] = (ut / ut.norm(dim=1, keepdim=True)).T

    def _cond_kept(self, cur, parts):
        """sigma_1 / the smallest column norm of W (buffer `cur`) that the
        reference's cut eps32 * max(m, n) * sigma_1 keeps (solvers.py:18-21)."""
        w = self.W[cur][0].float()
        for x in self.W[cur][1:parts]:
            w += x.float()
        nrm = w.pow(2).sum(1).sqrt()
        s1 = nrm.max()
        kept = nrm[nrm > np.finfo(np.float32).eps * max(self.m, self.n) * s1]
        return float(s1 / kept.min()) if kept.numel() else math.inf

    def _w_from_v(self, vt, ap, cond_kept=math.inf, ap_parts=None):
        """W^T = V^T A^T.  Exact float products summed in FP64
        (jb_gemm_f64acc) in general: a small kept column sigma_j carries the
        product's error times sigma_1 / sigma_j.  When every column the cut
        keeps is within TENSOR_W_COND of sigma_1, the six-term BF16 product on
        the tensor cores instead (hi, mid, lo splits of both operands, FP32
        chains of at most 128): about 2^-24 sigma_1 absolute in each column,
        so at most TENSOR_W_COND x 2^-24 (2e-6) relative to a kept one."""
        if cond_kept <= TENSOR_W_COND:
            return gemm_parts(list(split3_bf16(vt)), list(ap_parts if ap_parts is not None else split3_bf16(ap)),
                              chain128=True)[0]
        wt = torch.empty(self.npad, self.mpad, dtype=torch.float32, device=self.device)
        N.check(N.lib().jb_gemm_f64acc(vt.data_ptr(), ap.data_ptr(), wt.data_ptr(), self.npad, self.mpad, self.npad,
                                       self.npad, self.npad, self.mpad, _st(self.device)), "jb_gemm_f64acc")
        return wt

    def _sweep(self, cur, parts, inner_sweeps, inner_tol):
        """Enqueue one sweep (nb - 1 rounds) on the current stream; returns the
        buffer index holding the result (the rounds alternate buffers and
        their count is odd)."""
        lib = N.lib()
        st = _st(self.device)
        P, b = self.P, self.b
        for r in range(self.nb - 1):
            Wp = [x.view(P, 2 * b, self.mpad) for x in self.W[cur][:parts]]
            Vp = [x.view(P, 2 * b, self.npad) for x in self.V[cur][:parts]]
            # Grams of every slot: G_k = X_k X_k^T with X_k = 2b rows of W^T.
            gemm_parts(Wp, None, self.G, syrk=True, chain128=True, split_k=self.gram_split)
            self._eig(0, P, parts, r, inner_sweeps, inner_tol, st)
            # X_k <- vv^T X_k (rows of W^T), same for V, each rotated row
            # written (as BF16 parts) straight into its next-round slot.
            # (one launch for both: the same Q^T and row map)
            nxt = 1 - cur
            gemm_parts_rows2(self.Qt[:parts], Wp, self.W[nxt][:parts], Vp, self.V[nxt][:parts], self.maps[r],
                             b_mn=True)
            cur = nxt
        return cur

    def _dataflow_deps(self):
        """Per round r (of a sweep) and next-round slot k: src[r][k], the
        round-r slots whose updates write slot k's rows of round r + 1; war[r][k],
        the round-r slots that read the rows slot k's round r + 1 update
        overwrites (its blocks' positions two rounds on, in the buffer round r
        read).  Both sets have at most two slots."""
        if getattr(self, "_deps", None) is None:
            R, pos = self.nb - 1, self.pos
            src, war = [], []
            for r in range(R):
                nr, nnr = (r + 1) % R, (r + 2) % R
                src.append([sorted({int(pos[r, i, 0]), int(pos[r, j, 0])}) for i, j in self.sched[nr]])
                war.append([sorted({int(pos[nnr, i, 0]), int(pos[nnr, j, 0])}) for i, j in self.sched[nr]])
            self._deps = (src, war)
        return self._deps

    def _sweep_dataflow(self, cur, parts, inner_sweeps, inner_tol):
        """One sweep as a per-slot dataflow: slot k's Gram, eigen-solve and
        W / V updates run on stream k; the Gram of next-round slot k waits only
        for the two updates that write its rows, and an update waits for the
        round-before readers of the rows it overwrites.  Captured into a CUDA
        graph, one slot's products run on the SMs the other slots'
        eigen-solves leave free, instead of every round's products waiting for
        the slowest eigen-solve.  The same kernels and arithmetic per slot as
        _sweep."""
        lib = N.lib()
        P, b, R = self.P, self.b, self.nb - 1
        L = 2 * b
        src, war = self._dataflow_deps()
        main = torch.cuda.current_stream(self.device)
        if getattr(self, "_slot_streams", None) is None:
            self._slot_streams = [torch.cuda.Stream(self.device) for _ in range(P)]
        streams = self._slot_streams
        fork = torch.cuda.Event()
        fork.record(main)
        for st in streams:
            st.wait_event(fork)
        ev_w = [[torch.cuda.Event() for _ in range(P)] for _ in range(R)]
        ev_v = [[torch.cuda.Event() for _ in range(P)] for _ in range(R)]
        for r in range(R):
            nxt = 1 - cur
            Wp = [x.view(P, L, self.mpad) for x in self.W[cur][:parts]]
            Vp = [x.view(P, L, self.npad) for x in self.V[cur][:parts]]
            for k in range(P):
                st = streams[k]
                with torch.cuda.stream(st):
                    if r > 0:
                        for q in src[r - 1][k]:
                            st.wait_event(ev_w[r - 1][q])
                    gemm_parts([x[k:k + 1] for x in Wp], None, self.G[k:k + 1], syrk=True, chain128=True,
                               split_k=self.slot_split)
                    qt = self._eig(k, 1, parts, r, inner_sweeps, inner_tol, st.cuda_stream)
                    if r > 0:
                        for q in war[r - 1][k]:
                            st.wait_event(ev_w[r - 1][q])
                    rows = self.maps[r][k * L:(k + 1) * L]
                    gemm_parts_rows(qt, [x[k:k + 1] for x in Wp], self.W[nxt][:parts], rows, b_mn=True)
                    ev_w[r][k].record(st)
                    if r > 0:
                        for q in war[r - 1][k]:
                            st.wait_event(ev_v[r - 1][q])
                    gemm_parts_rows(qt, [x[k:k + 1] for x in Vp], self.V[nxt][:parts], rows, b_mn=True)
                    ev_v[r][k].record(st)
            cur = nxt
        for k in range(P):
            main.wait_event(ev_w[R - 1][k])
            main.wait_event(ev_v[R - 1][k])
        return cur

    def _eig_variant(self, parts):
        if 2 * self.b not in (64, 128):
            return 0
        fp32 = (parts == 2 and self.eig_fp32_two_part) or (parts == 3 and self._eig_fp32_three_part)
        return self.eig_variant | (N.EIG_FP32 if fp32 else 0) | (N.EIG_DEFER_Q if self.eig_defer_q else 0)

    def _eig(self, k, count, parts, r, inner_sweeps, inner_tol, stream):
        """Eigen-solves of slots k .. k + count - 1 of round r (jb_block_eig_ws),
        with slot k's workspace region when Q is deferred."""
        lib = N.lib()
        L = 2 * self.b
        variant = self._eig_variant(parts)
        ws, ws_bytes = None, 0
        if variant & N.EIG_DEFER_Q:
            per = int(lib.jb_block_eig_workspace_bytes(1, L, inner_sweeps))
            if self._eig_ws is None or self._eig_ws_slot < per:
                self._eig_ws = torch.empty(self.P * per, dtype=torch.uint8, device=self.device)
                self._eig_ws_slot = per
            per = self._eig_ws_slot
            ws, ws_bytes = self._eig_ws.data_ptr() + k * per, count * per
        qt = [x[k:k + count] for x in self.Qt[:parts]]
        N.check(lib.jb_block_eig_ws(self.G[k].data_ptr(), qt[0].data_ptr(), qt[1].data_ptr(),
                                    qt[2].data_ptr() if parts == 3 else None, self.off[r, k:].data_ptr(),
                                    self.dmax[r, k:].data_ptr(), self.isweeps[k:].data_ptr(), count, L, inner_sweeps,
                                    inner_tol, self.live.data_ptr(), variant, ws, ws_bytes, stream),
                "jb_block_eig_ws")
        return qt

    def _post_sweep_off(self, cur, parts, live_rel):
        """The reference's convergence test after a sweep (solvers.py:51-58),
        on the device into self.post_off: the largest |g_pq| / sqrt(g_pp g_qq)
        over pairs of live columns (g_pp > live_rel * max g) of G = W^T W, G
        formed on the tensor cores from the stored parts of W (all rows of W^T
        at once; their slot order does not change the maximum).  The in-sweep
        off of the eigen-solves sees a pair only when its slot meets it in the
        next sweep, one sweep later than this test.  No host sync: it is
        captured with the sweep."""
        w = list(self.W[cur][:parts])
        g = gemm_parts(w, w, self.Gfull, chain128=True)
        d = g.diagonal().clamp_min(0)
        live = d > live_rel * d.max()
        # 1 / sqrt(g_pp) for live columns, 0 for the others (which drops their pairs)
        inv = torch.where(live, d.sqrt(), torch.full_like(d, math.inf)).reciprocal()
        corr = g.abs().mul_(inv[:, None]).mul_(inv[None, :])
        corr.fill_diagonal_(0)
        self.post_off.copy_(corr.max().reshape(1))

    def _run_sweep(self, cur, parts, inner_sweeps, inner_tol, use_graphs, post_rel=None):
        """One sweep, replayed from a CUDA graph after its first (eager) run:
        the ~4 (nb - 1) launches of a sweep then cost one host call.  The
        graphs hold only this plan's buffers; the live floor is read on the
        device (self.live).  post_rel: also run the post-sweep test
        (_post_sweep_off) with that live floor, in the same graph."""
        key = (cur, parts, inner_sweeps, inner_tol, self._eig_variant(parts), self.gram_split, self.schedule,
               self.slot_split, post_rel)
        sweep = self._sweep_dataflow if self.schedule == "dataflow" else self._sweep

        def body():
            nxt = sweep(cur, parts, inner_sweeps, inner_tol)
            if post_rel is not None:
                self._post_sweep_off(nxt, parts, post_rel)
            return nxt

        if not use_graphs or key not in self._seen:
            self._seen.add(key)
            return body()
        g = self._graphs.get(key)
        if g is None:
            # the plan's graphs replay one at a time on one stream: one memory
            # pool serves the temporaries of all of them
            if self._pool is None:
                self._pool = torch.cuda.graph_pool_handle()
            g = torch.cuda.CUDAGraph()
            with torch.cuda.graph(g, pool=self._pool):
                body()
            self._graphs[key] = g
        g.replay()
        return 1 - cur

    def _load(self, a):
        """Check a, scale it by 2^-e (exact), and place its columns (rows of
        W^T) and the identity V in the slots of round 0 (buffer 0).  Returns
        (A padded, its transpose, e)."""
        lib = N.lib()
        dev, st = self.device, _st(self.device)
        m, n = self.m, self.n
        if tuple(a.shape) != (m, n) or a.dtype != torch.float32 or a.device != dev:
            raise ValueError("input must be a float32 (m, n) tensor on the plan's device")
        if not bool(torch.isfinite(a).all()):
            raise ValueError("input contains NaN or infinity")
        amax = float(a.abs().max())
        e = math.frexp(amax)[1] if amax > 0 else 0
        # A padded (mpad x npad), scaled by 2^-e (exact); W^T rows = columns of A.
        ap = torch.zeros(self.mpad, self.npad, dtype=torch.float32, device=dev)
        ap[:m, :n] = a * (2.0 ** -e)
        at = ap.t().contiguous()                                   # npad x mpad
        eye = torch.eye(self.npad, dtype=torch.float32, device=dev)
        for x in self.W + self.V:
            x[2].zero_()
        for buf, src, L in ((self.W[0], at, self.mpad), (self.V[0], eye, self.npad)):
            N.check(lib.jb_rows_scatter(src.data_ptr(), self.init_map.data_ptr(), buf[0].data_ptr(), buf[1].data_ptr(),
                                        None, None, self.npad, L, st), "scatter")
        return ap, at, e

    def tune(self, a: torch.Tensor, *, repeats=2):
        """Autotuner of the launch choices, on a's two-part sweeps (CUDA
        events, after a warm-up sweep); the fastest of each is kept for every
        later solve, and no choice changes a result beyond rounding:
          * the register eigen-solve's layout (4, 8 or 16 columns of G per
            warp; slot widths 64 and 128) and the Gram's split along K (about
            one wave of CTAs over the SMs, or twice that), timed as eager
            launches of the batched schedule;
          * then the schedule, batched or per-slot dataflow (with the per-slot
            Gram split the fewest CTAs TMEM allows, or twice that), timed as
            replays of the captured sweep graph.
        Returns {choice: ms per sweep}."""
        base_split = self.gram_split
        variants = (4, 8, 16) if 2 * self.b in (64, 128) else (8,)
        times = {}
        _, at, _ = self._load(a)
        self.live.fill_(1e-4 * float((at * at).sum(1).max()))     # the two-part stage's live floor
        self.schedule = "batched"
        cur = 0

        def timed(step, warm=1):                                   # ms per sweep
            nonlocal cur
            for _ in range(warm):
                cur = step(cur)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            for _ in range(repeats):
                cur = step(cur)
            e1.record()
            torch.cuda.synchronize(self.device)
            return e0.elapsed_time(e1) / repeats

        for dq in ((False, True) if 2 * self.b in (64, 128) else (False,)):
            for v in variants:
                for sp in (base_split, 2 * base_split):
                    self.eig_variant, self.gram_split, self.eig_defer_q = v, sp, dq
                    times[f"eig_cols_per_warp={v},gram_split={sp},defer_q={int(dq)}"] = timed(
                        lambda c: self._sweep(c, 2, 1, 1e-7))
        best = min(times, key=times.get)
        v, sp, dq = [int(x.split("=")[1]) for x in best.split(",")]
        self.eig_variant, self.gram_split, self.eig_defer_q = v, sp, bool(dq)
        graph_times = {}
        for sched, split in (("batched", 1), ("dataflow", 1), ("dataflow", 2)):
            self.schedule, self.slot_split = sched, split
            # a sweep has an odd number of rounds, so the buffer parity alternates:
            # two eager sweeps and two captures before the timed replays
            graph_times[(sched, split)] = timed(lambda c: self._run_sweep(c, 2, 1, 1e-7, True), warm=4)
            times[f"graph schedule={sched},slot_split={split}"] = graph_times[(sched, split)]
        self.schedule, self.slot_split = min(graph_times, key=graph_times.get)
        self.tuned = times
        return times

    def solve(self, a: torch.Tensor, *, tol_phase1=5e-6, switch=5e-2, max_sweeps=30, max_two_part=12,
              inner_sweeps=1, inner_tol=1e-7, polar_steps=2, require_convergence=True, use_graphs=True,
              post_check=True, post_end=0.05):
        """SVD of a (m x n float32, CUDA).  Returns U (m x n), S (n), Vh (n x n),
        info dict.

        The off value of a sweep is its largest pair ratio |g_pq| / sqrt(g_pp
        g_qq) over live columns.  Sweeps first run with two-part (3xBF16)
        operands, whose storage carries an absolute error of ~2^-16 sigma_1
        into every column: their off counts only columns of norm >= 1e-2
        sigma_1 (for which that error is harmless) and the stage ends when it
        is <= `switch` (or after `max_two_part` sweeps).  The three-part
        (6xBF16, ~FP32) sweeps then count the reference's live set (norm above
        eps32 * max(m, n) * the largest norm, solvers.py:55-57) and run until
        off <= tol_phase1, the reference's 40 eps32 (solvers.py:41).  Early
        sweeps are not monotone (columns migrate between blocks while the
        per-pair sort settles), so a stall -- off not halving for two sweeps
        -- only ends the solve once off < 1e-4, the FP32 floor regime.
        post_check: after every sweep also run the reference's own test on
        the Gram of the whole W (_post_sweep_off); the stage switch and the
        end of the solve then come one sweep sooner, the end only when that
        off is below post_end * tol_phase1 (0.05: a margin for the Gram's
        FP32-level rounding; on the configured cases 0.5 gives the same sweep
        counts and accuracy)."""
        lib = N.lib()
        dev, st = self.device, _st(self.device)
        m, n, b, P, R = self.m, self.n, self.b, self.P, self.nb - 1
        ap, at, e = self._load(a)
        cur = 0
        sweeps = 0
        off_hist = []
        parts = 2
        live_rel = (np.finfo(np.float32).eps * max(m, n)) ** 2
        dmax = float((at * at).sum(1).max())
        best, stall, converged, stage_sweeps = float("inf"), 0, False, 0
        self._eig_fp32_three_part = False
        post_hist = []
        ap_parts = None
        n_polar = n_wtensor = 0            # tensor-core products outside the sweeps, for info
        for sweeps in range(1, max_sweeps + 1):
            self.live.fill_((live_rel if parts == 3 else 1e-4) * dmax)
            stage_sweeps += 1
            cur = self._run_sweep(cur, parts, inner_sweeps, inner_tol, use_graphs,
                                  (live_rel if parts == 3 else 1e-4) if post_check else None)
            vals = torch.stack([self.off.max(), self.dmax.max(), self.post_off[0]]).cpu()   # one sync
            off = float(vals[0])
            dmax = max(dmax, float(vals[1]))
            off_hist.append((off, parts))
            post = float(vals[2]) if post_check else math.inf
            post_hist.append(post)
            if off < 0.5 * best:
                best, stall = off, 0
            elif off < 1e-4:
                stall += 1
            if parts == 3 and (off <= tol_phase1 or post <= post_end * tol_phase1 or stall >= 2):
                converged = True
                break
            if parts == 2 and (off <= switch or post <= switch or stage_sweeps >= max_two_part):
                # Re-synchronise before the accurate sweeps: V made orthogonal,
                # W = A V recomputed from the exact input (the 16-bit sweeps
                # left W's small columns off by ~2^-16 sigma_1 / sigma_j).
                parts_before, parts = parts, 3
                best, stall, stage_sweeps = float("inf"), 0, 0
                vt = self._combine_v(cur)
                vt = self._polar(vt, polar_steps)
                ck = self._cond_kept(cur, parts_before)
                ap_parts = split3_bf16(ap) if ck <= TENSOR_W_COND else None
                wt = self._w_from_v(vt, ap, ck, ap_parts)
                n_polar += polar_steps
                n_wtensor += int(ck <= TENSOR_W_COND)
                self._eig_fp32_three_part = ck <= TENSOR_W_COND
                for buf, src, L in ((self.W[cur], wt, self.mpad), (self.V[cur], vt, self.npad)):
                    N.check(lib.jb_rows_scatter(src.data_ptr(), self.init_map.data_ptr(), buf[0].data_ptr(),
                                                buf[1].data_ptr(), buf[2].data_ptr(), None, self.npad, L, st),
                            "scatter")
        if not converged and require_convergence:
            raise RuntimeError("block Jacobi did not converge")
        # The data now sits in round 0's layout of the next sweep.
        vt = self._polar(self._combine_v(cur), polar_steps)
        ck = self._cond_kept(cur, parts)
        wt = self._w_from_v(vt, ap, ck, ap_parts if ck <= TENSOR_W_COND else None)   # npad x mpad
        w_product = "six-term BF16 (tensor cores)" if ck <= TENSOR_W_COND else "FP64-accumulated"
        U = torch.empty(self.mpad, n, dtype=torch.float32, device=dev)
        S = torch.empty(n, dtype=torch.float32, device=dev)
        Vh = torch.empty(n, self.npad, dtype=torch.float32, device=dev)
        sig = torch.empty(self.npad, dtype=torch.float64, device=dev)
        perm = torch.empty(self.npad, dtype=torch.int32, device=dev)
        N.check(lib.jb_block_finish(wt.data_ptr(), vt.data_ptr(), U.data_ptr(), S.data_ptr(), Vh.data_ptr(),
                                    sig.data_ptr(), perm.data_ptr(), self.mpad, self.npad, n, e, max(m, n), st),
                "jb_block_finish")
        eig2 = "FP32" if self.eig_fp32_two_part else "FP64"
        eig3 = "FP32" if self._eig_fp32_three_part else "FP64"
        kept = int((S > 0).sum())
        self._polish_kept(U, kept)
        n_polar += polar_steps
        n_wtensor += int(ck <= TENSOR_W_COND)
        # Columns of cut sigma: the reference's completion vectors (_finish_columns,
        # solvers.py:18-21 -> primitives.py:430-455), on the device.
        from .solvers import _complete_null_columns
        U = _complete_null_columns(U[:m][None], (S > 0)[None])[0]
        info = {"algorithm": "block_jacobi", "block_sweeps": sweeps, "off_per_sweep": off_hist,
                "post_sweep_off": post_hist, "converged": converged,
                "reached_tol": off_hist[-1][0] <= tol_phase1 or post_hist[-1] <= post_end * tol_phase1,
                "precision": f"tensor-core sweeps (3xBF16 with {eig2} block eigen-solves, then 6xBF16 with "
                             f"{eig3} ones); 6xBF16 Newton-Schulz V, {w_product} W = A V",
                "eig_precision": (eig2, eig3),
                "cond_kept": ck, "kept_columns": kept,
                # the tensor-core products outside the sweeps: Newton-Schulz
                # steps on V, W = A V products, the re-orthogonalisation of U
                "polar_steps": n_polar, "tensor_w_products": n_wtensor}
        return U, S, Vh[:, :n].contiguous(), info
