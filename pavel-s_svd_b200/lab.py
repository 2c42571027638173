"""The algorithm laboratory's Jacobi on the GPU: ``jacobi(a, trace=...)``
mirrors algorithm_laboratory/algorithms.py:105-157 of uncle-Slava/Pavel-s_SVD
(same arguments, checks, errors, trace calls and result), with its rounds run
by this library's ``jb_jacobi_rounds`` kernel on the matrix's W and V in
device memory instead of torch's per-round tensor operations.

The trace sees what the laboratory's own trace sees:
  * stage('jacobi_rotation', sweep, round=i) around each round, and with
    record_rotations a checkpoint('rotation_i', sweep, tensors={W, V, p, q})
    after it;
  * checkpoint('sweep', sweep, tensors={W, V}, scalars={max_active_pair_correlation,
    tolerance}, factors=...) after every sweep the trace wants;
  * record('convergence', ...), stage('sort_and_normalize'), checkpoint('final').
Without a trace that records anything (``trace.enabled`` false, no
record_rotations) a whole sweep is one launch.  A trace is any object with
the laboratory's interface (svdbench/laboratory/trace.py:38-43); the default
does nothing.
"""
from __future__ import annotations

from contextlib import nullcontext

import torch

from . import native as N

_DTYPE = {torch.float32: 0, torch.float64: 1, torch.complex64: 2, torch.complex128: 3}


class NullTrace:
    """A trace that records nothing (svdbench/laboratory/trace.py:38-43)."""
    enabled = False

    def wants(self, iteration=None):
        return False

    def stage(self, *args, **kwargs):
        return nullcontext()

    def checkpoint(self, *args, **kwargs):
        return None

    def record(self, *args, **kwargs):
        return None


def _schedule(n, device):
    """The laboratory's schedule (algorithms.py:121-126): rounds of the
    round-robin tournament on n + n % 2 players (primitives.py:309-313)
    without the pairs that reach past n, empty rounds left out; the index
    tensors p, q of each round."""
    np_ = n + n % 2
    players = list(range(np_))
    out = []
    for _ in range(np_ - 1):
        pairs = [(min(players[i], players[np_ - 1 - i]), max(players[i], players[np_ - 1 - i])) for i in range(np_ // 2)]
        players = [players[0]] + [players[-1]] + players[1:-1]
        pairs = [(p, q) for p, q in pairs if p < n and q < n]
        if pairs:
            out.append((torch.tensor([p for p, _ in pairs], device=device), torch.tensor([q for _, q in pairs],
                                                                                         device=device)))
    return out


def jacobi(a, trace=None, max_sweeps=40, tol=None, record_rotations=False, require_convergence=True, **unused):
    """One dense CUDA matrix (real or complex): (U, s, Vh) as the
    laboratory's jacobi returns them."""
    trace = trace if trace is not None else NullTrace()
    if a.ndim != 2 or a.layout != torch.strided or max_sweeps < 1:
        raise ValueError('Jacobi expects one dense matrix and positive max_sweeps')
    if a.device.type != 'cuda' or a.dtype not in _DTYPE:
        raise RuntimeError('the B200 laboratory Jacobi runs on CUDA float32/64 or complex64/128 matrices only')
    wide = a.shape[0] < a.shape[1]
    x = a.mH if wide else a
    scale = x.abs().max()
    scale = torch.where(scale > 0, scale, torch.ones_like(scale))
    w = (x / scale).resolve_conj().contiguous().clone()
    m, n = w.shape
    v = torch.eye(n, dtype=a.dtype, device=a.device)
    eps = torch.finfo(a.real.dtype).eps
    tol = 10 * eps if tol is None else tol
    if tol <= 0:
        raise ValueError('Tolerance must be positive')
    schedule = _schedule(n, a.device)
    rounds = n + n % 2 - 1 if len(schedule) else 0
    lib = N.lib()
    off = torch.zeros(1, dtype=torch.float64, device=a.device)
    stream = torch.cuda.current_stream(a.device).cuda_stream

    def run(r0, r1):
        N.check(lib.jb_jacobi_rounds(w.data_ptr(), v.data_ptr(), _DTYPE[a.dtype], m, n, r0, r1, float(tol),
                                     off.data_ptr(), stream), 'jb_jacobi_rounds')

    def factors():
        s = w.abs().square().sum(0).sqrt()
        order = s.argsort(descending=True)
        s, ww, vv = s[order], w[:, order], v[:, order]
        live = s > eps * max(m, n) * s[:1]
        u = ww / torch.where(live, s, torch.ones_like(s))
        from .solvers import _complete_null_columns
        u = _complete_null_columns(u[None], live[None])[0]
        s = torch.where(live, s, torch.zeros_like(s)) * scale
        return (vv, s, u.mH) if wide else (u, s, vv.mH)

    per_round = record_rotations or getattr(trace, 'enabled', True)
    converged = False
    sweep = 0
    with torch.no_grad():
        for sweep in range(1, max_sweeps + 1):
            off.zero_()
            if per_round:
                for index, (p, q) in enumerate(schedule):
                    with trace.stage('jacobi_rotation', sweep, round=index):
                        run(index, index + 1)
                    if record_rotations:
                        trace.checkpoint(f'rotation_{index}', sweep, tensors={'W': w, 'V': v, 'p': p, 'q': q})
            elif rounds:
                run(0, rounds)
            sweep_off = off[0].to(a.real.dtype)
            if trace.wants(sweep):
                trace.checkpoint('sweep', sweep, tensors={'W': w, 'V': v},
                                 scalars={'max_active_pair_correlation': sweep_off, 'tolerance': tol},
                                 factors=factors())
            if bool(sweep_off <= tol):
                converged = True
                break
        trace.record('convergence', converged=converged, sweeps=sweep, tolerance=tol)
        if not converged and require_convergence:
            raise RuntimeError(f'Jacobi did not converge in {max_sweeps} sweeps; inspect the saved trace')
        with trace.stage('sort_and_normalize'):
            result = factors()
        trace.checkpoint('final', factors=result)
    return result
