"""Benchmark of the batched one-sided Jacobi SVD on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload (one step): the uneven batch of 8192 float32 matrices, n ~ U{8..64},
m ~ U{n..2n}, entries N(0,1), seed 1, solved by ONE persistent launch
replayed from a captured CUDA graph, in the mixed precision that meets
sigma-rel-err <= 1e-5 against FP64 LAPACK (checked on rank 0 after timing).
The same batch is then timed in plain FP32 (the reference's arithmetic) for
the mixed / plain factor.

--gpus N (N > 1) without a torchrun environment starts N ranks itself (one
process per GPU, torch.distributed.run on 127.0.0.1).  --scaling weak (the
default): every rank solves its own batch of 8192 (rank r > 0 uses seed
1 + 1000 r: independent matrices, same distribution); --scaling strong: the
one seed-1 batch is split across the ranks by cost (batch.shard_by_cost).
No collective touches the data: the ranks share only barriers and the
max-over-ranks timing.
Metric: matrices/s (whole job).  Each step is timed with CUDA events on the
launching stream; a 256 MiB buffer is written between steps (outside the
events) so every step starts with a cold L2.

--workload selects one of the other configurations (one JSON line each):
  plain_single     256x128 f32, s_i = 10^(-4i/127), tol 1e-6, <= 30 sweeps
  clustered_large  4096x1024 f32, 64 clusters x 16, blocked Jacobi b = 32
  tall_lowrank     8192x2048 f32 rank 64 + noise, blocked Jacobi b = 64
  warm_family      65536 x 128x64 f32 family: network trained on 60000,
                   warm vs plain timed on 4096 held-out matrices
  extensions       the paths around the Jacobi kernels (complex Jacobi,
                   the QR-based solvers, gram_jacobi, jacobi_eigh, the
                   laboratory's traced Jacobi): one line each, with accuracy
                   against LAPACK and the NumPy oracle timed beside it

--impl reference: the reference algorithm's CPU implementation, timed on the
host cores of this machine on a bounded sample of the same workload: the C
restatement in oracle/ (all threads; the reference is Python, so nothing of
it compiles into a native library) gives the line's value, and the
reference's own svdbench.standalone.svd(x, 'jacobi') (PyTorch on CPU, all
threads, one call per matrix as a harness runs it; imported unchanged from
the install in baseline/_ref when present) is timed beside it.  Under
torchrun only rank 0 runs it.
"""
from __future__ import annotations

import argparse
import importlib
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "Jacobi SVD matrices/s at sigma-rel-err<=1e-5 vs FP64 (uneven batch)"
WORKLOAD = "uneven_batch_8192"
COUNT = 8192
# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) of one solve of
# this workload, the four launches of the two size classes (rb32_kernel_t
# 256- and 128-thread, rb64_kernel 512- and 256-thread), from one ncu capture
# (those metrics only) of `bench.py --steps 1 --warmup 3 --no-cpu-baseline`.
MEASURED_TRAFFIC_PER_SOLVE = 289.0e6
TRAFFIC_SOURCE = ("ncu dram__bytes_read.sum + dram__bytes_write.sum of the four solve launches of one step, "
                  "captured at the library of commit 013b917 (the FP32 and FP64 solve kernels unchanged since)")


MIXED = ("mixed (FP32 sweeps, then FP64 sweeps from the Newton-Schulz orthogonalised V, "
         "W = A V recomputed in FP64)")


def workload_config(n_gpus, scaling="weak", precision=MIXED):
    per_gpu = COUNT if scaling == "weak" else f"{COUNT} / {n_gpus}, split by cost (batch.shard_by_cost)"
    return {"workload": WORKLOAD, "matrices_per_gpu": per_gpu, "n_range": [8, 64], "m_range": "[n, 2n]",
            "dtype": "float32", "seed": 1, "tol": "10*eps32 (reference default)", "max_sweeps": 60,
            "precision": precision, "scaling_mode": scaling,
            "parallelism": f"dp{n_gpus} (independent matrices per GPU, no collective)",
            "l2": "256 MiB write between steps, outside the timed events"}


def load_matrices(rank, world=1, scaling="weak"):
    """This rank's matrices: its own seeded batch (weak scaling), or its
    cost-balanced share of the one seed-1 batch (strong scaling)."""
    wl = importlib.import_module("pavel-s_svd_b200.workloads")
    if scaling == "strong":
        B = importlib.import_module("pavel-s_svd_b200.batch")
        mats = wl.uneven_batch(COUNT, seed=1)
        m = np.array([a.shape[0] for a in mats])
        n = np.array([a.shape[1] for a in mats])
        return [mats[i] for i in B.shard_by_cost(m, n, world)[rank]]
    return wl.uneven_batch(COUNT, seed=1 if rank == 0 else 1 + 1000 * rank)


def rank_command(nprocs, script, argv, port):
    """The command that starts `nprocs` ranks of `script` on this node, one
    per GPU, rendezvous on 127.0.0.1."""
    return [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={nprocs}",
            "--master-addr=127.0.0.1", f"--master-port={port}", str(script), *argv]


def launch_ranks(nprocs, script, argv, timeout=None):
    """Run `script` as `nprocs` ranks and return their launcher's exit code."""
    import socket
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    return subprocess.run(rank_command(nprocs, script, argv, port), timeout=timeout).returncode


def cpu_model():
    try:
        for line in Path("/proc/cpuinfo").read_text().splitlines():
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return None


def reduce_max(x, device):
    """Max of x over the ranks of the default process group (x itself
    without one): every multi-GPU time is the slowest rank's."""
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    if dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def algorithmic(m, n):
    """Compulsory HBM bytes and FP work of one solve of the batch.
    bytes: read A, write U (m x k), S (k), Vh (k x n), descriptors (48 B) and
    status/sweeps (8 B) per matrix.  flop/sweep of one matrix on its tall view
    (mt x nt): nt(nt-1)/2 pairs x (12 mt + 6 nt)."""
    m = m.astype(np.int64); n = n.astype(np.int64)
    k = np.minimum(m, n)
    nbytes = int((4 * (m * n + m * k + k + k * n) + 48 + 8).sum())
    mt, nt = np.maximum(m, n), np.minimum(m, n)
    flop_per_sweep = nt * (nt - 1) // 2 * (12 * mt + 6 * nt)
    return nbytes, flop_per_sweep


class ClockSampler:
    """nvidia-smi samples during the timed region (every 200 ms)."""

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "samples": len(sm), "reasons": sorted(reasons)}


class NvmlClockSampler:
    """SM clock and clock-event reasons read through NVML every 5 ms on a
    background thread while the timed region runs (reads only).  Falls back
    to nvidia-smi (ClockSampler) when NVML is unavailable."""

    REASONS = (("hw_slowdown", 0x8), ("hw_thermal_slowdown", 0x40), ("sw_thermal_slowdown", 0x20),
               ("sw_power_cap", 0x4))

    def __init__(self, device, index):
        self.device, self.index = device, index
        self.samples, self.smax, self.fallback = [], None, None
        self._stop = threading.Event()

    def _handle(self, nv):
        import torch
        try:
            pr = torch.cuda.get_device_properties(self.device)
            bus = f"{pr.pci_domain_id:08x}:{pr.pci_bus_id:02x}:{pr.pci_device_id:02x}.0"
            return nv.nvmlDeviceGetHandleByPciBusId(bus)
        except Exception:
            return nv.nvmlDeviceGetHandleByIndex(self.index)

    def __enter__(self):
        try:
            import pynvml as nv
            nv.nvmlInit()
            self.nv, self.h = nv, self._handle(nv)
            self.smax = float(nv.nvmlDeviceGetMaxClockInfo(self.h, nv.NVML_CLOCK_SM))
        except Exception:
            self.fallback = ClockSampler(self.index).__enter__()
            return self
        self.thread = threading.Thread(target=self._poll, daemon=True)
        self.thread.start()
        return self

    def _poll(self):
        nv = self.nv
        while not self._stop.is_set():
            try:
                sm = float(nv.nvmlDeviceGetClockInfo(self.h, nv.NVML_CLOCK_SM))
                rs = int(nv.nvmlDeviceGetCurrentClocksEventReasons(self.h))
                self.samples.append((sm, rs))
            except Exception:
                pass
            self._stop.wait(0.005)

    def __exit__(self, *exc):
        if self.fallback is not None:
            return self.fallback.__exit__(*exc)
        self._stop.set()
        self.thread.join(timeout=2)
        try:
            self.nv.nvmlShutdown()
        except Exception:
            pass

    def summary(self):
        if self.fallback is not None:
            return self.fallback.summary()
        sm = [a for a, _ in self.samples]
        reasons = sorted({nm for _, r in self.samples for nm, bit in self.REASONS if r & bit})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": self.smax,
                "samples": len(sm), "reasons": reasons, "source": "nvml, every 5 ms"}


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def cpu_port_sample(mats, seconds=12.0, threads=0):
    """Time the C oracle on consecutive chunks of the workload until about
    `seconds` of wall time; returns (matrices/s, matrices solved, threads)."""
    from oracle import c_oracle
    B = importlib.import_module("pavel-s_svd_b200.batch")
    threads = threads or c_oracle.max_threads()
    done, elapsed, i = 0, 0.0, 0
    chunk = 256
    while elapsed < seconds and i < len(mats):
        part = mats[i:i + chunk]
        flat, m, n, a_off = B.pack(part)
        k = np.minimum(m, n)
        desc = np.zeros(len(part), B.DESC_DTYPE)
        desc["m"], desc["n"], desc["rank"], desc["a_off"] = m, n, k, a_off
        desc["u_off"], _ = B._aligned_offsets(m * k)
        desc["s_off"], _ = B._aligned_offsets(k)
        desc["v_off"], _ = B._aligned_offsets(k * n)
        t = time.perf_counter()
        c_oracle.svd_uneven(flat.numpy(), desc, threads=threads)
        elapsed += time.perf_counter() - t
        done += len(part)
        i += chunk
    return done / elapsed, done, threads, elapsed


def reference_pytorch_sample(mats, seconds=10.0):
    """Time the reference's own svd(x, 'jacobi') (svdbench.standalone,
    PyTorch on CPU, imported unchanged from the install in baseline/_ref)
    one call per matrix, as a harness loops over matrices of different
    shapes, on consecutive matrices of the workload for about `seconds`.
    Returns (matrices/s, matrices, threads, seconds) or None when the
    install is absent."""
    ref = ROOT / "baseline" / "_ref"
    if not (ref / "svdbench").is_dir():
        return None
    import torch
    if str(ref) not in sys.path:
        sys.path.insert(0, str(ref))
    from svdbench.standalone import svd as ref_svd
    threads = os.cpu_count() or 1
    torch.set_num_threads(threads)
    ref_svd(torch.from_numpy(mats[0]), 'jacobi')                       # warm-up
    done, t0 = 0, time.perf_counter()
    while done < len(mats) and time.perf_counter() - t0 < seconds:
        ref_svd(torch.from_numpy(mats[done]), 'jacobi')
        done += 1
    el = time.perf_counter() - t0
    return done / el, done, threads, el


def run_reference(args, rank, world):
    """The CPU reference arm: rank 0 times the oracle port (the line's value)
    and the reference's own PyTorch CPU Jacobi beside it; other ranks exit."""
    if rank != 0:
        return
    mats = load_matrices(0)
    per_step = []
    sample = 0
    threads = 0
    for step in range(args.warmup + args.steps):
        rate, done, threads, el = cpu_port_sample(mats, seconds=args.ref_seconds)
        if step >= args.warmup:
            per_step.append(rate)
            sample = done
    value = statistics.median(per_step)
    fp32 = "fp32 (the reference's FP32 Jacobi arithmetic, solvers.py:24-27)"
    line = {"metric": METRIC, "value": value, "unit": "matrices/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * sample / value, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded)",
            "config": workload_config(world, "weak", fp32), "impl": "reference",
            "cpu_baseline": {"value": value, "unit": "matrices/s", "cores": threads, "kind": "port",
                             "cpu": cpu_model(),
                             "sample": f"first {sample} matrices of the workload per step (~{args.ref_seconds:.0f} s),"
                                       " C restatement of the reference Jacobi (oracle/), fp32 as the reference"},
            "e2e": {"value": value, "unit": "matrices/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    if not args.no_reference_pytorch:
        got = reference_pytorch_sample(mats, seconds=args.ref_seconds)
        if got is None:
            line["reference_pytorch"] = {"unavailable": "baseline/_ref holds no install of the reference"}
        else:
            rate, done, thr, el = got
            line["reference_pytorch"] = {
                "value": rate, "unit": "matrices/s", "cores": thr, "kind": "reference", "cpu": cpu_model(),
                "sample": f"first {done} matrices of the workload ({el:.1f} s), svdbench.standalone.svd(x, "
                          "'jacobi') imported unchanged, one call per matrix (the reference batches only "
                          "equal shapes), torch.set_num_threads(all host threads)",
                "c_port_over_reference": value / rate}
    print(json.dumps(line), flush=True)


def measure_fp_peaks(dev):
    """FP32 (scalar and packed) and FP64 CUDA-core peaks of this GPU, TFLOP/s:
    jb_fma_loop (independent FMA chains, registers only), best of 3 runs
    timed with CUDA events."""
    import torch
    N = importlib.import_module("pavel-s_svd_b200.native")
    lib = N.lib()
    sink = torch.zeros(1 << 16, dtype=torch.float32, device=dev)
    blocks = torch.cuda.get_device_properties(dev).multi_processor_count * 8
    out = {}
    for mode, name, iters in ((0, "fp32_scalar_tflops", 40000), (1, "fp32_packed_tflops", 40000),
                              (2, "fp64_tflops", 8000)):
        best = float("inf")
        for _ in range(4):
            e0, e1 = _events()
            e0.record()
            N.check(lib.jb_fma_loop(mode, blocks, iters, sink.data_ptr(), torch.cuda.current_stream(dev).cuda_stream),
                    "jb_fma_loop")
            e1.record()
            torch.cuda.synchronize(dev)
            best = min(best, e0.elapsed_time(e1))
        out[name] = lib.jb_fma_loop_flops(blocks, iters) / (best / 1e3) / 1e12
    out["fp32_tflops"] = max(out["fp32_scalar_tflops"], out["fp32_packed_tflops"])
    out["how"] = ("jb_fma_loop: 8 CTAs x 256 threads per SM, 16 independent FMA chains per thread, best of 4 "
                  "CUDA-event timings")
    return out


def check_accuracy(plan, mats, limit=None):
    """Max relative sigma error vs FP64 LAPACK over values above 2x the
    reference cut, and the worst reconstruction error, on rank 0."""
    worst_sig, worst_rec = 0.0, 0.0
    S = plan.S.cpu().numpy()
    U = plan.U.cpu().numpy()
    Vh = plan.Vh.cpu().numpy()
    idx = range(len(mats)) if limit is None else range(0, len(mats), max(1, len(mats) // limit))
    for i in idx:
        a = mats[i].astype(np.float64)
        m, n = a.shape
        k = min(m, n)
        s = S[plan.s_off[i]:plan.s_off[i] + k].astype(np.float64)
        sr = np.linalg.svd(a, compute_uv=False)
        sel = sr > 2 * np.finfo(np.float32).eps * max(m, n) * sr[0]
        worst_sig = max(worst_sig, float(np.max(np.abs(s[sel] - sr[sel]) / sr[sel])))
        u = U[plan.u_off[i]:plan.u_off[i] + m * k].reshape(m, k).astype(np.float64)
        vh = Vh[plan.v_off[i]:plan.v_off[i] + k * n].reshape(k, n).astype(np.float64)
        worst_rec = max(worst_rec, float(np.linalg.norm(a - (u * s) @ vh) / np.linalg.norm(a)))
    return worst_sig, worst_rec


def time_replays(graph, flush, stream, steps):
    """CUDA-event times (ms) of `steps` graph replays, L2 flushed between them
    (outside the events)."""
    import torch
    times = []
    with _timed_range():
        for step in range(steps):
            flush.fill_(step & 0xff)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            graph.replay()
            e1.record(stream)
            times.append((e0, e1))
        torch.cuda.synchronize()
    return [a.elapsed_time(b) for a, b in times]


def run_ours(args, rank, world, local_rank):
    import torch
    import torch.distributed as dist
    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    pkg = importlib.import_module("pavel-s_svd_b200")
    B = importlib.import_module("pavel-s_svd_b200.batch")
    mats = load_matrices(rank, world, args.scaling)
    total = COUNT * world if args.scaling == "weak" else COUNT
    flat_host, m, n, a_off = B.pack(mats)
    flat = flat_host.to(dev)
    # launch choices picked by the autotuner on this batch, in preparation (outside every timed region)
    choice, tune_ms = B.tune(m, n, flat, precision=args.precision)
    plan = B.UnevenBatch(m, n, dev, a_off=a_off, precision=args.precision, launch=choice)
    nbytes, flop_per_sweep = algorithmic(m, n)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    stream = torch.cuda.current_stream(dev)
    graph = plan.capture(flat)
    for _ in range(args.warmup):
        flush.fill_(1)
        graph.replay()
    torch.cuda.synchronize(dev)
    sweeps = plan.check()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize(dev)
    with NvmlClockSampler(dev, local_rank) as clocks:
        step_ms = time_replays(graph, flush, stream, args.steps)
    if world > 1:
        dist.barrier()
    total_ms = reduce_max(sum(step_ms), dev)
    ms_per_step = total_ms / args.steps
    value = total / (ms_per_step / 1e3)

    # End to end through the public host-to-host API (batch.StreamedUneven):
    # pinned host input -> device, solve, U/S/Vh and status -> pinned host,
    # status checked (check() synchronises and raises on any failed matrix),
    # all inside the timed region; the batch runs in 8 chunks (small first
    # and last ones) on two compute streams so that the copies of one chunk
    # overlap the solve of another.
    streamed = B.StreamedUneven(m, n, dev, chunks=8, precision=args.precision, launch=choice)
    host_in, host_u, host_s, host_v = streamed.host_buffers()
    host_in.copy_(flat_host[:host_in.numel()])
    h2d, d2h = streamed.device_bytes_per_run()

    def e2e_step():
        streamed.run(host_in, host_u, host_s, host_v)
        streamed.check()

    for _ in range(args.warmup):
        e2e_step()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize(dev)
    e2e_ev = []
    for _ in range(args.steps):
        flush.fill_(3)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        e2e_step()
        e1.record(stream)
        e2e_ev.append((e0, e1))
    torch.cuda.synchronize(dev)
    e2e_ms = reduce_max(sum(a.elapsed_time(b) for a, b in e2e_ev), dev)
    e2e_value = total / (e2e_ms / args.steps / 1e3)
    # the host-to-host result equals the device solve's (same kernels per matrix)
    e2e_same = bool(torch.equal(host_s[:plan.S.numel()], plan.S.cpu()))

    if rank != 0:
        return
    graph.replay()
    torch.cuda.synchronize(dev)
    sweeps = plan.check()
    sig_err, rec_err = check_accuracy(plan, mats, limit=None if args.full_check else 2048)
    hbm_peak, peak_kind = peaks()
    achieved_gbs = nbytes / (ms_per_step / 1e3) / 1e9
    flop = float((flop_per_sweep * sweeps).sum())
    fp_tflops = flop / (ms_per_step / 1e3) / 1e12
    fp_peaks = measure_fp_peaks(dev)
    del graph
    # The same batch in plain FP32 (the reference's arithmetic, V = I start,
    # its tolerance), timed the same way on this GPU: the mixed / plain factor.
    plain = None
    if args.precision == "mixed":
        p32 = B.UnevenBatch(m, n, dev, a_off=a_off, precision="fp32")
        g32 = p32.capture(flat)
        for _ in range(args.warmup):
            flush.fill_(1)
            g32.replay()
        ms32 = statistics.mean(time_replays(g32, flush, stream, args.steps))
        sw32 = p32.check()
        err32, rec32 = check_accuracy(p32, mats, limit=2048)
        rate32 = len(mats) / (ms32 / 1e3)
        plain = {"matrices_per_s_this_gpu": rate32, "ms_per_step": ms32, "sweeps_mean": float(sw32.mean()),
                 "max_rel_sigma_err_vs_fp64": err32, "max_reconstruction_rel_fro": rec32,
                 "meets_1e-5": bool(err32 <= 1e-5), "matrices_checked": 2048,
                 "mixed_over_plain_fp32": (len(mats) / (ms_per_step / 1e3)) / rate32,
                 "note": "plain FP32 one-sided Jacobi (precision='fp32', the reference's arithmetic) on the same "
                         "batch and GPU, graph replays timed like the headline"}
        del g32
    line = {"metric": METRIC, "value": value, "unit": "matrices/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": args.scaling,
            "vs_baseline": None, "dtype": "f32 in/out; f32+f64 sweeps" if args.precision == "mixed" else "f32",
            "data": "synthetic (seeded: n ~ U[8,64], m ~ U[n,2n], entries N(0,1))",
            "config": dict(workload_config(world, args.scaling, MIXED if args.precision == "mixed" else "fp32"),
                           launch=repr(choice), autotuner_ms={k: round(v, 3) for k, v in tune_ms.items()}),
            "accuracy": {"max_rel_sigma_err_vs_fp64": sig_err, "max_reconstruction_rel_fro": rec_err,
                         "matrices_checked": len(mats) if args.full_check else 2048,
                         "sweeps_mean": float(sweeps.mean()), "sweeps_max": int(sweeps.max())},
            "plain_fp32": plain,
            "roofline": {"bound": "hbm", "achieved": achieved_gbs, "peak": hbm_peak, "unit": "GB/s",
                         "frac": achieved_gbs / hbm_peak, "peak_kind": peak_kind,
                         "traffic": args.traffic_bytes if args.traffic_bytes is not None else
                         MEASURED_TRAFFIC_PER_SOLVE,
                         "traffic_source": TRAFFIC_SOURCE,
                         "algorithmic_bytes_per_launch": nbytes,
                         "note": "compulsory bytes only; the path is bound by the FP32/FP64 pipes, see fp_pipe"},
            "fp_pipe": {"achieved_tflops": fp_tflops, "flop_per_launch": flop,
                        "measured_peaks": fp_peaks,
                        "frac_of_measured_fp32": fp_tflops / fp_peaks["fp32_tflops"],
                        "note": "algorithmic flop = sum over matrices of sweeps x nt(nt-1)/2 (12 mt + 6 nt), FP32 "
                                "and FP64 sweeps together, against the measured FP32 peak"},
            "clocks": clocks.summary(), "gpu_launches": args.steps * plan.kernels_per_solve,
            "e2e": {"value": e2e_value, "unit": "matrices/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "api": "batch.StreamedUneven (8 chunks of cost 1:2:4:4:4:4:2:1, two compute streams, copies overlapped "
                           "with the solve)",
                    "singular_values_equal_device_solve": e2e_same}}
    if not args.no_cpu_baseline:
        rate, done, threads, el = cpu_port_sample(mats, seconds=args.ref_seconds)
        line["cpu_baseline"] = {"value": rate, "unit": "matrices/s", "cores": threads, "kind": "port",
                                "cpu": cpu_model(),
                                "sample": f"first {done} of the 8192 matrices ({el:.1f} s), C restatement of the "
                                          "reference Jacobi (oracle/), fp32 like the reference"}
    print(json.dumps(line), flush=True)


def _events():
    import torch
    return torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)


class _timed_range:
    """NVTX push/pop range "timed" around a timed region, so a profiler's
    launch list can be restricted to it (ncu --nvtx --nvtx-include timed/)."""

    def __enter__(self):
        import torch
        torch.cuda.nvtx.range_push("timed")

    def __exit__(self, *exc):
        import torch
        torch.cuda.nvtx.range_pop()


def lapack_check(a, U, S, Vh, cut_width):
    """Accuracy against FP64 LAPACK of the same float32 input; 'resolved'
    values are those above twice the reference cut eps32 * cut_width * sigma_1."""
    import scipy.linalg
    a64 = a.astype(np.float64)
    sr = scipy.linalg.svd(a64, compute_uv=False, lapack_driver="gesdd")
    s = S.cpu().numpy().astype(np.float64)
    k = len(s)
    cut = np.finfo(np.float32).eps * cut_width * sr[0]
    res = sr[:k] > 2 * cut
    big = sr[:k] >= 0.1 * sr[0]
    out = {"spectrum_error_over_sigma1": float(np.abs(s - sr[:k]).max() / sr[0]),
           "resolved_spectrum_max_relative_error": float(np.max(np.abs(s[res] - sr[:k][res]) / sr[:k][res])),
           "max_relative_error_sigma_ge_0.1_sigma1": float(np.max(np.abs(s[big] - sr[:k][big]) / sr[:k][big])),
           "resolved_values": int(res.sum())}
    if U is not None:
        u = U.cpu().numpy().astype(np.float64)
        vh = Vh.cpu().numpy().astype(np.float64)
        keep = s > 0
        out["orthogonality_u_max"] = float(np.abs(u[:, keep].T @ u[:, keep] - np.eye(keep.sum())).max())
        out["orthogonality_v_max"] = float(np.abs(vh @ vh.T - np.eye(vh.shape[0])).max())
        out["reconstruction_relative_fro"] = float(np.linalg.norm(a64 - (u[:, keep] * s[keep]) @ vh[keep]) /
                                                   np.linalg.norm(a64))
    return out


def run_plain_single(args):
    import torch
    S_ = importlib.import_module("pavel-s_svd_b200.solvers")
    wl = importlib.import_module("pavel-s_svd_b200.workloads")
    a_np = wl.plain_single()
    a = torch.from_numpy(a_np).cuda()
    res = {}
    for prec in ("fp32", "mixed"):
        x = a[None].contiguous()
        out = (torch.empty(1, 256, 128, device="cuda"), torch.empty(1, 128, device="cuda"),
               torch.empty(1, 128, 128, device="cuda"))
        info = torch.empty(2, 1, dtype=torch.int32, device="cuda")
        ws = S_.Workspace()
        run = lambda: S_.launch_batched(x, 128, 0, 1e-6, 30, prec, out, info, ws)
        for _ in range(args.warmup):
            run()
        torch.cuda.synchronize()
        e0, e1 = _events()
        e0.record()
        for _ in range(args.steps):
            run()
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / args.steps
        acc = lapack_check(a_np, out[0][0], out[1][0], out[2][0], 256)
        res[prec] = {"ms": ms, "matrices_per_s": 1e3 / ms, "sweeps": int(info[0, 0]), **acc}
    from oracle import c_oracle
    t = time.perf_counter()
    _, so, _, swo, _ = c_oracle.svd_batched(a_np[None], tol=1e-6, max_sweeps=30, threads=1)
    cpu_ms = (time.perf_counter() - t) * 1e3
    line = {"metric": "Jacobi SVD matrices/s (single 256x128 matrix)", "value": res["mixed"]["matrices_per_s"],
            "unit": "matrices/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": res["mixed"]["ms"], "higher_is_better": True, "scaling": "none (single matrix)",
            "vs_baseline": None, "dtype": "f32 in/out", "data": "synthetic (seeded: Haar U, V; s_i = 10^(-4i/127))",
            "config": {"workload": "plain_single_256x128", "tol": 1e-6, "max_sweeps": 30},
            "variants": res, "cpu_baseline": {"value": 1e3 / cpu_ms, "unit": "matrices/s", "cores": 1,
                                              "kind": "port", "sample": "the one matrix, C oracle (fp32)",
                                              "sweeps": int(swo[0])}}
    print(json.dumps(line), flush=True)


def cpu_sweep_sample(a_np, width):
    """CPU cost of one sweep of the plain one-sided Jacobi on a (the C
    restatement of the reference's jacobi_svd, oracle/): disjoint blocks of
    `width` columns, one per host thread, each run for one sweep at once; a
    sweep's pairs are independent within a round, so the full sweep on the
    same threads is extrapolated as (pairs of a) / (pairs of a block) x the
    wall time / the blocks run side by side.  Returns (seconds per sweep,
    threads, wall seconds, blocks)."""
    from oracle import c_oracle
    m, n = a_np.shape
    threads = c_oracle.max_threads()
    blocks = max(1, min(threads, n // width))
    sub = np.stack([a_np[:, k * width:(k + 1) * width] for k in range(blocks)])
    t = time.perf_counter()
    c_oracle.svd_batched(sub, values_only=True, max_sweeps=1, threads=blocks)
    wall = time.perf_counter() - t
    per_sweep = wall * (n * (n - 1)) / (width * (width - 1)) / blocks
    return per_sweep, blocks, wall, blocks


def run_blocked(args, name):
    import torch
    wl = importlib.import_module("pavel-s_svd_b200.workloads")
    BJ = importlib.import_module("pavel-s_svd_b200.blocked")
    if name == "clustered_large":
        a_np, b = wl.clustered_large(), 32
    else:
        a_np, b = wl.tall_lowrank(), 64
    m, n = a_np.shape
    a = torch.from_numpy(a_np).cuda()
    plan = BJ.BlockJacobi(m, n, b)
    tune_ms = plan.tune(a)                               # launch choices, in preparation
    for _ in range(max(args.warmup, 2)):               # eager first sweeps, then the sweep graphs captured
        U, S, Vh, info = plan.solve(a)
    torch.cuda.synchronize()
    times = []
    with _timed_range():
        for _ in range(args.steps):
            e0, e1 = _events()
            e0.record()
            U, S, Vh, info = plan.solve(a, use_graphs=not args.eager)
            e1.record()
            torch.cuda.synchronize()
            times.append(e0.elapsed_time(e1))
    ms = float(np.median(times))
    R, P, mp, npd = plan.nb - 1, plan.P, plan.mpad, plan.npad
    per_round = P * (2 * mp * (2 * b) ** 2 * 2 + 2 * npd * (2 * b) ** 2)       # Gram + W and V updates
    terms = [3 if p == 2 else 6 for _, p in info["off_per_sweep"]]
    # the sweeps' Gram and update products, and the post-sweep Gram of the whole W
    tensor_flop = sum(R * per_round * t + 2 * npd * npd * mp * t for t in terms)
    # outside the sweeps, all six-term: Newton-Schulz steps on V (two npad^3
    # products each), W = A V on the tensor cores, the two products of U's
    # re-orthogonalisation (kept columns rounded up to 8)
    r8 = -(-info["kept_columns"] // 8) * 8 if info["kept_columns"] > 1 else 0
    tensor_flop += 6 * (info["polar_steps"] * 2 * 2 * npd ** 3 + info["tensor_w_products"] * 2 * npd * mp * npd
                        + 2 * 2 * r8 * r8 * mp)
    acc = lapack_check(a_np, U, S, Vh, max(m, n))
    line = {"metric": f"blocked Jacobi SVD matrices/s ({m}x{n}, b={b})", "value": 1e3 / ms, "unit": "matrices/s",
            "n_gpus": 1, "steps": args.steps, "warmup": max(args.warmup, 2), "ms_per_step": ms,
            "higher_is_better": True,
            "scaling": "none (single matrix)", "vs_baseline": None,
            "dtype": "f32 in/out; bf16x3/bf16x6 tensor; " + "/".join(sorted({x.lower() for x in info["eig_precision"]}))
                     + " eig",
            "config": {"workload": name, "m": m, "n": n, "block_size": b,
                       "launch": {"eig_cols_per_warp": plan.eig_variant, "gram_split": plan.gram_split,
                                  "schedule": plan.schedule, "slot_split": plan.slot_split,
                                  "eig_fp32_two_part": plan.eig_fp32_two_part, "eig_defer_q": plan.eig_defer_q},
                       "autotuner_ms_per_sweep": {k: round(v, 3) for k, v in tune_ms.items()}},
            "data": ("synthetic (seeded: Haar U, V; 64 clusters x 16, cond 1e6)" if name == "clustered_large"
                     else "synthetic (seeded: rank-64 Gaussian product + N(0, 1e-6) noise)"),
            "block_sweeps": info["block_sweeps"], "off_per_sweep": info["off_per_sweep"],
            "post_sweep_off": info["post_sweep_off"],
            "converged": info["converged"], "reached_tol": info["reached_tol"],
            "tensor_flop_per_solve": tensor_flop, "tensor_tflops_whole_solve": tensor_flop / (ms / 1e3) / 1e12,
            "accuracy": acc}
    pk = json.loads((ROOT / "MEASURED_PEAKS.json").read_text()) if (ROOT / "MEASURED_PEAKS.json").exists() else {}
    peak, kind = (float(pk["bf16_tflops_sustained"]), "measured sustained") if "bf16_tflops_sustained" in pk \
        else (1400.0, "fallback sustained")
    achieved = tensor_flop / (ms / 1e3) / 1e12
    line["roofline"] = {"bound": "tensor", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                        "frac": achieved / peak, "peak_kind": kind, "traffic": None,
                        "note": "tensor flops over the whole solve (every BF16 term counted): the sweeps' Gram and "
                                "update products, the post-sweep Grams, the Newton-Schulz steps, W = A V where it "
                                "runs on the tensor cores, U's re-orthogonalisation; the solve is bound by the "
                                "16-slot eigen-solves that set each round's pace"}
    if not args.no_plain:
        # the plain FP32 CUDA path at the same shape: the reference's block
        # rounds (solvers.py:30-68), every pair's inner one-sided Jacobi in
        # FP32 on the CUDA cores (pair QR first), updates as FP32 GEMMs
        S_ = importlib.import_module("pavel-s_svd_b200.solvers")
        e0, e1 = _events()
        torch.cuda.synchronize()
        e0.record()
        try:
            u2, s2, vh2, st2 = S_._composed_svd(a[None], "block_jacobi", False, False, True, n,
                                                {"block_size": b, "precision": "fp32"})
            e1.record()
            torch.cuda.synchronize()
            pms = e0.elapsed_time(e1)
            acc2 = lapack_check(a_np, u2[0], s2[0], vh2[0], max(m, n))
            line["plain_fp32"] = {
                "matrices_per_s": 1e3 / pms, "ms": pms, "block_sweeps": st2.get("block_sweeps"),
                "inner_jacobi_sweeps_max": st2.get("jacobi_sweeps"), "accuracy": acc2,
                "meets_1e-5": bool(acc2["resolved_spectrum_max_relative_error"] <= 1e-5),
                "tensor_over_plain_fp32": pms / ms,
                "note": "svd(a, 'block_jacobi', block_size=b) through the block rounds with precision='fp32': "
                        "the reference's algorithm on this library's FP32 CUDA-core kernels, one call"}
        except RuntimeError as err:
            torch.cuda.synchronize()
            line["plain_fp32"] = {"failed": str(err)}
    if not args.no_cpu_baseline:
        per_sweep, thr, wall, blocks = cpu_sweep_sample(a_np, 128)
        k = line.get("plain_fp32", {}).get("block_sweeps") or info["block_sweeps"]
        line["cpu_baseline"] = {
            "value": 1.0 / (per_sweep * k), "unit": "matrices/s", "cores": thr, "kind": "port", "cpu": cpu_model(),
            "seconds_per_sweep_extrapolated": per_sweep,
            "sample": f"one sweep of the plain one-sided Jacobi (C restatement) on {blocks} disjoint {m}x128 column "
                      f"blocks at once ({wall:.1f} s), extrapolated by pair count to one sweep of the whole matrix, "
                      f"times {k} sweeps (the block sweeps of the plain FP32 path; a block sweep of the reference "
                      f"does at least one sweep's work, so this overstates the CPU's throughput)"}
    print(json.dumps(line), flush=True)


def run_warm(args):
    import torch
    W = importlib.import_module("pavel-s_svd_b200.warmstart")
    wl = importlib.import_module("pavel-s_svd_b200.workloads")
    a_np, theta = wl.warm_family(count=65536, device="cuda")
    a = torch.from_numpy(a_np).cuda()
    tr, te = a[:60000].contiguous(), a[60000:64096].contiguous()
    e0, e1 = _events()
    e0.record()
    v_tr, _ = W.plain_v(tr)
    net = W.WarmStartMLP(seed=0)
    hist = W.train(net, tr, v_tr, epochs=15, batch=512, lr=1e-3, order="assign")
    e1.record()
    torch.cuda.synchronize()
    train_ms = e0.elapsed_time(e1)
    solver = W.WarmSolver(net, m=128, n=64, batch=4096)
    solver32 = W.WarmSolver(net, m=128, n=64, batch=4096, precision="fp32")
    eye = torch.eye(64, device="cuda").expand(4096, 64, 64).contiguous()
    ideal = wl.family_v(theta[60000:64096], device="cuda").contiguous()
    res = {}
    # plain_fp32 / plain: the Jacobi alone from V = I (the plain solvers);
    # warm: sketch -> network -> in-kernel QR and fallback test -> Jacobi;
    # identity_through_pipeline: V0 = I through the QR preparation and the
    # Jacobi (the warm path's cost without the network); ideal_start: the
    # generator's own V(theta) through the same preparation, and ideal_solve
    # the Jacobi alone from it (what a perfect network with a free start gives)
    variants = (("plain_fp32", eye, True), ("plain", eye, True), ("warm", None, False),
                ("identity_through_pipeline", eye, False), ("ideal_start", ideal, False), ("ideal_solve", ideal, True))
    for label, v0, direct in variants:
        solver = solver32 if label == "plain_fp32" else W.WarmSolver(net, m=128, n=64, batch=4096)
        run = (lambda: solver.solve_from(te, v0)) if direct else (lambda: solver.launch(te, v0=v0))
        for _ in range(args.warmup):
            run()
        torch.cuda.synchronize()
        e0, e1 = _events()
        e0.record()
        for _ in range(args.steps):
            run()
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / args.steps
        sweeps, used = solver.check()
        worst = 0.0
        S = solver.S.cpu().numpy()
        for i in range(0, 4096, 64):
            sr = np.linalg.svd(te[i].cpu().numpy().astype(np.float64), compute_uv=False)
            worst = max(worst, float(np.max(np.abs(S[i] - sr) / sr)))
        res[label] = {"ms": ms, "matrices_per_s": 4096 / (ms / 1e3), "sweeps_mean": float(sweeps.mean()),
                      "kept": float(used.mean()), "max_rel_sigma_err_vs_fp64_sample": worst}
    # the warm path's parts, each timed alone
    x = W.sketch(te)
    v0n = net.predict_v0(te).contiguous()
    sol = W.WarmSolver(net, m=128, n=64, batch=4096)
    lib = importlib.import_module("pavel-s_svd_b200.native").lib()
    st = torch.cuda.current_stream().cuda_stream

    def prep():
        lib.jb_warm_prep_f32(te.data_ptr(), v0n.data_ptr(), sol.vstart.data_ptr(), sol.used.data_ptr(),
                             sol.off[0].data_ptr(), sol.off[1].data_ptr(), 4096, 128, 64, st)
    parts = {"sketch": _time_gpu(lambda: W.sketch(te), args.steps, args.warmup),
             "network": _time_gpu(lambda: net.forward(x), args.steps, args.warmup),
             "qr_and_fallback_prep": _time_gpu(prep, args.steps, args.warmup)}
    prep()
    vs = sol.vstart.transpose(-1, -2).contiguous()     # back to launch's layout (vectors as columns)
    parts["jacobi_from_prepared_start"] = _time_gpu(lambda: sol.solve_from(te, vs), args.steps, args.warmup)
    line = {"metric": "Jacobi SVD matrices/s, learned warm start vs plain (128x64 family, 4096 held-out)",
            "value": res["warm"]["matrices_per_s"], "unit": "matrices/s", "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": res["warm"]["ms"], "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32 in/out; f32+f64 sweeps; bf16 network",
            "data": "synthetic (seeded: U Haar, log-uniform s, V = expm(0.3 L(theta)))", "config": {"workload": "warm_family", "train": 60000,
                                                                         "held_out": 4096, "epochs": 15},
            "train_ms": train_ms, "loss_first_last": [hist[0], hist[-1]], "variants": res,
            "warm_over_plain": res["warm"]["matrices_per_s"] / res["plain"]["matrices_per_s"],
            "warm_parts_ms": parts,
            "note": "plain_fp32 / plain = the plain FP32 / mixed-precision Jacobi from V = I alone; warm = sketch, "
                    "network, in-kernel Householder QR of V0 with the identity fallback test, then the Jacobi; "
                    "identity_through_pipeline = V0 = I through that QR preparation; ideal_start / ideal_solve = "
                    "the generator's own V(theta) with / without the preparation: what a perfect network would give"}
    print(json.dumps(line), flush=True)


def _time_gpu(fn, steps, warmup):
    """Median ms of fn() over `steps` runs, each bracketed by CUDA events on
    the current stream, a 256 MiB write between runs (outside the events)."""
    import torch
    flush = torch.empty(64 << 20, dtype=torch.float32, device="cuda")
    for _ in range(warmup):
        fn()
    torch.cuda.synchronize()
    times = []
    for i in range(steps):
        flush.fill_(i & 0xff)
        e0, e1 = _events()
        e0.record()
        fn()
        e1.record()
        torch.cuda.synchronize()
        times.append(e0.elapsed_time(e1))
    return statistics.median(times)


def _time_cpu(fn, count, seconds=3.0):
    """Matrices/s of fn() (which solves `count` matrices) over about
    `seconds` of wall time, at least once."""
    t0 = time.perf_counter()
    runs = 0
    while True:
        fn()
        runs += 1
        el = time.perf_counter() - t0
        if el >= seconds:
            return runs * count / el


def run_extensions(args):
    """One line per path around the Jacobi kernels, on seeded synthetic
    batches: the device time of the public call (inputs resident), the
    largest relative sigma error against FP64 LAPACK on the batch, and the
    NumPy oracle (the reference's algorithm restated, one host thread) on a
    sample of the same batch."""
    import torch
    pkg = importlib.import_module("pavel-s_svd_b200")
    eigh = importlib.import_module("pavel-s_svd_b200.eigh")
    qrm = importlib.import_module("pavel-s_svd_b200.qr")
    lab = importlib.import_module("pavel-s_svd_b200.lab")
    from oracle import jacobi_oracle as O
    rng = np.random.default_rng(61)

    def sig_err(a, s, k=None):
        a64 = a.astype(np.complex128 if np.iscomplexobj(a) else np.float64)
        sr = np.linalg.svd(a64, compute_uv=False)
        k = k or s.shape[-1]
        s = np.asarray(s, np.float64)[..., :k]
        return float((np.abs(s - sr[..., :k]) / sr[..., :1]).max())

    def line(row, a_np, ms, acc, cpu_rate, cpu_sample, config, dtype):
        b = a_np.shape[0]
        print(json.dumps({"metric": f"{row} matrices/s", "value": b / (ms / 1e3), "unit": "matrices/s",
                          "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
                          "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": dtype,
                          "data": "synthetic (seeded: N(0,1) entries; the projected solvers s_i = 0.8^i)",
                          "config": dict(workload=row, **config),
                          "accuracy": acc, "cpu_baseline": {"value": cpu_rate, "unit": "matrices/s", "cores": 1,
                                                            "kind": "port", "sample": cpu_sample}}), flush=True)

    # complex Jacobi
    for dt, tdt in ((np.complex64, torch.complex64), (np.complex128, torch.complex128)):
        a = (rng.standard_normal((1024, 48, 32)) + 1j * rng.standard_normal((1024, 48, 32))).astype(dt)
        t = torch.from_numpy(a).cuda()
        ms = _time_gpu(lambda: pkg.svd(t, "jacobi"), args.steps, args.warmup)
        _, s, _ = pkg.svd(t, "jacobi")
        cpu = _time_cpu(lambda: O.svd(a[:8], "jacobi"), 8)
        line(f"complex Jacobi {np.dtype(dt).name}", a, ms, {"max_rel_sigma_err_vs_lapack": sig_err(a, s.cpu().numpy())},
             cpu, "8 matrices, NumPy oracle jacobi_svd", {"shape": [1024, 48, 32]}, np.dtype(dt).name)
    # QR-based solvers
    # the projected solvers approximate the leading triplets: inputs with a
    # decaying spectrum (s_i = 0.8^i, Haar-like factors) where that is meaningful
    uu = np.linalg.qr(rng.standard_normal((256, 256, 96)))[0]
    vv = np.linalg.qr(rng.standard_normal((256, 96, 96)))[0]
    decaying = (uu * 0.8 ** np.arange(96)) @ np.swapaxes(vv, 1, 2)
    cases = (("qr", rng.standard_normal((1024, 96, 32)).astype(np.float32), {}),
             ("tsqr", rng.standard_normal((128, 1024, 32)), {"tile_rows": 128}),
             ("randomized", decaying, {"rank": 8, "iterations": 2}),
             ("block_krylov", decaying, {"rank": 8, "iterations": 2}))
    for alg, a, kw in cases:
        t = torch.from_numpy(a).cuda()
        ms = _time_gpu(lambda: pkg.svd(t, alg, **kw), args.steps, args.warmup)
        _, s, _ = pkg.svd(t, alg, **kw)
        k = kw.get("rank")
        okw = dict(kw)
        if alg in ("randomized", "block_krylov"):
            ell = min(k + 8, min(a.shape[-2:]))
            okw["initial_basis"] = rng.standard_normal((4, a.shape[-1], ell)).astype(a.dtype)
        cpu = _time_cpu(lambda: O.svd(a[:4], alg, **okw), 4)
        line(f"svd '{alg}'", a, ms, {"max_rel_sigma_err_vs_lapack": sig_err(a, s.cpu().numpy(), k)}, cpu,
             "4 matrices, NumPy oracle", {"shape": list(a.shape), **kw}, a.dtype.name)
    # the QR kernel alone
    a = rng.standard_normal((1024, 128, 64)).astype(np.float32)
    t = torch.from_numpy(a).cuda()
    ms = _time_gpu(lambda: qrm.qr(t), args.steps, args.warmup)
    q, r = qrm.qr(t)
    q64, r64 = q.cpu().numpy().astype(np.float64), r.cpu().numpy().astype(np.float64)
    acc = {"max_abs_QR_minus_A": float(np.abs(q64 @ r64 - a).max()),
           "max_abs_QtQ_minus_I": float(np.abs(np.swapaxes(q64, 1, 2) @ q64 - np.eye(64)).max())}
    cpu = _time_cpu(lambda: O.qr(a[:16]), 16)
    line("Householder QR (jb_qr_f32)", a, ms, acc, cpu, "16 matrices, NumPy oracle qr", {"shape": [1024, 128, 64]},
         "float32")
    # gram_jacobi and jacobi_eigh
    a = rng.standard_normal((1024, 64, 32))
    t = torch.from_numpy(a).cuda()
    ms = _time_gpu(lambda: pkg.svd(t, "gram_jacobi"), args.steps, args.warmup)
    _, s, _ = pkg.svd(t, "gram_jacobi")
    g = np.swapaxes(a, 1, 2) @ a
    cpu = _time_cpu(lambda: O.jacobi_eigh(g[:8]), 8)
    line("svd 'gram_jacobi'", a, ms, {"max_rel_sigma_err_vs_lapack": sig_err(a, s.cpu().numpy())}, cpu,
         "8 Grams, NumPy oracle jacobi_eigh", {"shape": [1024, 64, 32]}, "float64")
    h = torch.from_numpy(g).cuda()
    ms = _time_gpu(lambda: eigh.jacobi_eigh(h), args.steps, args.warmup)
    w, _, _ = eigh.jacobi_eigh(h)
    wr = np.linalg.eigvalsh(g)
    line("jacobi_eigh", g, ms, {"max_rel_eig_err_vs_lapack": float((np.abs(w.cpu().numpy() - wr) /
                                                                     np.abs(wr).max(-1, keepdims=True)).max())},
         cpu, "8 matrices, NumPy oracle jacobi_eigh", {"shape": [1024, 32, 32]}, "float64")
    # block_jacobi in rounds (float64 and complex input): one batched Jacobi
    # call per round of the block tournament
    for dt in (np.float64, np.complex64):
        a = rng.standard_normal((256, 96, 64))
        if dt == np.complex64:
            a = a + 1j * rng.standard_normal((256, 96, 64))
        a = a.astype(dt)
        t = torch.from_numpy(a).cuda()
        ms = _time_gpu(lambda: pkg.svd(t, "block_jacobi", block_size=8), args.steps, args.warmup)
        _, s, _ = pkg.svd(t, "block_jacobi", block_size=8)
        cpu = _time_cpu(lambda: O.svd(a[:2], "block_jacobi", block_size=8), 2)
        line(f"svd 'block_jacobi' rounds {np.dtype(dt).name}", a, ms,
             {"max_rel_sigma_err_vs_lapack": sig_err(a, s.cpu().numpy())}, cpu, "2 matrices, NumPy oracle",
             {"shape": [256, 96, 64], "block_size": 8}, np.dtype(dt).name)
    # the laboratory's Jacobi (one matrix, no trace: a sweep per launch)
    a = rng.standard_normal((1, 128, 64))
    t = torch.from_numpy(a[0]).cuda()
    ms = _time_gpu(lambda: lab.jacobi(t), args.steps, args.warmup)
    _, s, _ = lab.jacobi(t)
    cpu = _time_cpu(lambda: O.svd(a, "jacobi"), 1)
    line("laboratory jacobi (one matrix)", a, ms, {"max_rel_sigma_err_vs_lapack": sig_err(a, s.cpu().numpy()[None])},
         cpu, "the one matrix, NumPy oracle jacobi_svd", {"shape": [128, 64]}, "float64")


def main():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=("ours", "reference"), default="ours")
    ap.add_argument("--workload", choices=("uneven_batch", "plain_single", "clustered_large", "tall_lowrank",
                                           "warm_family", "extensions"), default="uneven_batch")
    ap.add_argument("--precision", choices=("mixed", "fp32"), default="mixed")
    ap.add_argument("--scaling", choices=("weak", "strong"), default="weak",
                    help="weak: a batch of 8192 per GPU; strong: one batch of 8192 split across the GPUs by cost")
    ap.add_argument("--no-reference-pytorch", action="store_true",
                    help="reference arm: skip timing the reference's own PyTorch CPU Jacobi")
    ap.add_argument("--ref-seconds", type=float, default=12.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-plain", action="store_true",
                    help="blocked workloads: skip the plain FP32 CUDA block-rounds comparison")
    ap.add_argument("--eager", action="store_true",
                    help="blocked workloads: launch the timed solve's kernels one by one instead of replaying the "
                         "captured sweep graphs (for a profiler's launch list; the line is then no bench number)")
    ap.add_argument("--full-check", action="store_true")
    ap.add_argument("--traffic-bytes", type=float, default=None,
                    help="per-launch DRAM bytes from an ncu capture, reported as roofline.traffic")
    args = ap.parse_args()
    if args.warmup < 3:
        ap.error("at least 3 warm-up steps")
    if "WORLD_SIZE" not in os.environ and args.gpus > 1:
        # one process per GPU: start the ranks (the same command line under torchrun)
        sys.exit(launch_ranks(args.gpus, Path(__file__).resolve(), sys.argv[1:]))
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local_rank = int(os.environ.get("LOCAL_RANK", 0))
    if world != args.gpus:
        ap.error(f"--gpus {args.gpus} but WORLD_SIZE is {world}: one rank per GPU")
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    if args.workload != "uneven_batch":
        {"plain_single": run_plain_single, "warm_family": run_warm, "extensions": run_extensions}.get(
            args.workload, lambda a: run_blocked(a, args.workload))(args)
        return
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local_rank))
    try:
        run_ours(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
