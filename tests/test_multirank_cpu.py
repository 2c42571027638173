"""Host logic of the multi-GPU bench path, run as two `gloo` ranks on CPU.

The batched workload shards by matrix: every rank solves its own seeded
batch (weak scaling) with no collective on the solve path; the only
collectives are the timing reductions (max over ranks) and barriers.  These
tests start two processes that take the same steps bench.py takes under
torchrun, without a GPU."""
import json
import os
import re
import socket
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent

CHILD = r"""
import json, os, sys, datetime
sys.path.insert(0, os.environ["REPO"])
import numpy as np
import torch.distributed as dist
dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
rank, world = dist.get_rank(), dist.get_world_size()
import bench
out = {"rank": rank, "world": world}
# the slowest rank's time is the job's time
out["max"] = bench.reduce_max(10.0 + rank, "cpu")
# every rank draws its own batch of the same distribution
mats = bench.load_matrices(rank)
out["count"] = len(mats)
out["digest"] = float(sum(float(a[0, 0]) for a in mats[:64]))
out["shapes"] = [list(a.shape) for a in mats[:8]]
digests = [None] * world
dist.all_gather_object(digests, out["digest"])
out["all_digests"] = digests
# strong scaling: each rank's cost-balanced share of the one seed-1 batch
import importlib
B = importlib.import_module("pavel-s_svd_b200.batch")
full = bench.load_matrices(0)
fm = np.array([a.shape[0] for a in full]); fn = np.array([a.shape[1] for a in full])
share = B.shard_by_cost(fm, fn, world)[rank]
mine = bench.load_matrices(rank, world, "strong")
out["share_same_matrices"] = all(np.array_equal(full[i], a) for i, a in zip(share, mine))
out["share_cost"] = float(B.matrix_cost(fm[share], fn[share]).sum())
out["total_cost"] = float(B.matrix_cost(fm, fn).sum())
shares = [None] * world
dist.all_gather_object(shares, share.tolist())
out["all_shares"] = shares
# the reference arm: rank 0 alone works and prints
class A: warmup = 3; steps = 1; ref_seconds = 0.2
if rank != 0:
    out["reference_returned"] = bench.run_reference(A, rank, world) is None
dist.barrier()
dist.destroy_process_group()
print("RESULT " + json.dumps(out), flush=True)
"""


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_gloo_ranks_shard_and_reduce():
    port = _free_port()
    procs = []
    for rank in range(2):
        env = dict(os.environ, RANK=str(rank), WORLD_SIZE="2", LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                   MASTER_PORT=str(port), REPO=str(ROOT), OMP_NUM_THREADS="1")
        procs.append(subprocess.Popen([sys.executable, "-c", CHILD], env=env, stdout=subprocess.PIPE,
                                      stderr=subprocess.PIPE, text=True))
    results = []
    for p in procs:
        out, err = p.communicate(timeout=240)
        assert p.returncode == 0, err[-2000:]
        line = [x for x in out.splitlines() if x.startswith("RESULT ")][-1]
        results.append(json.loads(line[len("RESULT "):]))
    results.sort(key=lambda r: r["rank"])
    # max over ranks, identical on every rank
    assert [r["max"] for r in results] == [11.0, 11.0]
    # weak scaling: each rank has a full batch, and the batches differ
    assert all(r["count"] == 8192 for r in results)
    assert results[0]["all_digests"] == results[1]["all_digests"]
    assert results[0]["digest"] != results[1]["digest"]
    assert results[1]["reference_returned"] is True
    # strong scaling: every matrix exactly once over the ranks, costs balanced
    got = sorted(results[0]["all_shares"][0] + results[0]["all_shares"][1])
    assert got == list(range(8192))
    assert all(r["share_same_matrices"] for r in results)
    costs = [r["share_cost"] for r in results]
    assert abs(sum(costs) - results[0]["total_cost"]) <= 1e-6 * results[0]["total_cost"]
    assert max(costs) / min(costs) <= 1.001


RANK_SCRIPT = r"""
import datetime, json, os, torch.distributed as dist
dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
t = __import__("torch").tensor([float(dist.get_rank() + 1)])
dist.all_reduce(t)
print("RANK " + json.dumps({"rank": dist.get_rank(), "world": dist.get_world_size(),
                            "local": int(os.environ["LOCAL_RANK"]), "sum": float(t)}), flush=True)
dist.destroy_process_group()
"""


def test_bench_starts_one_rank_per_gpu(tmp_path):
    """bench.py --gpus N without a torchrun environment starts N ranks
    through bench.launch_ranks (torch.distributed.run on 127.0.0.1, one
    process per GPU); here the launched script is a two-rank gloo job."""
    sys.path.insert(0, str(ROOT))
    import bench
    cmd = bench.rank_command(4, "x.py", ["--gpus", "4"], 29999)
    assert cmd[1:3] == ["-m", "torch.distributed.run"] and "--nproc-per-node=4" in cmd
    assert "--master-addr=127.0.0.1" in cmd and cmd[-3:] == ["x.py", "--gpus", "4"]
    script = tmp_path / "ranks.py"
    script.write_text(RANK_SCRIPT)
    out = subprocess.run([sys.executable, "-c", f"import sys; sys.path.insert(0, {str(ROOT)!r}); import bench; "
                          f"sys.exit(bench.launch_ranks(2, {str(script)!r}, [], timeout=200))"],
                         capture_output=True, text=True, timeout=240,
                         env=dict(os.environ, OMP_NUM_THREADS="1"))
    assert out.returncode == 0, out.stderr[-2000:]
    # the two ranks write to one stream, so their lines may interleave
    ranks = sorted((json.loads(x) for x in re.findall(r"RANK (\{[^{}]*\})", out.stdout)), key=lambda r: r["rank"])
    assert [(r["rank"], r["world"], r["local"], r["sum"]) for r in ranks] == [(0, 2, 0, 3.0), (1, 2, 1, 3.0)]
