"""Host logic of the multi-GPU bench path, run as two `gloo` ranks on CPU.

The batched workload shards by matrix: every rank solves its own seeded
batch (weak scaling) with no collective on the solve path; the only
collectives are the timing reductions (max over ranks) and barriers.  These
tests start two processes that take the same steps bench.py takes under
torchrun, without a GPU."""
import json
import os
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
