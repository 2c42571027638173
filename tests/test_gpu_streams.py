"""Solves enqueued at the same time on different CUDA streams (two host
threads, one stream each) give the same results as the same solves one after
the other: each stream has its own default workspace (ticket counters,
scratch), so concurrent persistent launches do not take each other's work."""
import importlib
import threading

import pytest
import torch

pytestmark = pytest.mark.gpu


def test_concurrent_streams_match_sequential():
    pkg = importlib.import_module("pavel-s_svd_b200")
    g = torch.Generator(device="cuda").manual_seed(11)
    inputs = [torch.randn(2048, 64, 40, device="cuda", generator=g),
              torch.randn(2048, 48, 48, device="cuda", generator=g, dtype=torch.float64),
              torch.randn(64, 600, 30, device="cuda", generator=g)]
    algs = ["jacobi", "jacobi", "qr"]
    ref = [pkg.svd(x, alg) for x, alg in zip(inputs, algs)]
    torch.cuda.synchronize()
    out, errors = [None] * len(inputs), []

    def work(i):
        try:
            s = torch.cuda.Stream()
            with torch.cuda.stream(s):
                for _ in range(3):
                    out[i] = pkg.svd(inputs[i], algs[i])
            s.synchronize()
        except Exception as e:      # surfaced below
            errors.append(e)

    threads = [threading.Thread(target=work, args=(i,)) for i in range(len(inputs))]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    assert not errors, errors
    for (u, s, vh), (u0, s0, vh0) in zip(out, ref):
        assert torch.equal(s, s0) and torch.equal(u, u0) and torch.equal(vh, vh0)
