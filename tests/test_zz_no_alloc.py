"""The allocation-free entry point jb_svd_batched_f32_noalloc, through the C ABI.

It serves callers that cannot allocate device memory when they solve:
plug-ins whose host framework owns every device allocation through its own
pool, and latency-bound paths that must not call cudaMalloc/cudaFree (which
can synchronise the whole device).  Its scratch is a
fixed 16 MiB device array inside the library, so its results must equal
those of jb_svd_batched_f32 with a caller-provided workspace, call after call
(the array keeps the previous call's contents).

This file is collected last on purpose; it passes alone in a fresh process as
well as after the other tests.
"""
import numpy as np
import pytest
import torch

from conftest import sigma_tol

pytestmark = pytest.mark.gpu


def _outputs(b, m, n, dev):
    k = min(m, n)
    u = torch.empty(b, m, k, dtype=torch.float32, device=dev)
    s = torch.empty(b, k, dtype=torch.float32, device=dev)
    vh = torch.empty(b, k, n, dtype=torch.float32, device=dev)
    info = torch.full((2, b), -1, dtype=torch.int32, device=dev)
    return u, s, vh, info


def _with_workspace(lib, x, prec):
    b, m, n = x.shape
    u, s, vh, info = _outputs(b, m, n, x.device)
    ws = torch.empty(max(lib.jb_workspace_bytes(m, n, b, 4, prec, 0), 256), dtype=torch.uint8, device=x.device)
    stream = torch.cuda.current_stream().cuda_stream
    rc = lib.jb_svd_batched_f32(x.data_ptr(), u.data_ptr(), s.data_ptr(), vh.data_ptr(), b, m, n, min(m, n), 0,
                                0.0, 60, prec, info[0].data_ptr(), info[1].data_ptr(), ws.data_ptr(), ws.numel(),
                                stream)
    assert rc == 0
    torch.cuda.synchronize()
    return u, s, vh, info


def _no_alloc(lib, x, prec):
    b, m, n = x.shape
    u, s, vh, info = _outputs(b, m, n, x.device)
    stream = torch.cuda.current_stream().cuda_stream
    rc = lib.jb_svd_batched_f32_noalloc(x.data_ptr(), u.data_ptr(), s.data_ptr(), vh.data_ptr(), b, m, n,
                                        min(m, n), 0, 0.0, 60, prec, info[0].data_ptr(), info[1].data_ptr(), stream)
    assert rc == 0
    torch.cuda.synchronize()
    return u, s, vh, info


@pytest.mark.parametrize("prec", [0, 1])  # JB_PREC_NATIVE, JB_PREC_MIXED
@pytest.mark.parametrize("shape", [(96, 48, 32), (40, 20, 33), (8, 160, 100)])
def test_no_alloc_matches_workspace_entry(pkg, prec, shape):
    lib = pkg.native.lib()
    rng = np.random.default_rng(2026)
    x = torch.from_numpy(rng.standard_normal(shape).astype(np.float32)).cuda()
    ref_u, ref_s, ref_vh, ref_info = _with_workspace(lib, x, prec)
    assert (ref_info[1] == 0).all()
    tol = sigma_tol(np.float32)
    for _ in range(2):  # two calls in a row share the same scratch array
        u, s, vh, info = _no_alloc(lib, x, prec)
        assert (info[1] == 0).all()
        assert torch.equal(info[0], ref_info[0])
        top = ref_s.abs().amax(-1, keepdim=True)
        assert float(((s - ref_s).abs() / top).max()) <= tol
        assert float((u - ref_u).abs().max()) <= tol
        assert float((vh - ref_vh).abs().max()) <= tol


def test_no_alloc_rejects_requests_beyond_its_scratch(pkg):
    lib = pkg.native.lib()
    b, m, n = 1100, 64, 64  # mixed precision needs 4 * 1100 * 64^2 bytes > 16 MiB
    x = torch.zeros(b, m, n, dtype=torch.float32, device="cuda")
    u, s, vh, info = _outputs(b, m, n, x.device)
    rc = lib.jb_svd_batched_f32_noalloc(x.data_ptr(), u.data_ptr(), s.data_ptr(), vh.data_ptr(), b, m, n, n, 0,
                                        0.0, 60, 1, info[0].data_ptr(), info[1].data_ptr(),
                                        torch.cuda.current_stream().cuda_stream)
    assert rc == pkg.native.JB_ETOOBIG
    assert 4 * b * n * n > pkg.native.NOALLOC_SCRATCH_BYTES
