"""batch.StreamedUneven: host-to-host uneven solve with the copies of one
chunk overlapped with the solve of another gives the same U, S, Vh and
sweeps as one UnevenBatch solve of the whole batch (the kernels solve each
matrix the same way whatever its neighbours), and raises like it."""
import importlib

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def test_streamed_equals_single_launch():
    B = importlib.import_module("pavel-s_svd_b200.batch")
    wl = importlib.import_module("pavel-s_svd_b200.workloads")
    mats = wl.uneven_batch(700, seed=5)
    flat, m, n, a_off = B.pack(mats)
    ref = B.UnevenBatch(m, n, "cuda", a_off=a_off)
    ref.launch(flat.cuda())
    sweeps_ref = ref.check()
    for chunks in (1, 3, 8):
        st = B.StreamedUneven(m, n, "cuda", chunks=chunks)
        hin, hu, hs, hv = st.host_buffers()
        hin.copy_(flat[:hin.numel()])
        st.run(hin, hu, hs, hv)
        sweeps = st.check()
        assert np.array_equal(sweeps, sweeps_ref)
        assert torch.equal(hs[:ref.S.numel()], ref.S.cpu())
        assert torch.equal(hu[:ref.U.numel()], ref.U.cpu())
        assert torch.equal(hv[:ref.Vh.numel()], ref.Vh.cpu())
        h2d, d2h = st.device_bytes_per_run()
        assert h2d == 4 * st.a_total and d2h > h2d


def test_streamed_raises_on_nonfinite_input():
    B = importlib.import_module("pavel-s_svd_b200.batch")
    mats = [np.random.default_rng(i).standard_normal((12, 8)).astype(np.float32) for i in range(6)]
    mats[4][3, 2] = np.nan
    flat, m, n, _ = B.pack(mats)
    st = B.StreamedUneven(m, n, "cuda", chunks=2)
    hin, hu, hs, hv = st.host_buffers()
    hin.copy_(flat[:hin.numel()])
    st.run(hin, hu, hs, hv)
    with pytest.raises(ValueError, match="NaN or infinity"):
        st.check()


def test_launch_choices_and_autotuner():
    """Every launch choice the autotuner varies (pair order, block width,
    FP32-phase exit ratio, one size class instead of two) converges to the
    same singular values within the mixed path's bound; tune() returns the
    fastest of them and caches it."""
    B = importlib.import_module("pavel-s_svd_b200.batch")
    N = importlib.import_module("pavel-s_svd_b200.native")
    wl = importlib.import_module("pavel-s_svd_b200.workloads")
    mats = wl.uneven_batch(600, seed=9)
    flat, m, n, a_off = B.pack(mats)
    x = flat.cuda()
    ref = None
    for cand in B.TUNE_CANDIDATES:
        plan = B.UnevenBatch(m, n, "cuda", a_off=a_off, launch=cand)
        plan.launch(x)
        sw = plan.check()
        assert sw.min() >= 1
        s = plan.S.cpu().numpy()
        if ref is None:
            ref = s
        else:
            assert float(np.abs(s - ref).max() / np.abs(ref).max()) <= 1e-6, repr(cand)
    best, times = B.tune(m, n, x)
    assert repr(best) in times and len(times) == len(B.TUNE_CANDIDATES)
    assert times[repr(best)] == min(times.values())
    assert B.tune(m, n, x)[0] is best                      # cached
    assert B.Launch(N.ROUND_ROBIN | N.BLOCK_WIDTH_8).flags == 12
    assert repr(B.Launch(N.ONE_SIZE_CLASS)) == "Launch(one_size_class, exit_ratio=0)"
