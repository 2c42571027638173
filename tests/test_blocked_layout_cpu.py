"""The host-side index tables of the blocked tensor-core solver (blocked.py),
checked on CPU: the pair-slot schedule of a block sweep, the row maps that
send every rotated row of W^T and V^T to its slot in the next round, and the
per-slot dataflow dependencies.  The kernels read these tables as they are,
so a wrong entry would pair the wrong blocks or scatter rows over each
other; the GPU parity tests only see the end result.

The schedule must be the reference's circle-method tournament, round by round
and slot by slot (primitives.py:309-313, restated by the oracle's
round_robin), so that the block rounds meet the column blocks in the
reference's order."""
import importlib
import types

import numpy as np
import pytest
import torch

from oracle import jacobi_oracle as O


def _blocked():
    return importlib.import_module("pavel-s_svd_b200.blocked")


def _plan(monkeypatch, m, n, b):
    """A BlockJacobi plan with CPU buffers; the SM count of a B200 stands in
    for the device query (only the Gram's K split reads it)."""
    monkeypatch.setattr(torch.cuda, "get_device_properties",
                        lambda dev: types.SimpleNamespace(multi_processor_count=148))
    return _blocked().BlockJacobi(m, n, b, device="cpu")


# (m, n, b): the block counts of the 4096 x 1024 (b = 32) and 8192 x 2048
# (b = 64) configurations at m = n, a ragged n (padded to whole blocks and an
# even block count), and the smallest plan (one slot)
SHAPES = ((1024, 1024, 32), (2048, 2048, 64), (300, 200, 32), (96, 72, 24), (64, 64, 32), (16, 16, 8))


@pytest.mark.parametrize("nb", (2, 4, 6, 8, 16, 32, 64, 128))
def test_schedule_is_the_reference_tournament(nb):
    B = _blocked()
    got = B.schedule(nb)
    assert got == list(O.round_robin(nb))
    pairs = [p for row in got for p in row]
    assert len(pairs) == nb * (nb - 1) // 2 == len(set(pairs))      # every block pair once per sweep
    for row in got:                                                   # a round's slots are disjoint
        blocks = [x for p in row for x in p]
        assert sorted(blocks) == list(range(nb))


@pytest.mark.parametrize("m,n,b", SHAPES)
def test_plan_sizes(monkeypatch, m, n, b):
    p = _plan(monkeypatch, m, n, b)
    assert p.nb % 2 == 0 and p.nb * b >= n > (p.nb - 2) * b
    assert p.npad == p.nb * b and p.P == p.nb // 2
    assert p.mpad % 8 == 0 and p.mpad - 8 < m <= p.mpad
    rows = p.P * 2 * b
    assert tuple(p.W[0][0].shape) == (rows, p.mpad) and tuple(p.V[1][2].shape) == (rows, p.npad)
    assert tuple(p.G.shape) == (p.P, 2 * b, 2 * b) and tuple(p.Gfull.shape) == (p.npad, p.npad)
    assert p.gram_split == max(1, 148 // p.P)


def _layout(p, r):
    """row of column c in round r's layout: slot k of the pair holding c's
    block, half h = 0 for the pair's first block, then the offset in the block."""
    b = p.b
    out = np.empty(p.npad, np.int64)
    for k, (i, j) in enumerate(p.sched[r]):
        for h, blk in enumerate((i, j)):
            out[blk * b:(blk + 1) * b] = k * 2 * b + h * b + np.arange(b)
    return out


@pytest.mark.parametrize("m,n,b", SHAPES)
def test_row_maps_follow_the_tournament(monkeypatch, m, n, b):
    p = _plan(monkeypatch, m, n, b)
    R, rows = p.nb - 1, p.P * 2 * b
    maps, back = p.maps.numpy(), p.back_maps.numpy()
    assert maps.shape == (R, rows) and back.shape == (R, p.npad)
    assert np.array_equal(p.init_map.numpy(), _layout(p, 0))
    for r in range(R):
        lay, nxt = _layout(p, r), _layout(p, (r + 1) % R)
        assert np.array_equal(np.sort(maps[r]), np.arange(rows))        # a permutation of the rows
        assert np.array_equal(maps[r][lay], nxt)                        # column c's row moves with c
        assert np.array_equal(back[r][lay], np.arange(p.npad))          # back map inverts the layout
        assert np.array_equal(p.pos[r, :, 0], lay[::b] // (2 * b))      # pos agrees with the layout
    # one sweep of row maps brings every column back to its round-0 row
    cur = p.init_map.numpy().astype(np.int64)
    for r in range(R):
        cur = maps[r][cur]
    assert np.array_equal(cur, p.init_map.numpy())


@pytest.mark.parametrize("m,n,b", SHAPES)
def test_dataflow_dependencies_follow_the_row_maps(monkeypatch, m, n, b):
    """src[r][k]: the round-r slots whose updates write rows of slot k in round
    r + 1; war[r][k]: the round-r slots that read the rows (of the other buffer)
    which slot k's round r + 1 update overwrites."""
    p = _plan(monkeypatch, m, n, b)
    R, w = p.nb - 1, 2 * b
    maps = p.maps.numpy()
    src, war = p._dataflow_deps()
    assert len(src) == len(war) == R
    for r in range(R):
        nr = (r + 1) % R
        for k in range(p.P):
            writers = {kk for kk in range(p.P) if np.any(maps[r][kk * w:(kk + 1) * w] // w == k)}
            assert src[r][k] == sorted(writers)
            overwritten = set((maps[nr][k * w:(k + 1) * w] // w).tolist())
            assert war[r][k] == sorted(overwritten)
            assert 1 <= len(src[r][k]) <= 2 and 1 <= len(war[r][k]) <= 2


def test_plan_argument_errors(monkeypatch):
    for m, n, b in ((64, 128, 32), (256, 256, 4), (256, 256, 12), (256, 256, 72)):
        with pytest.raises(ValueError):
            _plan(monkeypatch, m, n, b)
