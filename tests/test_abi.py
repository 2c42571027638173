"""The C-ABI library loads and exports every entry point include/*.h
declares -- CPU only, no compute calls."""
import ctypes
import re
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent


def declared_symbols():
    names = []
    for h in sorted((ROOT / "include").glob("*.h")):
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        names += re.findall(r"JB_API\s+[\w\s\*]+?\b(jb_\w+)\s*\(", text)
    return names


def test_header_declares_entry_points():
    names = declared_symbols()
    assert "jb_svd_batched_f32" in names and "jb_svd_uneven_f32" in names
    assert len(names) == len(set(names))


def test_library_exports_every_declared_symbol(pkg):
    lib = pkg.native.load()
    for name in declared_symbols():
        assert hasattr(lib, name), name
    assert tuple(n for n in declared_symbols() if n in pkg.native.SYMBOLS) == tuple(
        n for n in pkg.native.SYMBOLS if n in declared_symbols())


def test_library_is_sm100a_and_torch_free(pkg):
    import subprocess
    so = pkg.native.load()._name
    out = subprocess.run(["ldd", so], capture_output=True, text=True).stdout
    # the names the library links and where they resolve, without the load
    # addresses (random hex, which may spell "c10")
    deps = [line.split("(0x")[0] for line in out.splitlines()]
    assert deps and not any("torch" in d or "c10" in d for d in deps), deps


def test_workspace_query_is_host_only(pkg):
    lib = pkg.native.load()
    assert lib.jb_version() >= 100
    small = lib.jb_workspace_bytes(128, 64, 8192, 4, 0, 0)
    assert 0 < small < 1 << 20
    mixed = lib.jb_workspace_bytes(128, 64, 8192, 4, 1, 0)
    assert mixed >= small + 8192 * 64 * 64 * 4  # FP32-phase V of every matrix
    assert lib.jb_workspace_bytes(0, 4, 1, 4, 0, 0) == 0
    assert lib.jb_workspace_bytes(4, 4, 1, 3, 0, 0) == 0


def test_descriptor_layout_matches_header(pkg):
    B = __import__("importlib").import_module("pavel-s_svd_b200.batch")
    assert pkg.native.DESC_BYTES == 56 == B.DESC_DTYPE.itemsize
    assert pkg.native.MatrixDesc.a_off.offset == 16


def test_argument_errors_return_codes_without_a_device(pkg):
    lib = pkg.native.load()
    # rank 0 and max_sweeps 0 are rejected before any CUDA call
    assert lib.jb_svd_batched_f32(None, None, None, None, 1, 4, 4, 0, 0, 0.0, 30, 0, None, None, None, 0,
                                  None) == pkg.native.JB_EINVAL
    assert lib.jb_svd_batched_f64(None, None, None, None, 1, 4, 4, 4, 0, 0.0, 0, None, None, None, 0,
                                  None) == pkg.native.JB_EINVAL
    assert lib.jb_svd_uneven_f32(None, None, None, None, None, None, 1, 4, 4, 0.0, 30, 0, None, None, None, 0,
                                 None) == pkg.native.JB_EINVAL


def test_tensor_entry_argument_errors_without_a_device(pkg):
    """The tensor-core product entries reject bad output arguments before any
    CUDA call.  The pointer values are never dereferenced: each call fails in
    the first argument check."""
    lib, EINVAL = pkg.native.load(), pkg.native.JB_EINVAL
    ptrs = lambda *v: (ctypes.c_void_p * 3)(*v)            # noqa: E731
    ok, bad = ptrs(0x1000, 0x2000, 0x3000), ptrs(0x1008, 0x2000, 0x3000)
    rows2 = lambda out, out2, b2, nparts, ld, ld2, n2: lib.jb_gemm_bf16x_rows2(   # noqa: E731
        ok, ok, b2, 0, out, out2, nparts, None, ld, ld2, 64, 64, n2, 64, 64, 64, 64, 1, 0, 0, 0, 1.0, None, None)
    assert rows2(None, ok, ok, 1, 64, 64, 64) == EINVAL            # no output parts
    assert rows2(ok, None, ok, 1, 64, 64, 64) == EINVAL            # no second output
    assert rows2(ok, ok, None, 1, 64, 64, 64) == EINVAL            # no second B
    assert rows2(ok, ok, ok, 0, 64, 64, 64) == EINVAL              # 1 to 3 parts
    assert rows2(ok, ok, ok, 4, 64, 64, 64) == EINVAL
    assert rows2(ok, ok, ok, 1, 60, 64, 64) == EINVAL              # ld_out below N
    assert rows2(ok, ok, ok, 1, 68, 64, 64) == EINVAL              # ld_out not a multiple of 8
    assert rows2(ok, ok, ok, 1, 64, 56, 64) == EINVAL              # ld_out2 below N2
    assert rows2(ok, ok, ok, 1, 64, 64, 0) == EINVAL               # empty second product
    assert rows2(bad, ok, ok, 1, 64, 64, 64) == EINVAL             # parts 16-byte aligned
    assert rows2(ok, bad, ok, 1, 64, 64, 64) == EINVAL
    rows = lambda out, nparts, ld: lib.jb_gemm_bf16x_rows(ok, ok, 0, out, nparts, None, ld, 64, 64, 64, 64, 64,  # noqa: E731
                                                          1, 0, 0, 1.0, None, None)
    assert rows(None, 1, 64) == EINVAL and rows(ok, 0, 64) == EINVAL
    assert rows(ok, 1, 68) == EINVAL and rows(bad, 1, 64) == EINVAL     # ld_out a multiple of 8; aligned parts
    f64acc = lib.jb_gemm_f64acc
    assert f64acc(None, 0x1000, 0x2000, 8, 8, 8, 8, 8, 8, None) == EINVAL
    assert f64acc(0x1000, 0x2000, 0x3000, 0, 8, 8, 8, 8, 8, None) == EINVAL
    assert f64acc(0x1000, 0x2000, 0x3000, 8, 8, 8, 4, 8, 8, None) == EINVAL       # lda below K
    assert f64acc(0x1000, 0x2000, 0x3000, 8, 8, 8, 8, 8, 4, None) == EINVAL       # ldc below N
