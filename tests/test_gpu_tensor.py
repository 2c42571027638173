"""tcgen05 GEMM (jb_gemm_bf16) against a PyTorch FP32 reference of the same op.

Tolerances: the plain BF16 product is compared with torch's FP32 matmul of
the same BF16 inputs (FP32 accumulation on both sides): rel. Frobenius error
<= 1e-5.  The 3xBF16 product of FP32 inputs is compared with an FP64 matmul:
rel. Frobenius error <= 5e-5 (about 2^-16 per product term)."""
import importlib

import pytest
import torch

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def T():
    return importlib.import_module("pavel-s_svd_b200.tensor")


def rel(a, b):
    return float((a.double() - b.double()).norm() / b.double().norm())


@pytest.mark.parametrize("M,N,K,batch,split", [(128, 128, 64, 1, 1), (300, 200, 520, 1, 1), (64, 64, 4096, 3, 4),
                                                 (1000, 256, 2080, 1, 1), (128, 1024, 1024, 2, 1), (77, 33, 8, 1, 1)])
def test_plain_bf16_gemm(T, M, N, K, batch, split):
    g = torch.Generator(device="cuda").manual_seed(M * N + K)
    a = torch.randn(batch, M, K, device="cuda", generator=g).bfloat16()
    b = torch.randn(batch, N, K, device="cuda", generator=g).bfloat16()
    flag = torch.zeros(1, dtype=torch.int32, device="cuda")
    c = T.gemm(a, b, split_k=split, error_flag=flag)
    ref = a.float() @ b.float().transpose(-1, -2)
    torch.cuda.synchronize()
    assert int(flag) == 0
    assert rel(c, ref) <= 1e-5


def test_accumulate_and_alpha(T):
    a = torch.randn(256, 192, device="cuda").bfloat16()
    b = torch.randn(160, 192, device="cuda").bfloat16()
    c0 = torch.randn(256, 160, device="cuda")
    c = c0.clone()
    T.gemm(a, b, c, alpha=-0.5, beta=1.0)
    ref = c0 - 0.5 * (a.float() @ b.float().T)
    assert rel(c, ref) <= 1e-5


def test_split3_product_accuracy(T):
    g = torch.Generator(device="cuda").manual_seed(5)
    x = torch.randn(4, 4096, 64, device="cuda", generator=g)
    y = torch.randn(4, 4096, 64, device="cuda", generator=g)
    xh, xl = T.split_bf16(x.transpose(-1, -2).contiguous())   # (4, 64, 4096)
    yh, yl = T.split_bf16(y.transpose(-1, -2).contiguous())
    c = T.gemm(xh, yh, a_lo=xl, b_lo=yl, split_k=8)
    ref = x.double().transpose(-1, -2) @ y.double()
    e3 = rel(c, ref)
    c1 = T.gemm(xh, yh)
    assert e3 <= 5e-5 and e3 < rel(c1, ref) / 20


@pytest.mark.parametrize("M,N,K,batch", [(128, 256, 64, 1), (64, 1000, 128, 5), (200, 304, 72, 2)])
def test_mn_major_b(T, M, N, K, batch):
    """B given as K x N (N contiguous): C = A B (the update products of the
    blocked Jacobi)."""
    g = torch.Generator(device="cuda").manual_seed(M + N + K)
    a = torch.randn(batch, M, K, device="cuda", generator=g)
    bt = torch.randn(batch, K, N, device="cuda", generator=g)
    ah, al = T.split_bf16(a)
    bh, bl = T.split_bf16(bt)
    c1 = T.gemm_parts([ah], [bh], b_mn=True)
    assert rel(c1, ah.float() @ bh.float()) <= 1e-5
    c3 = T.gemm_parts([ah, al], [bh, bl], b_mn=True)
    assert rel(c3, a.double() @ bt.double()) <= 5e-5


def test_split6_reaches_fp32_accuracy(T):
    """The tensor-memory accumulator loses accuracy over long K chains, so the
    accurate modes bound the chain with split-K (128 K per chain here)."""
    g = torch.Generator(device="cuda").manual_seed(9)
    x = torch.randn(2, 300, 2048, device="cuda", generator=g)
    y = torch.randn(2, 260, 2048, device="cuda", generator=g)
    c6 = T.gemm_parts(T.split3_bf16(x), T.split3_bf16(y), split_k=16)
    ref = x.double() @ y.double().transpose(-1, -2)
    e6 = rel(c6, ref)
    e3 = rel(T.gemm_parts(T.split_bf16(x), T.split_bf16(y), split_k=16), ref)
    assert e6 <= 2e-6 and e6 < e3 / 2.5
    bt = torch.randn(2, 2048, 304, device="cuda", generator=g)
    c6m = T.gemm_parts(T.split3_bf16(x), T.split3_bf16(bt), b_mn=True, split_k=16)
    assert rel(c6m, x.double() @ bt.double()) <= 2e-6


@pytest.mark.parametrize("M,N,K,batch", [(300, 260, 2048, 2), (64, 64, 4096, 16), (128, 128, 8192, 4),
                                         (96, 200, 1000, 3)])
def test_chain128_accumulators(T, M, N, K, batch):
    """CHAIN128: chains of <= 128 along K in separate tensor-memory
    accumulators summed in FP32 -- the accuracy of split-K 128 without its
    atomics (and with far fewer CTAs along K)."""
    g = torch.Generator(device="cuda").manual_seed(M + N + K + batch)
    x = torch.randn(batch, M, K, device="cuda", generator=g)
    y = torch.randn(batch, N, K, device="cuda", generator=g)
    ref = x.double() @ y.double().transpose(-1, -2)
    flag = torch.zeros(1, dtype=torch.int32, device="cuda")
    c6 = T.gemm_parts(T.split3_bf16(x), T.split3_bf16(y), chain128=True, error_flag=flag)
    torch.cuda.synchronize()
    assert int(flag) == 0
    assert rel(c6, ref) <= 2e-6
    c3 = T.gemm_parts(T.split_bf16(x), T.split_bf16(y), chain128=True)
    assert rel(c3, ref) <= 5e-5


@pytest.mark.parametrize("M,K,batch,parts", [(64, 4096, 16, 3), (128, 8192, 16, 2), (40, 1000, 5, 3)])
def test_syrk_gram(T, M, K, batch, parts):
    """SYRK (B = A, one TMA stream for both operands): the block-pair Gram."""
    g = torch.Generator(device="cuda").manual_seed(M + K)
    x = torch.randn(batch, M, K, device="cuda", generator=g) * torch.logspace(0, -3, M, device="cuda")[:, None]
    sp = (T.split3_bf16 if parts == 3 else T.split_bf16)(x)
    c = T.gemm_parts(list(sp), None, syrk=True, chain128=True)
    ref = x.double() @ x.double().transpose(-1, -2)
    assert rel(c, ref) <= (2e-6 if parts == 3 else 5e-5)
    # entry-wise: relative to the column norms (what the Jacobi ratio needs)
    d = ref.diagonal(dim1=-2, dim2=-1).sqrt()
    scaled = (c.double() - ref).abs() / (d[..., :, None] * d[..., None, :])
    # FP32 accumulation over K: ~1e-6 relative per entry for the 6-term product
    assert float(scaled.max()) <= (5e-6 if parts == 3 else 5e-5)
    assert torch.equal(c, c.transpose(-1, -2)) or float((c - c.transpose(-1, -2)).abs().max()) <= 1e-6 * float(c.abs().max())


@pytest.mark.parametrize("parts", [1, 2, 3])
def test_rows_output_parts_and_map(T, parts):
    """jb_gemm_bf16x_rows: alpha A B (B N-contiguous) written as BF16 parts
    into mapped rows equals the FP32 product, split and scattered."""
    g = torch.Generator(device="cuda").manual_seed(parts)
    batch, M, K, L = 8, 64, 64, 1000
    a = torch.randn(batch, M, K, device="cuda", generator=g)
    bt = torch.randn(batch, K, L, device="cuda", generator=g)
    sa = T.split3_bf16(a)[:max(parts, 1)] if parts > 1 else (T.split_bf16(a)[0],)
    sb = T.split3_bf16(bt)[:max(parts, 1)] if parts > 1 else (T.split_bf16(bt)[0],)
    rows = batch * M
    perm = torch.randperm(rows, generator=torch.Generator().manual_seed(5)).to(torch.int32).cuda()
    out = [torch.full((rows, 1008), 7.0, dtype=torch.bfloat16, device="cuda") for _ in range(parts)]
    T.gemm_parts_rows(list(sa), list(sb), out, perm, b_mn=True, alpha=0.5)
    c = 0.5 * T.gemm_parts(list(sa), list(sb), b_mn=True).reshape(rows, L)
    got = torch.zeros(rows, L, dtype=torch.float32, device="cuda")
    for o in out:
        got += o[:, :L].float()
    expect = torch.empty_like(got)
    expect[perm.long()] = c
    # the parts carry 8, 16 or 24 significant bits of the FP32 result
    tol = {1: 2 ** -8, 2: 2 ** -16, 3: 2 ** -23}[parts]
    assert float(((got - expect).abs() / expect.abs().clamp_min(1e-30)).max()) <= tol
    for o in out:  # the padding past N is untouched
        assert bool((o[:, L:] == 7.0).all())


@pytest.mark.parametrize("parts", [2, 3])
def test_rows2_equals_two_rows_calls(T, parts):
    """jb_gemm_bf16x_rows2: the two products of one launch (shared A and row
    map, each B with its own width and leading dimension) write exactly what
    two jb_gemm_bf16x_rows calls write, and leave the padding untouched."""
    g = torch.Generator(device="cuda").manual_seed(10 + parts)
    batch, M, K, L1, L2 = 6, 64, 64, 1000, 328          # B rows 16-byte aligned (TMA strides)
    a = torch.randn(batch, M, K, device="cuda", generator=g)
    b1 = torch.randn(batch, K, L1, device="cuda", generator=g)
    b2 = torch.randn(batch, K, L2, device="cuda", generator=g)
    sa, s1, s2 = (list(T.split3_bf16(x)[:parts]) for x in (a, b1, b2))
    rows = batch * M
    perm = torch.randperm(rows, generator=torch.Generator().manual_seed(3)).to(torch.int32).cuda()
    fused1 = [torch.full((rows, 1008), 7.0, dtype=torch.bfloat16, device="cuda") for _ in range(parts)]
    fused2 = [torch.full((rows, 336), 7.0, dtype=torch.bfloat16, device="cuda") for _ in range(parts)]
    sep1 = [x.clone() for x in fused1]
    sep2 = [x.clone() for x in fused2]
    T.gemm_parts_rows2(sa, s1, fused1, s2, fused2, perm, b_mn=True, alpha=0.5)
    T.gemm_parts_rows(sa, s1, sep1, perm, b_mn=True, alpha=0.5)
    T.gemm_parts_rows(sa, s2, sep2, perm, b_mn=True, alpha=0.5)
    torch.cuda.synchronize()
    for f, s_ in zip(fused1 + fused2, sep1 + sep2):
        assert torch.equal(f, s_)
    assert bool((fused2[0][:, L2:] == 7.0).all())
