// jb_tensor.cu - host side of the tcgen05 GEMM (jb_tc.cuh) and the small
// element-wise kernels that feed it: C-ABI entries jb_gemm_bf16 and
// jb_split_bf16 (include/jacobi_b200.h).
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>
#include <stdint.h>
#include <string.h>
#include <mutex>
#include "jacobi_b200.h"
#include "jb_tc.cuh"

namespace jb {
namespace tc {

static PFN_cuTensorMapEncodeTiled_v12000 g_encode = nullptr;
static std::mutex g_encode_mutex;

static PFN_cuTensorMapEncodeTiled_v12000 encoder() {
    std::lock_guard<std::mutex> lock(g_encode_mutex);
    if (!g_encode) {
        void *fn = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess || !fn)
            return nullptr;
        g_encode = (PFN_cuTensorMapEncodeTiled_v12000)fn;
    }
    return g_encode;
}

// 3-D map over a row-major BF16 array: x = inner (contiguous), y = rows, z =
// batch; boxes of 64 inner elements (one 128-byte swizzle row) x box_rows.
static bool make_map(CUtensorMap *map, const void *ptr, int64_t K, int64_t rows, int64_t ld, int64_t batch,
                     int64_t bstride, int box_rows) {
    auto enc = encoder();
    if (!enc) return false;
    cuuint64_t dims[3] = {(cuuint64_t)K, (cuuint64_t)rows, (cuuint64_t)batch};
    cuuint64_t strides[2] = {(cuuint64_t)ld * 2, (cuuint64_t)(batch > 1 ? bstride : rows * ld) * 2};
    cuuint32_t box[3] = {(cuuint32_t)BK, (cuuint32_t)box_rows, 1};
    cuuint32_t estr[3] = {1, 1, 1};
    CUresult r = enc(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 3, const_cast<void *>(ptr), dims, strides, box, estr,
                     CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                     CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS;
}

static size_t smem_bytes(int stages, int na, int nb, int bn) {
    return (size_t)stages * (na * A_TILE + nb * (uint32_t)bn * BK * 2) + (2 * stages + 1) * 8 + 16 + 1024;
}

template <int BN>
static int launch(TcParams &p, int64_t batch, cudaStream_t st) {
    const size_t per_stage = p.na * A_TILE + (p.a_as_b ? 0 : p.nb * (size_t)BN * BK * 2);
    int stages = (int)((227 * 1024 - 1024 - 64) / per_stage);
    if (stages > 6) stages = 6;
    // No more stages than k-blocks per CTA: short-K products (the rotation
    // updates, K = 2b) then leave room for several CTAs per SM.
    const int nk = (p.kchunk + BK - 1) / BK;
    if (stages > nk) stages = nk;
    if (stages < 1) return JB_ETOOBIG;
    p.stages = stages;
    const size_t smem = smem_bytes(stages, p.na, p.a_as_b ? 0 : p.nb, BN);
    auto kern = tc_gemm_kernel<BN>;
    if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
        return JB_ECUDA;
    // the column tiles of the first product, then (nx1 > 0) those of the second
    const int gx = (p.N + BN - 1) / BN + (p.nx1 > 0 ? (p.N2 + BN - 1) / BN : 0);
    dim3 grid((unsigned)gx, (unsigned)((p.M + BM - 1) / BM), (unsigned)(batch * p.splits));
    kern<<<grid, 128, smem, st>>>(p);
    return cudaGetLastError() == cudaSuccess ? JB_OK : JB_ECUDA;
}

__global__ void split_kernel(const float *x, __nv_bfloat16 *hi, __nv_bfloat16 *lo, __nv_bfloat16 *lo2, int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const float v = x[i];
        const __nv_bfloat16 h = __float2bfloat16_rn(v);
        hi[i] = h;
        if (lo) {
            const float r = v - __bfloat162float(h);
            const __nv_bfloat16 l = __float2bfloat16_rn(r);
            lo[i] = l;
            if (lo2) lo2[i] = __float2bfloat16_rn(r - __bfloat162float(l));
        }
    }
}

}  // namespace tc
}  // namespace jb

using namespace jb;

extern "C" {

int jb_gemm_bf16(const void *A0, const void *A1, const void *B0, const void *B1, int32_t mode, float *C, int64_t M,
                 int64_t N, int64_t K, int64_t lda, int64_t ldb, int64_t ldc, int64_t batch, int64_t strideA,
                 int64_t strideB, int64_t strideC, float alpha, float beta, int32_t split_k, int32_t *error_flag,
                 void *stream) {
    const void *A[3] = {A0, A1, nullptr}, *B[3] = {B0, B1, nullptr};
    return jb_gemm_bf16x(A, B, mode, C, M, N, K, lda, ldb, ldc, batch, strideA, strideB, strideC, alpha, beta,
                         split_k, error_flag, stream);
}

}  // extern "C"

namespace jb {
namespace tc {

// Validates the operands, builds the tensor maps and the K split.  Returns
// JB_OK and the tile width in *bn_out.
static int setup(const void *const *A, const void *const *B, int32_t mode, int64_t M, int64_t N, int64_t K,
                 int64_t lda, int64_t ldb, int64_t batch, int64_t strideA, int64_t strideB, int32_t split_k,
                 float alpha, int32_t *error_flag, TcParams &p, int &bn_out) {
    if (!A || !A[0] || M < 1 || N < 1 || K < 1 || batch < 1 || split_k < 1) return JB_EINVAL;
    const int kind = mode & 3;
    const int b_mn = (mode & JB_GEMM_B_MN) ? 1 : 0;
    const int chain128 = (mode & JB_GEMM_CHAIN128) ? 1 : 0;
    const int syrk = (mode & JB_GEMM_SYRK) ? 1 : 0;
    if (kind == 3 || (mode & ~(3 | JB_GEMM_B_MN | JB_GEMM_CHAIN128 | JB_GEMM_SYRK))) return JB_EINVAL;
    if (syrk && (b_mn || M != N || N > BM)) return JB_EINVAL;
    if (!syrk && (!B || !B[0])) return JB_EINVAL;
    const int nsplit = kind == JB_GEMM_PLAIN ? 1 : (kind == JB_GEMM_SPLIT3 ? 2 : 3);
    for (int i = 0; i < nsplit; ++i)
        if (!A[i] || ((uintptr_t)A[i] & 15) || (!syrk && (!B[i] || ((uintptr_t)B[i] & 15)))) return JB_EINVAL;
    if (lda % 8 || lda < K) return JB_EINVAL;
    if (!syrk && (ldb % 8 || (b_mn ? ldb < N : ldb < K))) return JB_EINVAL;
    if (batch > 1 && (strideA % 8 || (!syrk && strideB % 8))) return JB_EINVAL;
    if (M > (1 << 30) || N > (1 << 30)) return JB_ETOOBIG;
    memset(&p, 0, sizeof(p));
    int bn = N <= 64 ? 64 : (N <= 128 || nsplit == 3 ? 128 : 256);
    if (syrk && bn > BM) return JB_EINVAL;
    p.na = p.nb = nsplit;
    p.b_mn = b_mn;
    p.a_as_b = syrk;
    for (int a = 0; a < nsplit; ++a)
        if (!make_map(&p.ta[a], A[a], K, M, lda, batch, strideA, BM)) return JB_ECUDA;
    if (!syrk) {
        for (int b = 0; b < nsplit; ++b) {
            const bool ok = b_mn ? make_map(&p.tb[b], B[b], N, K, ldb, batch, strideB, BK)
                                 : make_map(&p.tb[b], B[b], K, N, ldb, batch, strideB, bn);
            if (!ok) return JB_ECUDA;
        }
    }
    p.M = (int)M; p.N = (int)N; p.K = (int)K;
    int64_t splits = split_k;
    if (chain128) {
        // up to 512 / bn accumulators of 128 along K per CTA
        const int64_t per_cta = (int64_t)(512 / bn) * 128;
        const int64_t need = (K + per_cta - 1) / per_cta;
        if (splits < need) splits = need;
    }
    int64_t chunk = (K + splits - 1) / splits;
    chunk = (chunk + BK - 1) / BK * BK;
    p.kchunk = (int)chunk;
    p.splits = (int)((K + chunk - 1) / chunk);
    if (batch * p.splits > 65535) return JB_ETOOBIG;
    if (chain128) {
        p.acc_kb = 128 / BK;
        const int chains = (int)((chunk + 127) / 128);
        int nacc = 1;
        while (nacc < chains) nacc *= 2;       // TMEM allocations are powers of two
        p.nacc = nacc;
    } else {
        p.acc_kb = (int)(chunk / BK);
        p.nacc = 1;
    }
    // Products of the split parts kept: hi*hi, hi*mid, mid*hi (3 terms), plus
    // hi*lo, mid*mid, lo*hi (6 terms): every pair whose exponents sum to at
    // most two splits below the leading term.
    static const int ta6[6] = {0, 0, 1, 0, 1, 2}, tb6[6] = {0, 1, 0, 2, 1, 0};
    p.nterm = nsplit == 1 ? 1 : (nsplit == 2 ? 3 : 6);
    for (int t = 0; t < p.nterm; ++t) { p.term_a[t] = ta6[t]; p.term_b[t] = tb6[t]; }
    p.alpha = alpha;
    p.error_flag = error_flag;
    bn_out = bn;
    return JB_OK;
}

static int dispatch(TcParams &p, int bn, int64_t batch, cudaStream_t st) {
    switch (bn) {
        case 64: return launch<64>(p, batch, st);
        case 128: return launch<128>(p, batch, st);
        default: return launch<256>(p, batch, st);
    }
}

}  // namespace tc
}  // namespace jb

extern "C" {

int jb_gemm_bf16x(const void *const *A, const void *const *B, int32_t mode, float *C, int64_t M, int64_t N, int64_t K,
                  int64_t lda, int64_t ldb, int64_t ldc, int64_t batch, int64_t strideA, int64_t strideB,
                  int64_t strideC, float alpha, float beta, int32_t split_k, int32_t *error_flag, void *stream) {
    if (!C || ldc < N) return JB_EINVAL;
    tc::TcParams p;
    int bn = 0;
    const int rc = tc::setup(A, B, mode, M, N, K, lda, ldb, batch, strideA, strideB, split_k, alpha, error_flag, p,
                             bn);
    if (rc != JB_OK) return rc;
    p.C = C; p.ldc = ldc; p.sC = strideC;
    p.beta = (p.splits > 1) ? 1.f : beta;
    cudaStream_t st = (cudaStream_t)stream;
    if (p.splits > 1 && beta == 0.f) {
        if (ldc == N && (batch == 1 || strideC == M * N)) {
            if (cudaMemsetAsync(C, 0, sizeof(float) * M * N * batch, st) != cudaSuccess) return JB_ECUDA;
        } else {
            for (int64_t z = 0; z < batch; ++z)
                if (cudaMemset2DAsync(C + z * strideC, ldc * sizeof(float), 0, N * sizeof(float), M, st) !=
                    cudaSuccess)
                    return JB_ECUDA;
        }
    }
    return tc::dispatch(p, bn, batch, st);
}

int jb_gemm_bf16x_rows(const void *const *A, const void *const *B, int32_t mode, void *const *out, int32_t nparts,
                       const int32_t *row_map, int64_t ld_out, int64_t M, int64_t N, int64_t K, int64_t lda,
                       int64_t ldb, int64_t batch, int64_t strideA, int64_t strideB, float alpha,
                       int32_t *error_flag, void *stream) {
    if (!out || nparts < 1 || nparts > 3 || ld_out < N || ld_out % 8) return JB_EINVAL;
    for (int i = 0; i < nparts; ++i)
        if (!out[i] || ((uintptr_t)out[i] & 15)) return JB_EINVAL;
    tc::TcParams p;
    int bn = 0;
    const int rc = tc::setup(A, B, mode, M, N, K, lda, ldb, batch, strideA, strideB, 1, alpha, error_flag, p, bn);
    if (rc != JB_OK) return rc;
    if (p.splits != 1) return JB_ETOOBIG;            // one CTA along K (the TMEM accumulators hold it)
    for (int i = 0; i < nparts; ++i) p.out_part[i] = (__nv_bfloat16 *)out[i];
    p.out_nparts = nparts;
    p.out_map = row_map;
    p.out_ld = ld_out;
    return tc::dispatch(p, bn, batch, (cudaStream_t)stream);
}

int jb_gemm_bf16x_rows2(const void *const *A, const void *const *B, const void *const *B2, int32_t mode,
                        void *const *out, void *const *out2, int32_t nparts, const int32_t *row_map, int64_t ld_out,
                        int64_t ld_out2, int64_t M, int64_t N, int64_t N2, int64_t K, int64_t lda, int64_t ldb,
                        int64_t ldb2, int64_t batch, int64_t strideA, int64_t strideB, int64_t strideB2, float alpha,
                        int32_t *error_flag, void *stream) {
    if (!out || !out2 || !B2 || nparts < 1 || nparts > 3 || N2 < 1 || ld_out < N || ld_out % 8 || ld_out2 < N2 ||
        ld_out2 % 8)
        return JB_EINVAL;
    for (int i = 0; i < nparts; ++i)
        if (!out[i] || ((uintptr_t)out[i] & 15) || !out2[i] || ((uintptr_t)out2[i] & 15)) return JB_EINVAL;
    tc::TcParams p;
    int bn = 0;
    const int rc = tc::setup(A, B, mode, M, N, K, lda, ldb, batch, strideA, strideB, 1, alpha, error_flag, p, bn);
    if (rc != JB_OK) return rc;
    if (p.splits != 1 || p.a_as_b) return JB_ETOOBIG;   // one CTA along K; B given
    // the second product: the same A, K, mode and split parts, its own B2
    if (ldb2 % 8 || (p.b_mn ? ldb2 < N2 : ldb2 < K) || (batch > 1 && strideB2 % 8) || N2 > (1 << 30))
        return JB_EINVAL;
    for (int i = 0; i < p.nb; ++i) {
        if (!B2[i] || ((uintptr_t)B2[i] & 15)) return JB_EINVAL;
        const bool ok = p.b_mn ? tc::make_map(&p.tb[3 + i], B2[i], N2, K, ldb2, batch, strideB2, tc::BK)
                               : tc::make_map(&p.tb[3 + i], B2[i], K, N2, ldb2, batch, strideB2, bn);
        if (!ok) return JB_ECUDA;
    }
    for (int i = 0; i < nparts; ++i) {
        p.out_part[i] = (__nv_bfloat16 *)out[i];
        p.out_part2[i] = (__nv_bfloat16 *)out2[i];
    }
    p.out_nparts = nparts;
    p.out_map = row_map;
    p.out_ld = ld_out;
    p.out_ld2 = ld_out2;
    p.nx1 = (int)((N + bn - 1) / bn);
    p.N2 = (int)N2;
    if ((int64_t)p.nx1 + (N2 + bn - 1) / bn > 0x7fffffff) return JB_ETOOBIG;
    return tc::dispatch(p, bn, batch, (cudaStream_t)stream);
}

int jb_split_bf16(const float *X, void *hi, void *lo, int64_t n, void *stream) {
    return jb_split3_bf16(X, hi, lo, nullptr, n, stream);
}

int jb_split3_bf16(const float *X, void *hi, void *mid, void *lo, int64_t n, void *stream) {
    if (!X || !hi || n < 0 || (lo && !mid)) return JB_EINVAL;
    if (n == 0) return JB_OK;
    int blocks = (int)((n + 255) / 256);
    if (blocks > 148 * 16) blocks = 148 * 16;
    tc::split_kernel<<<blocks, 256, 0, (cudaStream_t)stream>>>(X, (__nv_bfloat16 *)hi, (__nv_bfloat16 *)mid,
                                                               (__nv_bfloat16 *)lo, n);
    return cudaGetLastError() == cudaSuccess ? JB_OK : JB_ECUDA;
}

}  // extern "C"
