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

// 3-D map over a row-major BF16 array: x = K (contiguous), y = rows, z = batch.
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
    const size_t per_stage = p.na * A_TILE + p.nb * (size_t)BN * BK * 2;
    int stages = (int)((227 * 1024 - 1024 - 64) / per_stage);
    if (stages > 6) stages = 6;
    if (stages < 2) return JB_ETOOBIG;
    p.stages = stages;
    const size_t smem = smem_bytes(stages, p.na, p.nb, BN);
    auto kern = tc_gemm_kernel<BN>;
    if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
        return JB_ECUDA;
    dim3 grid((unsigned)((p.N + BN - 1) / BN), (unsigned)((p.M + BM - 1) / BM), (unsigned)(batch * p.splits));
    kern<<<grid, 128, smem, st>>>(p);
    return cudaGetLastError() == cudaSuccess ? JB_OK : JB_ECUDA;
}

__global__ void split_kernel(const float *x, __nv_bfloat16 *hi, __nv_bfloat16 *lo, int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const float v = x[i];
        const __nv_bfloat16 h = __float2bfloat16_rn(v);
        hi[i] = h;
        if (lo) lo[i] = __float2bfloat16_rn(v - __bfloat162float(h));
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
    if (!A0 || !B0 || !C || M < 1 || N < 1 || K < 1 || batch < 1 || split_k < 1) return JB_EINVAL;
    if (mode != JB_GEMM_PLAIN && mode != JB_GEMM_SPLIT3) return JB_EINVAL;
    if (mode == JB_GEMM_SPLIT3 && (!A1 || !B1)) return JB_EINVAL;
    if (lda % 8 || ldb % 8 || lda < K || ldb < K || ldc < N) return JB_EINVAL;
    if (batch > 1 && (strideA % 8 || strideB % 8)) return JB_EINVAL;
    const void *ptrs[4] = {A0, A1, B0, B1};
    for (const void *q : ptrs)
        if (q && ((uintptr_t)q & 15)) return JB_EINVAL;
    if (M > (1 << 30) || N > (1 << 30) || batch * split_k > 65535) return JB_ETOOBIG;
    tc::TcParams p;
    memset(&p, 0, sizeof(p));
    const int bn = N <= 64 ? 64 : (N <= 128 ? 128 : 256);
    p.na = mode == JB_GEMM_SPLIT3 ? 2 : 1;
    p.nb = p.na;
    for (int a = 0; a < p.na; ++a)
        if (!tc::make_map(&p.ta[a], a ? A1 : A0, K, M, lda, batch, strideA, tc::BM)) return JB_ECUDA;
    for (int b = 0; b < p.nb; ++b)
        if (!tc::make_map(&p.tb[b], b ? B1 : B0, K, N, ldb, batch, strideB, bn)) return JB_ECUDA;
    p.C = C; p.ldc = ldc; p.sC = strideC;
    p.M = (int)M; p.N = (int)N; p.K = (int)K;
    int64_t chunk = (K + split_k - 1) / split_k;
    chunk = (chunk + tc::BK - 1) / tc::BK * tc::BK;
    p.kchunk = (int)chunk;
    p.splits = (int)((K + chunk - 1) / chunk);
    if (mode == JB_GEMM_SPLIT3) {
        p.nterm = 3;
        p.term_a[0] = 0; p.term_b[0] = 0;   // hi * hi
        p.term_a[1] = 0; p.term_b[1] = 1;   // hi * lo
        p.term_a[2] = 1; p.term_b[2] = 0;   // lo * hi
    } else {
        p.nterm = 1;
    }
    p.alpha = alpha;
    p.beta = (p.splits > 1) ? 1.f : beta;
    p.error_flag = error_flag;
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
    switch (bn) {
        case 64: return tc::launch<64>(p, batch, st);
        case 128: return tc::launch<128>(p, batch, st);
        default: return tc::launch<256>(p, batch, st);
    }
}

int jb_split_bf16(const float *X, void *hi, void *lo, int64_t n, void *stream) {
    if (!X || !hi || n < 0) return JB_EINVAL;
    if (n == 0) return JB_OK;
    int blocks = (int)((n + 255) / 256);
    if (blocks > 148 * 16) blocks = 148 * 16;
    tc::split_kernel<<<blocks, 256, 0, (cudaStream_t)stream>>>(X, (__nv_bfloat16 *)hi, (__nv_bfloat16 *)lo, n);
    return cudaGetLastError() == cudaSuccess ? JB_OK : JB_ECUDA;
}

}  // extern "C"
