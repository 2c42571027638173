// jb_peak.cu - measured CUDA-core peaks for the rooflines of the FP32/FP64
// Jacobi kernels.  Each thread runs kChains independent fused multiply-add
// chains for `iters` steps (register operands only), so the loop is bound
// by the FP32 or FP64 pipe; the host times it with CUDA events and divides
// the flops by the time.  Three forms: scalar FP32 (fma.rn.f32), packed
// FP32 (fma.rn.f32x2, two lanes of FP32 per instruction, as the register
// Jacobi kernels issue them) and FP64 (fma.rn.f64).  No counterpart in the
// reference project; it serves the measurement only.
#include <cuda_runtime.h>
#include <stdint.h>
#include "jacobi_b200.h"

namespace jb {
namespace peak {

constexpr int kChains = 16;
constexpr int kThreads = 256;

__device__ __forceinline__ void ffma2(float &a0, float &a1, float x0, float x1, float y0, float y1) {
    asm(
        "{\n\t.reg .b64 ra, rx, ry;\n\t"
        "mov.b64 ra, {%0, %1};\n\tmov.b64 rx, {%2, %3};\n\tmov.b64 ry, {%4, %5};\n\t"
        "fma.rn.f32x2 ra, ra, rx, ry;\n\tmov.b64 {%0, %1}, ra;\n\t}"
        : "+f"(a0), "+f"(a1)
        : "f"(x0), "f"(x1), "f"(y0), "f"(y1));
}

// mode 0: FP32 scalar, 1: FP32 packed pairs, 2: FP64.  `sink` receives a
// value only when the (never met) condition holds, so no chain is dead code.
__global__ void __launch_bounds__(kThreads) fma_loop_kernel(int mode, int iters, float seed, float *sink) {
    const float x = 1.0f - 1e-7f * (float)(threadIdx.x & 7), y = 1e-7f * seed;
    if (mode == 2) {
        double a[kChains];
#pragma unroll
        for (int j = 0; j < kChains; ++j) a[j] = (double)(threadIdx.x + j) * 1e-3;
        const double xd = x, yd = y;
        for (int it = 0; it < iters; ++it)
#pragma unroll
            for (int j = 0; j < kChains; ++j) a[j] = fma(a[j], xd, yd);
        double s = 0.0;
#pragma unroll
        for (int j = 0; j < kChains; ++j) s += a[j];
        if (s == -1.2345) sink[blockIdx.x] = (float)s;
        return;
    }
    float a[kChains];
#pragma unroll
    for (int j = 0; j < kChains; ++j) a[j] = (float)(threadIdx.x + j) * 1e-3f;
    if (mode == 1) {
        for (int it = 0; it < iters; ++it)
#pragma unroll
            for (int j = 0; j < kChains; j += 2) ffma2(a[j], a[j + 1], x, x, y, y);
    } else {
        for (int it = 0; it < iters; ++it)
#pragma unroll
            for (int j = 0; j < kChains; ++j) a[j] = fmaf(a[j], x, y);
    }
    float s = 0.f;
#pragma unroll
    for (int j = 0; j < kChains; ++j) s += a[j];
    if (s == -1.2345f) sink[blockIdx.x] = s;
}

}  // namespace peak
}  // namespace jb

extern "C" {

double jb_fma_loop_flops(int32_t blocks, int32_t iters) {
    return 2.0 * jb::peak::kChains * jb::peak::kThreads * (double)blocks * (double)iters;
}

int jb_fma_loop(int32_t mode, int32_t blocks, int32_t iters, float *sink, void *stream) {
    if (mode < 0 || mode > 2 || blocks < 1 || iters < 1 || !sink) return JB_EINVAL;
    jb::peak::fma_loop_kernel<<<(unsigned)blocks, jb::peak::kThreads, 0, (cudaStream_t)stream>>>(mode, iters, 1.0f,
                                                                                                 sink);
    return cudaGetLastError() == cudaSuccess ? JB_OK : JB_ECUDA;
}

}  // extern "C"
