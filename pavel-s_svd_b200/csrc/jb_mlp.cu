// jb_mlp.cu - element-wise kernels of the warm-start network and its Gram
// sketch.  The network's matrix products run on jb_gemm_bf16 (jb_tensor.cu);
// these kernels do everything between them: the input sketch, bias +
// activation, the ReLU backward mask, bias gradients, the MSE gradient, the
// Adam step (which also refreshes the BF16 weights and their transposes) and
// BF16 transposes of activations.  No counterpart in the reference project,
// whose Jacobi always starts from V = I (svdbench/standalone/primitives.py:324).
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>
#include "jacobi_b200.h"

namespace jb {
namespace mlp {

__device__ __forceinline__ float ldf(const void *p, int64_t i, int is_f32) {
    return is_f32 ? ((const float *)p)[i] : __bfloat162float(((const __nv_bfloat16 *)p)[i]);
}

// dst[z][c][r] = bf16(src[z][r][c]); 32 x 32 tiles through shared memory.
__global__ void transpose_kernel(const void *src, int src_f32, __nv_bfloat16 *dst, int64_t rows, int64_t cols) {
    __shared__ float tile[32][33];
    const int64_t z = blockIdx.z;
    const int64_t r0 = (int64_t)blockIdx.y * 32, c0 = (int64_t)blockIdx.x * 32;
    const int64_t off = z * rows * cols;
    for (int i = threadIdx.y; i < 32; i += blockDim.y) {
        const int64_t r = r0 + i, c = c0 + threadIdx.x;
        if (r < rows && c < cols) tile[i][threadIdx.x] = ldf(src, off + r * cols + c, src_f32);
    }
    __syncthreads();
    for (int i = threadIdx.y; i < 32; i += blockDim.y) {
        const int64_t c = c0 + i, r = r0 + threadIdx.x;
        if (r < rows && c < cols) dst[off + c * rows + r] = __float2bfloat16_rn(tile[threadIdx.x][i]);
    }
}

__global__ void bias_act_kernel(const float *Z, const float *bias, void *out, int64_t rows, int64_t cols, int relu,
                                int out_bf16) {
    const int64_t n = rows * cols;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        float v = Z[i] + (bias ? bias[i % cols] : 0.f);
        if (relu) v = fmaxf(v, 0.f);
        if (out_bf16) ((__nv_bfloat16 *)out)[i] = __float2bfloat16_rn(v);
        else ((float *)out)[i] = v;
    }
}

__global__ void relu_backward_kernel(const float *dH, const __nv_bfloat16 *H, void *G, int out_bf16, int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const float g = __bfloat162float(H[i]) > 0.f ? dH[i] : 0.f;
        if (out_bf16) ((__nv_bfloat16 *)G)[i] = __float2bfloat16_rn(g);
        else ((float *)G)[i] = g;
    }
}

// out[c] = sum_r X[r][c]; one thread per column, rows strided by warps.
__global__ void col_sum_kernel(const float *X, float *out, int64_t rows, int64_t cols) {
    const int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (c >= cols) return;
    float acc = 0.f;
    for (int64_t r = 0; r < rows; ++r) acc += X[r * cols + c];
    out[c] = acc;
}

// dY = scale * (Y - T); loss += sum (Y - T)^2 (one atomic per block).
__global__ void mse_grad_kernel(const float *Y, const float *T, float *dY, float *loss, int64_t n, float scale) {
    __shared__ float red[32];
    float acc = 0.f;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const float d = Y[i] - T[i];
        dY[i] = scale * d;
        acc = fmaf(d, d, acc);
    }
    for (int o = 16; o; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        float s = 0.f;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += red[w];
        atomicAdd(loss, s);
    }
}

// Adam on a rows x cols parameter; refreshes its BF16 copy and, when wT is
// given, its BF16 transpose (cols x rows).
__global__ void adam_kernel(float *w, const float *g, float *m, float *v, __nv_bfloat16 *wb, __nv_bfloat16 *wT,
                            int64_t rows, int64_t cols, float lr, float b1, float b2, float eps, float c1, float c2) {
    const int64_t n = rows * cols;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const float gi = g[i];
        const float mi = b1 * m[i] + (1.f - b1) * gi;
        const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        const float wi = w[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
        w[i] = wi;
        const __nv_bfloat16 h = __float2bfloat16_rn(wi);
        if (wb) wb[i] = h;
        if (wT) {
            const int64_t r = i / cols, c = i - r * cols;
            wT[c * rows + r] = h;
        }
    }
}

// Features of one matrix (m x n row-major): the upper triangle (row-major,
// i <= j) of A^T A / ||A||_F^2, as BF16.  One CTA per matrix, A staged in
// shared memory.
__global__ void sketch_kernel(const float *A, __nv_bfloat16 *X, int64_t batch, int m, int n) {
    extern __shared__ float sa[];
    const int64_t z = blockIdx.x;
    if (z >= batch) return;
    const float *a = A + z * (int64_t)m * n;
    __shared__ float s_tr;
    float part = 0.f;
    for (int i = threadIdx.x; i < m * n; i += blockDim.x) {
        const float x = a[i];
        sa[i] = x;
        part = fmaf(x, x, part);
    }
    for (int o = 16; o; o >>= 1) part += __shfl_xor_sync(0xffffffffu, part, o);
    __shared__ float red[32];
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = part;
    __syncthreads();
    if (threadIdx.x == 0) {
        float s = 0.f;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += red[w];
        s_tr = s > 0.f ? 1.f / s : 0.f;
    }
    __syncthreads();
    const int nf = n * (n + 1) / 2;
    __nv_bfloat16 *x = X + z * (int64_t)nf;
    for (int f = threadIdx.x; f < nf; f += blockDim.x) {
        // f -> (i, j), i <= j, row-major upper triangle.
        int i = 0, rem = f;
        while (rem >= n - i) { rem -= n - i; ++i; }
        const int j = i + rem;
        float acc = 0.f;
        for (int r = 0; r < m; ++r) acc = fmaf(sa[r * n + i], sa[r * n + j], acc);
        x[f] = __float2bfloat16_rn(acc * s_tr);
    }
}

static int grid_for(int64_t n) {
    int64_t b = (n + 255) / 256;
    if (b > 148 * 32) b = 148 * 32;
    return (int)(b < 1 ? 1 : b);
}

}  // namespace mlp
}  // namespace jb

using namespace jb::mlp;

extern "C" {

int jb_transpose_bf16(const void *src, int32_t src_is_f32, void *dst, int64_t rows, int64_t cols, int64_t batch,
                      void *stream) {
    if (!src || !dst || rows < 1 || cols < 1 || batch < 1 || batch > 65535) return JB_EINVAL;
    dim3 grid((unsigned)((cols + 31) / 32), (unsigned)((rows + 31) / 32), (unsigned)batch);
    transpose_kernel<<<grid, dim3(32, 8), 0, (cudaStream_t)stream>>>(src, src_is_f32, (__nv_bfloat16 *)dst, rows,
                                                                     cols);
    return cudaGetLastError() == cudaSuccess ? JB_OK : JB_ECUDA;
}

int jb_bias_act(const float *Z, const float *bias, void *out, int64_t rows, int64_t cols, int32_t relu,
                int32_t out_bf16, void *stream) {
    if (!Z || !out || rows < 1 || cols < 1) return JB_EINVAL;
    bias_act_kernel<<<grid_for(rows * cols), 256, 0, (cudaStream_t)stream>>>(Z, bias, out, rows, cols, relu, out_bf16);
    return cudaGetLastError() == cudaSuccess ? JB_OK : JB_ECUDA;
}

int jb_relu_backward(const float *dH, const void *H, void *G, int32_t out_bf16, int64_t n, void *stream) {
    if (!dH || !H || !G || n < 1) return JB_EINVAL;
    relu_backward_kernel<<<grid_for(n), 256, 0, (cudaStream_t)stream>>>(dH, (const __nv_bfloat16 *)H, G, out_bf16,
                                                                        n);
    return cudaGetLastError() == cudaSuccess ? JB_OK : JB_ECUDA;
}

int jb_col_sum(const float *X, float *out, int64_t rows, int64_t cols, void *stream) {
    if (!X || !out || rows < 1 || cols < 1) return JB_EINVAL;
    col_sum_kernel<<<(unsigned)((cols + 127) / 128), 128, 0, (cudaStream_t)stream>>>(X, out, rows, cols);
    return cudaGetLastError() == cudaSuccess ? JB_OK : JB_ECUDA;
}

int jb_mse_grad(const float *Y, const float *T, float *dY, float *loss, int64_t n, float scale, void *stream) {
    if (!Y || !T || !dY || !loss || n < 1) return JB_EINVAL;
    mse_grad_kernel<<<grid_for(n), 256, 0, (cudaStream_t)stream>>>(Y, T, dY, loss, n, scale);
    return cudaGetLastError() == cudaSuccess ? JB_OK : JB_ECUDA;
}

int jb_adam(float *w, const float *g, float *m, float *v, void *w_bf16, void *wT_bf16, int64_t rows, int64_t cols,
            float lr, float beta1, float beta2, float eps, int32_t step, void *stream) {
    if (!w || !g || !m || !v || rows < 1 || cols < 1 || step < 1) return JB_EINVAL;
    const float c1 = 1.f - powf(beta1, (float)step), c2 = 1.f - powf(beta2, (float)step);
    adam_kernel<<<grid_for(rows * cols), 256, 0, (cudaStream_t)stream>>>(
        w, g, m, v, (__nv_bfloat16 *)w_bf16, (__nv_bfloat16 *)wT_bf16, rows, cols, lr, beta1, beta2, eps, c1, c2);
    return cudaGetLastError() == cudaSuccess ? JB_OK : JB_ECUDA;
}

int jb_gram_sketch(const float *A, void *X, int64_t batch, int32_t m, int32_t n, void *stream) {
    if (!A || !X || batch < 1 || m < 1 || n < 1 || (size_t)m * n * 4 > 200 * 1024) return JB_EINVAL;
    const size_t smem = (size_t)m * n * 4;
    if (cudaFuncSetAttribute(sketch_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
        return JB_ECUDA;
    sketch_kernel<<<(unsigned)batch, 256, smem, (cudaStream_t)stream>>>(A, (__nv_bfloat16 *)X, batch, m, n);
    return cudaGetLastError() == cudaSuccess ? JB_OK : JB_ECUDA;
}

}  // extern "C"
