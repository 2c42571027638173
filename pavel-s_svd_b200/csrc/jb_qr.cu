// jb_qr.cu - batched Householder QR of tall matrices: the reference's
// primitives.qr (svdbench/standalone/primitives.py:74-89) with its
// reflector convention householder_vec (:41-59, LAPACK xLARFG: beta =
// -sign(alpha) ||x||, tau = (beta - alpha) / beta, v = x / (alpha - beta),
// v_0 = 1; a column with nothing below the diagonal is left alone) and Q by
// backward accumulation of the reflectors onto [I; 0].  It is the QR inside
// the reference's 'qr', 'tsqr' and projected ('randomized', 'subspace',
// 'block_krylov') solvers (solvers.py:71-96, 185-220, 245-248).
//
// One CTA per matrix (grid-stride over the batch), computing in the input
// type as the reference does.  The work area is the matrix (m x n,
// column-major: a warp walks a column with unit stride) whose lower part
// keeps the reflectors, and Q (m x n, column-major); in shared memory when
// both fit, else in a per-CTA slot of the workspace.  Per column j: the
// norm below the diagonal (one CTA reduction), the reflector, then one warp
// per remaining column applies I - tau v v^T.  Columns of Q left of j are
// zero in rows >= j during the backward accumulation, so only columns
// j..n-1 are updated (the reference's products with those zeros change
// nothing).
#include <cuda_runtime.h>
#include <stdint.h>
#include <math.h>
#include "jacobi_b200.h"

namespace jb {
namespace qr {

constexpr int kThreads = 256;

template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
    for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Sum over the CTA (partials in double); every thread gets it.  Two barriers.
template <typename T>
__device__ T block_sum(T v, double *red) {
    v = warp_sum(v);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = (double)v;
    __syncthreads();
    double r = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) r += red[w];
    __syncthreads();
    return (T)r;
}

constexpr size_t kSmemLimit = 227 * 1024;

__device__ __forceinline__ float hyp(float a, float b) { return hypotf(a, b); }
__device__ __forceinline__ double hyp(double a, double b) { return hypot(a, b); }

__host__ __device__ inline size_t align16z(size_t x) { return (x + 15) & ~(size_t)15; }

// Shared memory: red (32 doubles) | tau (n) | [work area: 2 m n] when in_smem.
template <typename T>
__host__ __device__ inline size_t smem_bytes(int m, int n, bool in_smem) {
    return 32 * 8 + align16z((size_t)n * sizeof(T)) + (in_smem ? 2 * (size_t)m * n * sizeof(T) : 0);
}

template <typename T>
__global__ void __launch_bounds__(kThreads) qr_kernel(const T *A, T *Qo, T *Ro, int64_t batch, int m, int n,
                                                      int in_smem, T *gws) {
    extern __shared__ __align__(16) unsigned char smem[];
    double *red = (double *)smem;
    T *tau = (T *)(smem + 32 * 8);
    const size_t mn = (size_t)m * n;
    T *Wk = in_smem ? (T *)(smem + 32 * 8 + align16z((size_t)n * sizeof(T))) : gws + (size_t)blockIdx.x * 2 * mn;
    T *Qk = Wk + mn;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    for (int64_t z = blockIdx.x; z < batch; z += gridDim.x) {
        const T *a = A + z * (int64_t)mn;
        __syncthreads();
        for (size_t idx = threadIdx.x; idx < mn; idx += blockDim.x) {
            const int r = (int)(idx / n), c = (int)(idx - (size_t)r * n);
            Wk[(size_t)c * m + r] = a[idx];
        }
        __syncthreads();
        for (int j = 0; j < n; ++j) {
            T *x = Wk + (size_t)j * m;
            T part = T(0);
            for (int i = j + 1 + threadIdx.x; i < m; i += blockDim.x) part += x[i] * x[i];
            const T xnorm = sqrt(block_sum(part, red));   // block_sum ends with a barrier
            const T alpha = x[j];
            const bool trivial = xnorm == T(0);
            const T beta = trivial ? alpha : (alpha < T(0) ? T(1) : T(-1)) * hyp(fabs(alpha), xnorm);
            const T denom = trivial ? T(1) : alpha - beta;
            const T t = trivial ? T(0) : (beta - alpha) / (beta != T(0) ? beta : T(1));
            __syncthreads();
            for (int i = j + 1 + threadIdx.x; i < m; i += blockDim.x) x[i] = trivial ? T(0) : x[i] / denom;
            if (threadIdx.x == 0) { tau[j] = t; x[j] = beta; }
            __syncthreads();
            if (t != T(0)) {
                // columns j+1..n-1, rows j..m-1: y <- y - tau v (v^T y), v_j = 1
                for (int c = j + 1 + warp; c < n; c += nw) {
                    T *y = Wk + (size_t)c * m;
                    T w = T(0);
                    for (int i = j + lane; i < m; i += 32) w += (i == j ? T(1) : x[i]) * y[i];
                    w = warp_sum(w);
                    for (int i = j + lane; i < m; i += 32) y[i] -= t * (i == j ? T(1) : x[i]) * w;
                }
            }
            __syncthreads();
        }
        T *r = Ro + z * (int64_t)n * n;
        for (int idx = threadIdx.x; idx < n * n; idx += blockDim.x) {
            const int i = idx / n, c = idx - i * n;                   // R row-major, upper triangle
            r[idx] = i <= c ? Wk[(size_t)c * m + i] : T(0);
        }
        for (size_t idx = threadIdx.x; idx < mn; idx += blockDim.x) {
            const int c = (int)(idx / m), i = (int)(idx - (size_t)c * m);
            Qk[idx] = i == c ? T(1) : T(0);
        }
        __syncthreads();
        for (int j = n - 1; j >= 0; --j) {
            const T t = tau[j];
            if (t != T(0)) {
                const T *v = Wk + (size_t)j * m;
                for (int c = j + warp; c < n; c += nw) {
                    T *y = Qk + (size_t)c * m;
                    T w = T(0);
                    for (int i = j + lane; i < m; i += 32) w += (i == j ? T(1) : v[i]) * y[i];
                    w = warp_sum(w);
                    for (int i = j + lane; i < m; i += 32) y[i] -= t * (i == j ? T(1) : v[i]) * w;
                }
            }
            __syncthreads();
        }
        T *q = Qo + z * (int64_t)mn;
        for (size_t idx = threadIdx.x; idx < mn; idx += blockDim.x) {
            const int i = (int)(idx / n), c = (int)(idx - (size_t)i * n);   // Q row-major
            q[idx] = Qk[(size_t)c * m + i];
        }
    }
}

// Complex input (complex64 / complex128, interleaved re, im): the same
// algorithm with the reference's complex reflector (householder_vec for
// complex x: beta = -sign(Re alpha) hypot(|alpha|, ||x_2:||), real; the
// column is left alone only when nothing is below the diagonal AND alpha is
// real; tau = (beta - alpha) / beta and v = x / (alpha - beta) complex), the
// factorisation applying (I - conj(tau) v v^H) and Q accumulating
// (I - tau v v^H) as primitives.py:80-87 do.
template <typename R> struct Cx { R re, im; };
template <typename R> __device__ __forceinline__ Cx<R> cmul(Cx<R> a, Cx<R> b) {
    return Cx<R>{a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
}
template <typename R> __device__ __forceinline__ Cx<R> cmulc(Cx<R> a, Cx<R> b) {   // conj(a) b
    return Cx<R>{a.re * b.re + a.im * b.im, a.re * b.im - a.im * b.re};
}
template <typename R> __device__ __forceinline__ Cx<R> cdiv(Cx<R> a, Cx<R> b) {
    const R d = b.re * b.re + b.im * b.im;
    return Cx<R>{(a.re * b.re + a.im * b.im) / d, (a.im * b.re - a.re * b.im) / d};
}

template <typename R>
__global__ void __launch_bounds__(kThreads) cqr_kernel(const Cx<R> *A, Cx<R> *Qo, Cx<R> *Ro, int64_t batch, int m,
                                                       int n, int in_smem, Cx<R> *gws) {
    using C = Cx<R>;
    extern __shared__ __align__(16) unsigned char smem[];
    double *red = (double *)smem;
    C *tau = (C *)(smem + 32 * 8);
    const size_t mn = (size_t)m * n;
    C *Wk = in_smem ? (C *)(smem + 32 * 8 + align16z((size_t)n * sizeof(C))) : gws + (size_t)blockIdx.x * 2 * mn;
    C *Qk = Wk + mn;
    const C zero{R(0), R(0)}, one{R(1), R(0)};
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    for (int64_t z = blockIdx.x; z < batch; z += gridDim.x) {
        const C *a = A + z * (int64_t)mn;
        __syncthreads();
        for (size_t idx = threadIdx.x; idx < mn; idx += blockDim.x) {
            const int r = (int)(idx / n), c = (int)(idx - (size_t)r * n);
            Wk[(size_t)c * m + r] = a[idx];
        }
        __syncthreads();
        for (int j = 0; j < n; ++j) {
            C *x = Wk + (size_t)j * m;
            R part = R(0);
            for (int i = j + 1 + threadIdx.x; i < m; i += blockDim.x) part += x[i].re * x[i].re + x[i].im * x[i].im;
            const R xnorm = sqrt(block_sum(part, red));   // block_sum ends with a barrier
            const C alpha = x[j];
            const bool trivial = xnorm == R(0) && alpha.im == R(0);
            const R beta = trivial ? alpha.re
                                   : (alpha.re < R(0) ? R(1) : R(-1)) * hyp(hyp(alpha.re, alpha.im), xnorm);
            const C denom = trivial ? one : C{alpha.re - beta, alpha.im};
            const R bd = beta != R(0) ? beta : R(1);
            const C t = trivial ? zero : C{(beta - alpha.re) / bd, -alpha.im / bd};
            __syncthreads();
            for (int i = j + 1 + threadIdx.x; i < m; i += blockDim.x) x[i] = trivial ? zero : cdiv(x[i], denom);
            if (threadIdx.x == 0) { tau[j] = t; x[j] = C{beta, R(0)}; }
            __syncthreads();
            if (t.re != R(0) || t.im != R(0)) {
                // columns j+1..n-1, rows j..m-1: y <- y - conj(tau) v (v^H y), v_j = 1
                const C tc{t.re, -t.im};
                for (int c = j + 1 + warp; c < n; c += nw) {
                    C *y = Wk + (size_t)c * m;
                    C w = zero;
                    for (int i = j + lane; i < m; i += 32) {
                        const C p = cmulc(i == j ? one : x[i], y[i]);
                        w.re += p.re; w.im += p.im;
                    }
                    w.re = warp_sum(w.re); w.im = warp_sum(w.im);
                    const C tw = cmul(tc, w);
                    for (int i = j + lane; i < m; i += 32) {
                        const C d = cmul(i == j ? one : x[i], tw);
                        y[i].re -= d.re; y[i].im -= d.im;
                    }
                }
            }
            __syncthreads();
        }
        C *r = Ro + z * (int64_t)n * n;
        for (int idx = threadIdx.x; idx < n * n; idx += blockDim.x) {
            const int i = idx / n, c = idx - i * n;
            r[idx] = i <= c ? Wk[(size_t)c * m + i] : zero;
        }
        for (size_t idx = threadIdx.x; idx < mn; idx += blockDim.x) {
            const int c = (int)(idx / m), i = (int)(idx - (size_t)c * m);
            Qk[idx] = i == c ? one : zero;
        }
        __syncthreads();
        for (int j = n - 1; j >= 0; --j) {
            const C t = tau[j];
            if (t.re != R(0) || t.im != R(0)) {
                const C *v = Wk + (size_t)j * m;
                for (int c = j + warp; c < n; c += nw) {
                    C *y = Qk + (size_t)c * m;
                    C w = zero;
                    for (int i = j + lane; i < m; i += 32) {
                        const C p = cmulc(i == j ? one : v[i], y[i]);
                        w.re += p.re; w.im += p.im;
                    }
                    w.re = warp_sum(w.re); w.im = warp_sum(w.im);
                    const C tw = cmul(t, w);
                    for (int i = j + lane; i < m; i += 32) {
                        const C d = cmul(i == j ? one : v[i], tw);
                        y[i].re -= d.re; y[i].im -= d.im;
                    }
                }
            }
            __syncthreads();
        }
        C *q = Qo + z * (int64_t)mn;
        for (size_t idx = threadIdx.x; idx < mn; idx += blockDim.x) {
            const int i = (int)(idx / n), c = (int)(idx - (size_t)i * n);
            q[idx] = Qk[(size_t)c * m + i];
        }
    }
}

static int sm_count_of_device() {
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev))
        return 0;
    return sms;
}

template <typename T>
static bool fits_smem(int m, int n) {
    return smem_bytes<T>(m, n, true) <= kSmemLimit;
}

template <typename T>
static size_t workspace_bytes(int m, int n, int64_t batch) {
    if (fits_smem<T>(m, n)) return 0;
    int sms = sm_count_of_device();
    if (sms <= 0) sms = 148;
    const int64_t grid = batch < (int64_t)sms * 2 ? batch : (int64_t)sms * 2;
    return (size_t)grid * 2 * (size_t)m * n * sizeof(T);
}

template <typename T, typename K>
static int launch(K kern, const T *A, T *Q, T *R, int64_t batch, int m, int n, void *workspace, size_t ws_bytes,
                  cudaStream_t st) {
    const bool in_smem = fits_smem<T>(m, n);
    const size_t smem = smem_bytes<T>(m, n, in_smem);
    if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
        return JB_ECUDA;
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kThreads, smem) != cudaSuccess) return JB_ECUDA;
    const int sms = sm_count_of_device();
    if (sms <= 0 || per_sm < 1) return JB_ECUDA;
    int64_t grid = (int64_t)sms * per_sm;
    if (grid > batch) grid = batch;
    T *gws = nullptr;
    if (!in_smem) {
        const size_t per_cta = 2 * (size_t)m * n * sizeof(T);
        const int64_t fit = (int64_t)(ws_bytes / per_cta);
        if (!workspace || fit < 1) return JB_EWORKSPACE;
        if (grid > fit) grid = fit;
        gws = (T *)workspace;
    }
    kern<<<(unsigned)grid, kThreads, smem, st>>>(A, Q, R, batch, m, n, in_smem ? 1 : 0, gws);
    return cudaGetLastError() == cudaSuccess ? JB_OK : JB_ECUDA;
}

template <typename T, typename K>
static int entry(K kern, const T *A, T *Q, T *R, int64_t batch, int32_t m, int32_t n, void *workspace,
                 size_t ws_bytes, void *stream) {
    if (!A || !Q || !R || batch < 0 || n < 1 || m < n) return JB_EINVAL;
    if ((int64_t)m * n > ((int64_t)1 << 31)) return JB_ETOOBIG;
    if (batch == 0) return JB_OK;
    return launch<T>(kern, A, Q, R, batch, m, n, workspace, ws_bytes, (cudaStream_t)stream);
}

}  // namespace qr
}  // namespace jb

extern "C" {

size_t jb_qr_workspace_bytes(int32_t m, int32_t n, int64_t batch, int32_t elem) {
    if (n < 1 || m < n || batch < 0) return 0;
    if (elem == 16) return jb::qr::workspace_bytes<jb::qr::Cx<double>>(m, n, batch);
    return elem == 8 ? jb::qr::workspace_bytes<double>(m, n, batch) : jb::qr::workspace_bytes<float>(m, n, batch);
}

int jb_qr_f32(const float *A, float *Q, float *R, int64_t batch, int32_t m, int32_t n, void *workspace,
              size_t workspace_bytes, void *stream) {
    return jb::qr::entry<float>(jb::qr::qr_kernel<float>, A, Q, R, batch, m, n, workspace, workspace_bytes, stream);
}

int jb_qr_f64(const double *A, double *Q, double *R, int64_t batch, int32_t m, int32_t n, void *workspace,
              size_t workspace_bytes, void *stream) {
    return jb::qr::entry<double>(jb::qr::qr_kernel<double>, A, Q, R, batch, m, n, workspace, workspace_bytes,
                                 stream);
}

int jb_qr_c64(const void *A, void *Q, void *R, int64_t batch, int32_t m, int32_t n, void *workspace,
              size_t workspace_bytes, void *stream) {
    using E = jb::qr::Cx<float>;
    return jb::qr::entry<E>(jb::qr::cqr_kernel<float>, (const E *)A, (E *)Q, (E *)R, batch, m, n, workspace,
                            workspace_bytes, stream);
}

int jb_qr_c128(const void *A, void *Q, void *R, int64_t batch, int32_t m, int32_t n, void *workspace,
               size_t workspace_bytes, void *stream) {
    using E = jb::qr::Cx<double>;
    return jb::qr::entry<E>(jb::qr::cqr_kernel<double>, (const E *)A, (E *)Q, (E *)R, batch, m, n, workspace,
                            workspace_bytes, stream);
}

}  // extern "C"
