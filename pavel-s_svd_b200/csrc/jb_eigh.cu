// jb_eigh.cu - batched two-sided cyclic Jacobi eigen-solver for real
// symmetric matrices: the reference's jacobi_eigh
// (svdbench/standalone/primitives.py:370-427, the syevj structure), used by
// its gram_jacobi and polar_* families (solvers.py:109, 170).
//
// One CTA per matrix: G (n x n, padded to even n with a zero row and column,
// FP64) and V accumulated in FP64, in shared memory when they fit (n <= 118
// both, n <= 166 G alone), else in a per-CTA global area.  Per round of the
// round-robin tournament (primitives.py:309-313) the reference's plane
// rotation of every active
// pair, then G <- J^T G J and V <- V J.  A pair is active when
// |g_pq| > tol * max|G| (the reference's absolute criterion, with max|G|
// taken at the start of each sweep rather than each round), and the solve
// has converged after a sweep whose largest |g_pq| / max|G| is <= tol.
// Eigenvalues come out ascending with V's columns in the same order.
#include <cuda_runtime.h>
#include <stdint.h>
#include <math.h>
#include "jacobi_b200.h"

namespace jb {
namespace eigh {

__device__ __forceinline__ int circ(int pos, int r, int n) {
    if (pos == 0) return 0;
    int x = (pos - 1 - r) % (n - 1);
    if (x < 0) x += n - 1;
    return 1 + x;
}

constexpr int kThreads = 512;

// mode 2: G and V in shared memory; 1: G only; 0: neither
__host__ __device__ inline size_t smem_bytes(int np, int mode) {
    return (size_t)np * np * 8 * mode + (size_t)np * 8 + (size_t)np + 32 * 8 + (size_t)np * 4 + 64;
}

template <typename T>
__global__ void __launch_bounds__(kThreads) eigh_kernel(const T *H, T *W, T *Vout, int32_t *sweeps_out,
                                                        int32_t *status, int64_t batch, int n, double tol,
                                                        int max_sweeps, int mode, double *gv) {
    extern __shared__ __align__(16) unsigned char smem[];
    const int np = n + (n & 1), half = np / 2;
    const size_t nn = (size_t)np * np;
    double *area = gv ? gv + (size_t)blockIdx.x * nn * (2 - mode) : nullptr;  // this CTA's global arrays
    double *G = mode >= 1 ? (double *)smem : area;                // np x np, G[col * np + row]
    double *V = mode == 2 ? (double *)smem + nn : (mode == 1 ? area : area + nn);
    double *cs = (double *)smem + nn * mode;                      // c[half], s[half]
    double *red = cs + np;                                        // 32 warp partials
    int *perm = (int *)(red + 32);                                // np
    unsigned char *pq = (unsigned char *)(perm + np);             // p[half], q[half]
    __shared__ int s_any;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    for (int64_t z = blockIdx.x; z < batch; z += gridDim.x) {
        const T *h = H + z * (int64_t)n * n;
        __syncthreads();
        for (int i = threadIdx.x; i < np * np; i += blockDim.x) {
            const int c = i / np, r = i - c * np;
            double g = 0.0;
            if (r < n && c < n) g = 0.5 * ((double)h[(size_t)r * n + c] + (double)h[(size_t)c * n + r]);
            G[i] = g;
            V[i] = (r == c) ? 1.0 : 0.0;
        }
        int sweep = 0, converged = 0;
        for (sweep = 1; sweep <= max_sweeps; ++sweep) {
            __syncthreads();
            // max|G| at the sweep start (the reference's scale, primitives.py:395)
            double mx = 0.0;
            for (int i = threadIdx.x; i < np * np; i += blockDim.x) mx = fmax(mx, fabs(G[i]));
            for (int o = 16; o; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
            if (lane == 0) red[warp] = mx;
            if (threadIdx.x == 0) s_any = 0;
            __syncthreads();
            double scale = 0.0;
            for (int w = 0; w < nw; ++w) scale = fmax(scale, red[w]);
            const double thr = tol * scale;
            for (int r = 0; r < np - 1; ++r) {
                __syncthreads();
                for (int t = threadIdx.x; t < half; t += blockDim.x) {
                    int p = circ(t, r, np), q = circ(np - 1 - t, r, np);
                    if (p > q) { const int x = p; p = q; q = x; }
                    const double gpp = G[(size_t)p * np + p], gqq = G[(size_t)q * np + q], gpq = G[(size_t)q * np + p];
                    const double a = fabs(gpq);
                    double c = 1.0, s = 0.0;
                    if (a > thr) {
                        // tau = (gqq - gpp) / (2 a), t = sign(tau) / (|tau| + hypot(tau, 1)), t = 1 at tau = 0
                        const double tau = (gqq - gpp) / (2.0 * a);
                        const double tt = tau == 0.0 ? 1.0 : copysign(1.0, tau) / (fabs(tau) + hypot(tau, 1.0));
                        c = 1.0 / sqrt(1.0 + tt * tt);
                        s = tt * c * (gpq < 0.0 ? -1.0 : 1.0);
                        s_any = 1;
                    }
                    cs[t] = c;
                    cs[half + t] = s;
                    pq[t] = (unsigned char)p;
                    pq[half + t] = (unsigned char)q;
                }
                __syncthreads();
                // G <- J^T G J (2 x 2 blocks: row pair a, column pair b); V <- V J
                for (int b = warp; b < half; b += nw) {
                    const int u = pq[b], v = pq[half + b];
                    const double cb = cs[b], sb = cs[half + b];
                    double *cu = G + (size_t)u * np, *cv = G + (size_t)v * np;
                    for (int a = lane; a < half; a += 32) {
                        const int p = pq[a], q = pq[half + a];
                        const double ca = cs[a], sa = cs[half + a];
                        const double gpu = cu[p], gqu = cu[q], gpv = cv[p], gqv = cv[q];
                        const double rpu = ca * gpu - sa * gqu, rqu = sa * gpu + ca * gqu;
                        const double rpv = ca * gpv - sa * gqv, rqv = sa * gpv + ca * gqv;
                        cu[p] = cb * rpu - sb * rpv;
                        cv[p] = sb * rpu + cb * rpv;
                        cu[q] = cb * rqu - sb * rqv;
                        cv[q] = sb * rqu + cb * rqv;
                    }
                    if (cb != 1.0 || sb != 0.0) {
                        double *vu = V + (size_t)u * np, *vv = V + (size_t)v * np;
                        for (int i = lane; i < np; i += 32) {
                            const double x = vu[i], y = vv[i];
                            vu[i] = cb * x - sb * y;
                            vv[i] = sb * x + cb * y;
                        }
                    }
                }
            }
            __syncthreads();
            if (!s_any) { converged = 1; break; }
        }
        __syncthreads();
        // ascending, stable; the padding column (index n) is left out
        for (int j = threadIdx.x; j < n; j += blockDim.x) {
            const double dj = G[(size_t)j * np + j];
            int rk = 0;
            for (int i = 0; i < n; ++i) {
                const double di = G[(size_t)i * np + i];
                rk += (di < dj) || (di == dj && i < j);
            }
            perm[rk] = j;
        }
        __syncthreads();
        T *w = W + z * (int64_t)n;
        T *vo = Vout + z * (int64_t)n * n;
        for (int k = threadIdx.x; k < n; k += blockDim.x) w[k] = (T)G[(size_t)perm[k] * np + perm[k]];
        for (int k = threadIdx.x; k < n * n; k += blockDim.x) {
            const int i = k / n, j = k - i * n;                   // row-major output, column j = eigenvector j
            vo[k] = (T)V[(size_t)perm[j] * np + i];
        }
        if (threadIdx.x == 0) {
            if (sweeps_out) sweeps_out[z] = sweep > max_sweeps ? max_sweeps : sweep;
            if (status) status[z] = converged ? JB_ST_OK : JB_ST_NOT_CONVERGED;
        }
    }
}

// Complex Hermitian H (complex64 / complex128, interleaved re, im), computed
// in complex128: the reference's complex branch (primitives.py:393-421) --
// g_pp, g_qq real, s = t c g_pq / |g_pq|, G <- G J on columns (c g_p -
// conj(s) g_q, s g_p + c g_q), G <- J^H G on rows (c r_p - s r_q, conj(s) r_p
// + c r_q), V <- V J; the same round-robin pairs, scale and convergence test
// as the real kernel.  Shared memory: G (and V) as double pairs when they fit.
struct Z { double re, im; };
__device__ __forceinline__ Z zmul(Z a, Z b) { return Z{a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; }
__device__ __forceinline__ Z zconj(Z a) { return Z{a.re, -a.im}; }
__device__ __forceinline__ Z zaxpby(double ca, Z x, Z sb, Z y) {   // ca x + sb y
    const Z t = zmul(sb, y);
    return Z{ca * x.re + t.re, ca * x.im + t.im};
}

__host__ __device__ inline size_t zsmem_bytes(int np, int mode) {
    return (size_t)np * np * 16 * mode + (size_t)np * 24 + (size_t)np + 32 * 8 + (size_t)np * 4 + 64;
}

template <typename R>
__global__ void __launch_bounds__(kThreads) zeigh_kernel(const R *H, R *W, R *Vout, int32_t *sweeps_out,
                                                         int32_t *status, int64_t batch, int n, double tol,
                                                         int max_sweeps, int mode, Z *gv) {
    extern __shared__ __align__(16) unsigned char smem[];
    const int np = n + (n & 1), half = np / 2;
    const size_t nn = (size_t)np * np;
    Z *area = gv ? gv + (size_t)blockIdx.x * nn * (2 - mode) : nullptr;
    Z *G = mode >= 1 ? (Z *)smem : area;                      // G[col * np + row]
    Z *V = mode == 2 ? (Z *)smem + nn : (mode == 1 ? area : area + nn);
    double *cs = (double *)((Z *)smem + nn * mode);           // c[half]
    Z *sv = (Z *)(cs + half + (half & 1));                    // s[half]
    double *red = (double *)(sv + half);                      // 32 warp partials
    int *perm = (int *)(red + 32);                            // np
    unsigned char *pq = (unsigned char *)(perm + np);         // p[half], q[half]
    __shared__ int s_any;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    for (int64_t z = blockIdx.x; z < batch; z += gridDim.x) {
        const R *h = H + z * (int64_t)n * n * 2;
        __syncthreads();
        for (int i = threadIdx.x; i < np * np; i += blockDim.x) {
            const int c = i / np, r = i - c * np;
            Z g{0.0, 0.0};
            if (r < n && c < n) {   // (H + H^H) / 2
                const double ar = (double)h[2 * ((size_t)r * n + c)], ai = (double)h[2 * ((size_t)r * n + c) + 1];
                const double br = (double)h[2 * ((size_t)c * n + r)], bi = (double)h[2 * ((size_t)c * n + r) + 1];
                g = Z{0.5 * (ar + br), 0.5 * (ai - bi)};
            }
            G[i] = g;
            V[i] = Z{(r == c) ? 1.0 : 0.0, 0.0};
        }
        int sweep = 0, converged = 0;
        for (sweep = 1; sweep <= max_sweeps; ++sweep) {
            __syncthreads();
            double mx = 0.0;
            for (int i = threadIdx.x; i < np * np; i += blockDim.x) mx = fmax(mx, hypot(G[i].re, G[i].im));
            for (int o = 16; o; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
            if (lane == 0) red[warp] = mx;
            if (threadIdx.x == 0) s_any = 0;
            __syncthreads();
            double scale = 0.0;
            for (int w = 0; w < nw; ++w) scale = fmax(scale, red[w]);
            const double thr = tol * scale;
            for (int r = 0; r < np - 1; ++r) {
                __syncthreads();
                for (int t = threadIdx.x; t < half; t += blockDim.x) {
                    int p = circ(t, r, np), q = circ(np - 1 - t, r, np);
                    if (p > q) { const int x = p; p = q; q = x; }
                    const double gpp = G[(size_t)p * np + p].re, gqq = G[(size_t)q * np + q].re;
                    const Z gpq = G[(size_t)q * np + p];                  // row p, column q
                    const double a = hypot(gpq.re, gpq.im);
                    double c = 1.0;
                    Z s{0.0, 0.0};
                    if (a > thr) {
                        const double tau = (gqq - gpp) / (2.0 * a);
                        const double tt = tau == 0.0 ? 1.0 : copysign(1.0, tau) / (fabs(tau) + hypot(tau, 1.0));
                        c = 1.0 / sqrt(1.0 + tt * tt);
                        s = Z{tt * c * gpq.re / a, tt * c * gpq.im / a};
                        s_any = 1;
                    }
                    cs[t] = c;
                    sv[t] = s;
                    pq[t] = (unsigned char)p;
                    pq[half + t] = (unsigned char)q;
                }
                __syncthreads();
                // G <- J^H G J (2 x 2 blocks: row pair a, column pair b); V <- V J
                for (int b = warp; b < half; b += nw) {
                    const int u = pq[b], v = pq[half + b];
                    const double cb = cs[b];
                    const Z sb = sv[b], sbc = zconj(sb), msbc = Z{-sb.re, sb.im};
                    Z *cu = G + (size_t)u * np, *cv = G + (size_t)v * np;
                    for (int a = lane; a < half; a += 32) {
                        const int p = pq[a], q = pq[half + a];
                        const double ca = cs[a];
                        const Z sa = sv[a], msa = Z{-sa.re, -sa.im}, sac = zconj(sa);
                        const Z gpu = cu[p], gqu = cu[q], gpv = cv[p], gqv = cv[q];
                        // rows: r_p = c r_p - s r_q, r_q = conj(s) r_p + c r_q
                        const Z rpu = zaxpby(ca, gpu, msa, gqu), rqu = zaxpby(ca, gqu, sac, gpu);
                        const Z rpv = zaxpby(ca, gpv, msa, gqv), rqv = zaxpby(ca, gqv, sac, gpv);
                        // columns: g_u = c g_u - conj(s) g_v, g_v = s g_u + c g_v
                        cu[p] = zaxpby(cb, rpu, msbc, rpv);
                        cv[p] = zaxpby(cb, rpv, sb, rpu);
                        cu[q] = zaxpby(cb, rqu, msbc, rqv);
                        cv[q] = zaxpby(cb, rqv, sb, rqu);
                    }
                    if (cb != 1.0 || sb.re != 0.0 || sb.im != 0.0) {
                        Z *vu = V + (size_t)u * np, *vv = V + (size_t)v * np;
                        for (int i = lane; i < np; i += 32) {
                            const Z x = vu[i], y = vv[i];
                            vu[i] = zaxpby(cb, x, msbc, y);
                            vv[i] = zaxpby(cb, y, sb, x);
                        }
                    }
                    (void)sbc;
                }
            }
            __syncthreads();
            if (!s_any) { converged = 1; break; }
        }
        __syncthreads();
        for (int j = threadIdx.x; j < n; j += blockDim.x) {
            const double dj = G[(size_t)j * np + j].re;
            int rk = 0;
            for (int i = 0; i < n; ++i) {
                const double di = G[(size_t)i * np + i].re;
                rk += (di < dj) || (di == dj && i < j);
            }
            perm[rk] = j;
        }
        __syncthreads();
        R *w = W + z * (int64_t)n;
        R *vo = Vout + z * (int64_t)n * n * 2;
        for (int k = threadIdx.x; k < n; k += blockDim.x) w[k] = (R)G[(size_t)perm[k] * np + perm[k]].re;
        for (int k = threadIdx.x; k < n * n; k += blockDim.x) {
            const int i = k / n, j = k - i * n;
            const Z x = V[(size_t)perm[j] * np + i];
            vo[2 * k] = (R)x.re;
            vo[2 * k + 1] = (R)x.im;
        }
        if (threadIdx.x == 0) {
            if (sweeps_out) sweeps_out[z] = sweep > max_sweeps ? max_sweeps : sweep;
            if (status) status[z] = converged ? JB_ST_OK : JB_ST_NOT_CONVERGED;
        }
    }
}

constexpr size_t kSmemLimit = 227 * 1024;

template <typename R>
static int zlaunch(const R *H, R *W, R *V, int32_t *sweeps, int32_t *status, int64_t batch, int n, double tol,
                   int max_sweeps, void *workspace, size_t ws_bytes, cudaStream_t st) {
    const int np = n + (n & 1);
    const int mode = zsmem_bytes(np, 2) <= kSmemLimit ? 2 : (zsmem_bytes(np, 1) <= kSmemLimit ? 1 : 0);
    const size_t smem = zsmem_bytes(np, mode);
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev))
        return JB_ECUDA;
    int64_t grid = batch < (int64_t)sms * 4 ? batch : (int64_t)sms * 4;
    Z *gv = nullptr;
    if (mode < 2) {
        const int64_t fit = (int64_t)(ws_bytes / ((size_t)np * np * 16 * (2 - mode)));
        if (!workspace || fit < 1) return JB_EWORKSPACE;
        if (grid > fit) grid = fit;
        gv = (Z *)workspace;
    }
    auto kern = zeigh_kernel<R>;
    if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
        return JB_ECUDA;
    kern<<<(unsigned)grid, kThreads, smem, st>>>(H, W, V, sweeps, status, batch, n, tol, max_sweeps, mode, gv);
    return cudaGetLastError() == cudaSuccess ? JB_OK : JB_ECUDA;
}

template <typename T>
static int launch(const T *H, T *W, T *V, int32_t *sweeps, int32_t *status, int64_t batch, int n, double tol,
                  int max_sweeps, void *workspace, size_t ws_bytes, cudaStream_t st) {
    const int np = n + (n & 1);
    const int mode = smem_bytes(np, 2) <= kSmemLimit ? 2 : (smem_bytes(np, 1) <= kSmemLimit ? 1 : 0);
    const size_t smem = smem_bytes(np, mode);
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev))
        return JB_ECUDA;
    int64_t grid = batch < (int64_t)sms * 4 ? batch : (int64_t)sms * 4;
    double *gv = nullptr;
    if (mode < 2) {
        const int64_t fit = (int64_t)(ws_bytes / ((size_t)np * np * 8 * (2 - mode)));
        if (!workspace || fit < 1) return JB_EWORKSPACE;
        if (grid > fit) grid = fit;
        gv = (double *)workspace;
    }
    auto kern = eigh_kernel<T>;
    if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
        return JB_ECUDA;
    kern<<<(unsigned)grid, kThreads, smem, st>>>(H, W, V, sweeps, status, batch, n, tol, max_sweeps, mode, gv);
    return cudaGetLastError() == cudaSuccess ? JB_OK : JB_ECUDA;
}

}  // namespace eigh
}  // namespace jb

extern "C" {

size_t jb_eigh_workspace_bytes(int32_t n, int64_t batch) {
    if (n < 1 || batch < 0) return 0;
    const int np = n + (n & 1);
    const int mode = jb::eigh::smem_bytes(np, 2) <= jb::eigh::kSmemLimit ? 2
                   : (jb::eigh::smem_bytes(np, 1) <= jb::eigh::kSmemLimit ? 1 : 0);
    if (mode == 2) return 0;
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev))
        sms = 148;
    const int64_t grid = batch < (int64_t)sms * 4 ? batch : (int64_t)sms * 4;
    return (size_t)grid * np * np * 8 * (2 - mode);
}

int jb_eigh_f32(const float *H, float *W, float *V, int32_t *sweeps, int32_t *status, int64_t batch, int32_t n,
                double tol, int32_t max_sweeps, void *workspace, size_t workspace_bytes, void *stream) {
    if (!H || !W || !V || batch < 0 || n < 1 || n > 255 || max_sweeps < 1) return JB_EINVAL;
    if (batch == 0) return JB_OK;
    if (tol <= 0) tol = 10.0 * 1.1920928955078125e-07;
    return jb::eigh::launch<float>(H, W, V, sweeps, status, batch, n, tol, max_sweeps, workspace, workspace_bytes,
                                   (cudaStream_t)stream);
}

size_t jb_eigh_complex_workspace_bytes(int32_t n, int64_t batch) {
    if (n < 1 || batch < 0) return 0;
    const int np = n + (n & 1);
    const int mode = jb::eigh::zsmem_bytes(np, 2) <= jb::eigh::kSmemLimit ? 2
                   : (jb::eigh::zsmem_bytes(np, 1) <= jb::eigh::kSmemLimit ? 1 : 0);
    if (mode == 2) return 0;
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev))
        sms = 148;
    const int64_t grid = batch < (int64_t)sms * 4 ? batch : (int64_t)sms * 4;
    return (size_t)grid * np * np * 16 * (2 - mode);
}

int jb_eigh_c64(const void *H, float *W, void *V, int32_t *sweeps, int32_t *status, int64_t batch, int32_t n,
                double tol, int32_t max_sweeps, void *workspace, size_t workspace_bytes, void *stream) {
    if (!H || !W || !V || batch < 0 || n < 1 || n > 255 || max_sweeps < 1) return JB_EINVAL;
    if (batch == 0) return JB_OK;
    if (tol <= 0) tol = 10.0 * 1.1920928955078125e-07;
    return jb::eigh::zlaunch<float>((const float *)H, W, (float *)V, sweeps, status, batch, n, tol, max_sweeps,
                                    workspace, workspace_bytes, (cudaStream_t)stream);
}

int jb_eigh_c128(const void *H, double *W, void *V, int32_t *sweeps, int32_t *status, int64_t batch, int32_t n,
                 double tol, int32_t max_sweeps, void *workspace, size_t workspace_bytes, void *stream) {
    if (!H || !W || !V || batch < 0 || n < 1 || n > 255 || max_sweeps < 1) return JB_EINVAL;
    if (batch == 0) return JB_OK;
    if (tol <= 0) tol = 10.0 * 2.220446049250313e-16;
    return jb::eigh::zlaunch<double>((const double *)H, W, (double *)V, sweeps, status, batch, n, tol, max_sweeps,
                                     workspace, workspace_bytes, (cudaStream_t)stream);
}

int jb_eigh_f64(const double *H, double *W, double *V, int32_t *sweeps, int32_t *status, int64_t batch, int32_t n,
                double tol, int32_t max_sweeps, void *workspace, size_t workspace_bytes, void *stream) {
    if (!H || !W || !V || batch < 0 || n < 1 || n > 255 || max_sweeps < 1) return JB_EINVAL;
    if (batch == 0) return JB_OK;
    if (tol <= 0) tol = 10.0 * 2.220446049250313e-16;
    return jb::eigh::launch<double>(H, W, V, sweeps, status, batch, n, tol, max_sweeps, workspace, workspace_bytes,
                                    (cudaStream_t)stream);
}

}  // extern "C"
