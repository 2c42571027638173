// jb_complex.cu - batched one-sided Jacobi SVD of complex matrices: the
// reference's jacobi_svd (svdbench/standalone/primitives.py:316-367) for
// complex64 / complex128, which its own tests run through 'jacobi'
// (tests/test_standalone.py:47-54, 68-80, 92-98).
//
// The reference's arithmetic, in the input precision: W = A (tall, a zero
// column padding odd n), V = I; per round of the round-robin tournament
// (primitives.py:309-313) and pair (p, q):
//   app = ||w_p||^2, aqq = ||w_q||^2, apq = w_p^H w_q
//   ratio = |apq| / max(sqrt(app) sqrt(aqq), tiny)
//   active = ratio > tol and min(app, aqq) > eps^2 max over the round's pairs
//            of max(app, aqq)
//   tau = (aqq - app) / (2 |apq|), t = sign(tau) / (|tau| + hypot(tau, 1))
//   (t = 1 at tau = 0), c = 1 / sqrt(1 + t^2), s = t c apq / |apq|
//   w_p <- c w_p - conj(s) w_q,  w_q <- s w_p + c w_q   (same for V)
// until a sweep finds no active pair; then sigma = column norms, sorted
// descending, cut at eps max(m, n_padded) sigma_1, U = W / sigma.  Null
// completion of cut columns, full bases and truncation are the host's, as
// in the reference's svd() (solvers.py:300-304).
//
// One CTA per matrix (grid-stride).  W (m x np) and V (np x np), complex,
// column-major, in shared memory when they fit, else in a per-CTA slot of
// the workspace.  A round: one warp per pair computes its three products
// (lanes over rows, warp reduction), a barrier, then each warp takes the
// round's floor (a max over the pairs' norms in shared memory), rotates its
// pair of W and V columns and records the largest active ratio.
#include <cuda_runtime.h>
#include <stdint.h>
#include <math.h>
#include "jacobi_b200.h"

namespace jb {
namespace cx {

constexpr int kThreads = 512;
constexpr size_t kSmemLimit = 227 * 1024;

template <typename R> struct C { R re, im; };

template <typename R> __device__ __forceinline__ R eps();
template <> __device__ __forceinline__ float eps<float>() { return 1.1920928955078125e-07f; }
template <> __device__ __forceinline__ double eps<double>() { return 2.220446049250313e-16; }
template <typename R> __device__ __forceinline__ R tiny();
template <> __device__ __forceinline__ float tiny<float>() { return 1.1754943508222875e-38f; }
template <> __device__ __forceinline__ double tiny<double>() { return 2.2250738585072014e-308; }

__device__ __forceinline__ float hyp(float a, float b) { return hypotf(a, b); }
__device__ __forceinline__ double hyp(double a, double b) { return hypot(a, b); }

template <typename R>
__device__ __forceinline__ R wsum(R v) {
#pragma unroll
    for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
template <typename R>
__device__ __forceinline__ R wmax(R v) {
#pragma unroll
    for (int o = 16; o; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// Pair k of round r of the circle-method tournament on np players: position
// 0 is fixed, positions 1..np-1 rotate one step right per round, pair k
// joins positions k and np-1-k (primitives.py:309-313).
__device__ __forceinline__ void rr_pair(int r, int k, int np, int &p, int &q) {
    auto player = [&](int pos) { return pos == 0 ? 0 : 1 + ((pos - 1 - r) % (np - 1) + (np - 1)) % (np - 1); };
    const int a = player(k), b = player(np - 1 - k);
    p = a < b ? a : b;
    q = a < b ? b : a;
}

__host__ __device__ inline size_t al16(size_t x) { return (x + 15) & ~(size_t)15; }

// Shared memory: red (32 doubles) | app, aqq (np/2 R each) | apq (np/2 C) |
// sig (np R) | perm (np int) | [W (m np C) | V (np np C)] when in_smem.
template <typename R>
__host__ __device__ inline size_t smem_bytes(int m, int np, bool in_smem) {
    const int h = np / 2;
    size_t b = 32 * 8 + al16(2 * (size_t)h * sizeof(R)) + al16((size_t)h * sizeof(C<R>)) + al16((size_t)np * sizeof(R)) +
               al16((size_t)np * 4);
    if (in_smem) b += ((size_t)m * np + (size_t)np * np) * sizeof(C<R>);
    return b;
}

template <typename R>
__global__ void __launch_bounds__(kThreads) cjacobi_kernel(const C<R> *A, C<R> *U, R *S, C<R> *Vh, int32_t *sweeps_out,
                                                           int32_t *status, int64_t batch, int m, int n, R tol,
                                                           int max_sweeps, int in_smem, C<R> *gws) {
    extern __shared__ __align__(16) unsigned char smem[];
    const int np = n + (n & 1), half = np / 2;
    double *red = (double *)smem;
    unsigned char *p8 = smem + 32 * 8;
    R *app = (R *)p8;
    R *aqq = app + half;
    p8 += al16(2 * (size_t)half * sizeof(R));
    C<R> *apq = (C<R> *)p8;
    p8 += al16((size_t)half * sizeof(C<R>));
    R *sig = (R *)p8;
    p8 += al16((size_t)np * sizeof(R));
    int *perm = (int *)p8;
    p8 += al16((size_t)np * 4);
    const size_t wsz = (size_t)m * np, vsz = (size_t)np * np;
    C<R> *W = in_smem ? (C<R> *)p8 : gws + (size_t)blockIdx.x * (wsz + vsz);
    C<R> *V = W + wsz;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    for (int64_t z = blockIdx.x; z < batch; z += gridDim.x) {
        const C<R> *a = A + z * (int64_t)m * n;
        __syncthreads();
        for (size_t idx = threadIdx.x; idx < wsz; idx += blockDim.x) {
            const int c = (int)(idx / m), i = (int)(idx - (size_t)c * m);
            W[idx] = c < n ? a[(size_t)i * n + c] : C<R>{R(0), R(0)};
        }
        for (size_t idx = threadIdx.x; idx < vsz; idx += blockDim.x) {
            const int c = (int)(idx / np), i = (int)(idx - (size_t)c * np);
            V[idx] = C<R>{i == c ? R(1) : R(0), R(0)};
        }
        __syncthreads();
        int sweep = 0;
        bool converged = false;
        for (sweep = 1; sweep <= max_sweeps; ++sweep) {
            R off = R(0);
            for (int r = 0; r < np - 1; ++r) {
                for (int k = warp; k < half; k += nw) {
                    int p, q;
                    rr_pair(r, k, np, p, q);
                    const C<R> *wp = W + (size_t)p * m, *wq = W + (size_t)q * m;
                    R sp = 0, sq = 0, cr = 0, ci = 0;
                    for (int i = lane; i < m; i += 32) {
                        const C<R> x = wp[i], y = wq[i];
                        sp += x.re * x.re + x.im * x.im;
                        sq += y.re * y.re + y.im * y.im;
                        cr += x.re * y.re + x.im * y.im;      // conj(x) y
                        ci += x.re * y.im - x.im * y.re;
                    }
                    sp = wsum(sp); sq = wsum(sq); cr = wsum(cr); ci = wsum(ci);
                    if (lane == 0) { app[k] = sp; aqq[k] = sq; apq[k] = C<R>{cr, ci}; }
                }
                __syncthreads();
                R mx = R(0);
                for (int k = lane; k < half; k += 32) mx = fmax(mx, fmax(app[k], aqq[k]));
                const R floor_ = eps<R>() * eps<R>() * wmax(mx);
                for (int k = warp; k < half; k += nw) {
                    const R ap = app[k], aq = aqq[k];
                    const C<R> g = apq[k];
                    const R ag = hyp(g.re, g.im);
                    const R den = sqrt(ap) * sqrt(aq);
                    const R ratio = ag / fmax(den, tiny<R>());
                    const bool active = ratio > tol && fmin(ap, aq) > floor_;
                    if (!active) continue;
                    off = fmax(off, ratio);
                    const R tau = (aq - ap) / (R(2) * ag);
                    R t = tau == R(0) ? R(1) : copysign(R(1), tau) / (fabs(tau) + hyp(tau, R(1)));
                    const R c = R(1) / sqrt(R(1) + t * t);
                    const R tc = t * c;
                    const C<R> s{tc * (g.re / ag), tc * (g.im / ag)};
                    int p, q;
                    rr_pair(r, k, np, p, q);
                    C<R> *wp = W + (size_t)p * m, *wq = W + (size_t)q * m;
                    for (int i = lane; i < m; i += 32) {
                        const C<R> x = wp[i], y = wq[i];
                        // c x - conj(s) y ; s x + c y
                        wp[i] = C<R>{c * x.re - (s.re * y.re + s.im * y.im), c * x.im - (s.re * y.im - s.im * y.re)};
                        wq[i] = C<R>{(s.re * x.re - s.im * x.im) + c * y.re, (s.re * x.im + s.im * x.re) + c * y.im};
                    }
                    C<R> *vp = V + (size_t)p * np, *vq = V + (size_t)q * np;
                    for (int i = lane; i < np; i += 32) {
                        const C<R> x = vp[i], y = vq[i];
                        vp[i] = C<R>{c * x.re - (s.re * y.re + s.im * y.im), c * x.im - (s.re * y.im - s.im * y.re)};
                        vq[i] = C<R>{(s.re * x.re - s.im * x.im) + c * y.re, (s.re * x.im + s.im * x.re) + c * y.im};
                    }
                }
                __syncthreads();
            }
            // off of the sweep: the largest active ratio over its rounds
            R o = wmax(off);
            if (lane == 0) red[warp] = (double)o;
            __syncthreads();
            double bo = 0;
            for (int w = 0; w < nw; ++w) bo = fmax(bo, red[w]);
            __syncthreads();
            if ((R)bo <= tol) { converged = true; break; }
        }
        // sigma, order (descending; ties by column), cut, outputs
        for (int c = warp; c < n; c += nw) {
            const C<R> *w = W + (size_t)c * m;
            R ssq = 0;
            for (int i = lane; i < m; i += 32) ssq += w[i].re * w[i].re + w[i].im * w[i].im;
            ssq = wsum(ssq);
            if (lane == 0) sig[c] = sqrt(ssq);
        }
        __syncthreads();
        for (int j = threadIdx.x; j < n; j += blockDim.x) {
            const R sj = sig[j];
            int rk = 0;
            for (int i = 0; i < n; ++i) rk += (sig[i] > sj) || (sig[i] == sj && i < j);
            perm[rk] = j;
        }
        __syncthreads();
        const R s1 = sig[perm[0]];
        const R cut = eps<R>() * (R)(m > np ? m : np) * s1;
        C<R> *u = U + z * (int64_t)m * n;
        for (size_t idx = threadIdx.x; idx < (size_t)m * n; idx += blockDim.x) {
            const int i = (int)(idx / n), k = (int)(idx - (size_t)i * n);
            const int c = perm[k];
            const R sc = sig[c];
            const C<R> w = W[(size_t)c * m + i];
            u[idx] = sc > cut ? C<R>{w.re / sc, w.im / sc} : C<R>{R(0), R(0)};
        }
        R *so = S + z * (int64_t)n;
        for (int k = threadIdx.x; k < n; k += blockDim.x) {
            const R sc = sig[perm[k]];
            so[k] = sc > cut ? sc : R(0);
        }
        C<R> *vh = Vh + z * (int64_t)n * n;
        for (int idx = threadIdx.x; idx < n * n; idx += blockDim.x) {
            const int k = idx / n, j = idx - k * n;            // Vh[k][j] = conj(V[j][perm k])
            const C<R> v = V[(size_t)perm[k] * np + j];
            vh[idx] = C<R>{v.re, -v.im};
        }
        if (threadIdx.x == 0) {
            if (sweeps_out) sweeps_out[z] = sweep > max_sweeps ? max_sweeps : sweep;
            if (status) status[z] = converged ? JB_ST_OK : JB_ST_NOT_CONVERGED;
        }
    }
}

static int sm_count() {
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev))
        return 0;
    return sms;
}

template <typename R>
static size_t workspace_bytes(int m, int n, int64_t batch) {
    const int np = n + (n & 1);
    if (smem_bytes<R>(m, np, true) <= kSmemLimit) return 0;
    int sms = sm_count();
    if (sms <= 0) sms = 148;
    const int64_t grid = batch < (int64_t)sms ? batch : (int64_t)sms;
    return (size_t)grid * ((size_t)m * np + (size_t)np * np) * sizeof(C<R>);
}

template <typename R>
static int entry(const void *A, void *U, R *S, void *Vh, int32_t *sweeps, int32_t *status, int64_t batch, int32_t m,
                 int32_t n, double tol, int32_t max_sweeps, void *workspace, size_t ws_bytes, void *stream) {
    if (!A || !U || !S || !Vh || batch < 0 || n < 1 || m < n || max_sweeps < 1) return JB_EINVAL;
    if ((int64_t)m * (n + 1) > ((int64_t)1 << 30)) return JB_ETOOBIG;
    if (batch == 0) return JB_OK;
    const int np = n + (n & 1);
    const bool in_smem = smem_bytes<R>(m, np, true) <= kSmemLimit;
    const size_t smem = smem_bytes<R>(m, np, in_smem);
    if (smem > kSmemLimit) return JB_ETOOBIG;
    auto kern = cjacobi_kernel<R>;
    if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
        return JB_ECUDA;
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kThreads, smem) != cudaSuccess) return JB_ECUDA;
    const int sms = sm_count();
    if (sms <= 0 || per_sm < 1) return JB_ECUDA;
    int64_t grid = (int64_t)sms * per_sm;
    if (grid > batch) grid = batch;
    C<R> *gws = nullptr;
    if (!in_smem) {
        const size_t per_cta = ((size_t)m * np + (size_t)np * np) * sizeof(C<R>);
        const int64_t fit = (int64_t)(ws_bytes / per_cta);
        if (!workspace || fit < 1) return JB_EWORKSPACE;
        if (grid > fit) grid = fit;
        gws = (C<R> *)workspace;
    }
    const R t = tol > 0 ? (R)tol : R(10) * (sizeof(R) == 4 ? (R)1.1920928955078125e-07 : (R)2.220446049250313e-16);
    kern<<<(unsigned)grid, kThreads, smem, (cudaStream_t)stream>>>((const C<R> *)A, (C<R> *)U, S, (C<R> *)Vh, sweeps,
                                                                   status, batch, m, n, t, max_sweeps, in_smem ? 1 : 0,
                                                                   gws);
    return cudaGetLastError() == cudaSuccess ? JB_OK : JB_ECUDA;
}

}  // namespace cx
}  // namespace jb

extern "C" {

size_t jb_svd_complex_workspace_bytes(int32_t m, int32_t n, int64_t batch, int32_t elem) {
    if (n < 1 || m < n || batch < 0) return 0;
    return elem == 16 ? jb::cx::workspace_bytes<double>(m, n, batch) : jb::cx::workspace_bytes<float>(m, n, batch);
}

int jb_svd_batched_c64(const void *A, void *U, float *S, void *Vh, int64_t batch, int32_t m, int32_t n, double tol,
                       int32_t max_sweeps, int32_t *sweeps, int32_t *status, void *workspace, size_t workspace_bytes,
                       void *stream) {
    return jb::cx::entry<float>(A, U, S, Vh, sweeps, status, batch, m, n, tol, max_sweeps, workspace,
                                workspace_bytes, stream);
}

int jb_svd_batched_c128(const void *A, void *U, double *S, void *Vh, int64_t batch, int32_t m, int32_t n,
                        double tol, int32_t max_sweeps, int32_t *sweeps, int32_t *status, void *workspace,
                        size_t workspace_bytes, void *stream) {
    return jb::cx::entry<double>(A, U, S, Vh, sweeps, status, batch, m, n, tol, max_sweeps, workspace,
                                 workspace_bytes, stream);
}

}  // extern "C"
