// jb_lab.cu - rounds of the one-sided Jacobi applied in place to ONE
// matrix's W (m x n, m >= n) and V (n x n), both row-major as the caller's
// tensors: the laboratory's jacobi_rotation
// (algorithm_laboratory/algorithms.py:81-102) for a range of rounds of its
// schedule (:121-126, the round-robin tournament of primitives.py:309-313 on
// n + n % 2 players with the pairs that reach past n dropped).  It lets the
// laboratory's jacobi (:105-157) run on the GPU while its trace still sees
// W and V after every sweep, or after every round.
//
// Per round: one warp per pair forms app, aqq, apq (w_p^H w_q), a barrier,
// then every warp takes the round's floor eps^2 max(app, aqq) over its pairs,
// rotates its pair of W and V columns when ratio > tol and min(app, aqq) >
// floor, with c = rsqrt(1 + t^2) and s = t c apq / |apq| as the laboratory
// writes them, and keeps the largest active ratio.  At the end the CTA's
// largest active ratio is folded into *off (a max), so one call per round or
// per sweep gives the laboratory's per-sweep off.  Real inputs run through
// the same complex formulas with zero imaginary parts, which add nothing.
// One CTA (the laboratory solves one matrix at a time); W and V are copied to
// shared memory (column-major) for the launch when they fit, and back after.
#include <cuda_runtime.h>
#include <stdint.h>
#include <math.h>
#include <type_traits>
#include "jacobi_b200.h"

namespace jb {
namespace lab {

constexpr int kThreads = 512;

template <typename R> struct C { R re, im; };

template <typename R> __device__ __forceinline__ R eps();
template <> __device__ __forceinline__ float eps<float>() { return 1.1920928955078125e-07f; }
template <> __device__ __forceinline__ double eps<double>() { return 2.220446049250313e-16; }
template <typename R> __device__ __forceinline__ R tiny();
template <> __device__ __forceinline__ float tiny<float>() { return 1.1754943508222875e-38f; }
template <> __device__ __forceinline__ double tiny<double>() { return 2.2250738585072014e-308; }
__device__ __forceinline__ float hyp(float a, float b) { return hypotf(a, b); }
__device__ __forceinline__ double hyp(double a, double b) { return hypot(a, b); }
__device__ __forceinline__ float rs(float x) { return rsqrtf(x); }
__device__ __forceinline__ double rs(double x) { return rsqrt(x); }

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

template <typename R, bool CPLX>
__device__ __forceinline__ C<R> ld(const void *p, size_t i) {
    if constexpr (CPLX) return ((const C<R> *)p)[i];
    else return C<R>{((const R *)p)[i], R(0)};
}
template <typename R, bool CPLX>
__device__ __forceinline__ void st(void *p, size_t i, C<R> v) {
    if constexpr (CPLX) ((C<R> *)p)[i] = v;
    else ((R *)p)[i] = v.re;
}

__device__ __forceinline__ void rr_pair(int r, int k, int np, int &p, int &q) {
    auto player = [&](int pos) { return pos == 0 ? 0 : 1 + ((pos - 1 - r) % (np - 1) + (np - 1)) % (np - 1); };
    const int a = player(k), b = player(np - 1 - k);
    p = a < b ? a : b;
    q = a < b ? b : a;
}

template <typename R, bool CPLX>
__host__ __device__ inline size_t pair_bytes(int n) {
    const int half = (n + (n & 1)) / 2;
    return ((size_t)(2 * half + (half & 1)) * sizeof(R) + (size_t)half * sizeof(C<R>) + 15) & ~(size_t)15;
}

// Element (i, col) of a matrix with `rows` rows: column-major in shared
// memory, row-major (n columns) in the caller's arrays.
__device__ __forceinline__ size_t at(bool staged, int i, int col, int rows, int n) {
    return staged ? (size_t)col * rows + i : (size_t)i * n + col;
}

template <typename R, bool CPLX>
__global__ void __launch_bounds__(kThreads) rounds_kernel(void *Wg, void *Vg, int m, int n, int r0, int r1, R tol,
                                                          double *off_out, int staged) {
    extern __shared__ __align__(16) unsigned char smem[];
    const int np = n + (n & 1), half = np / 2;
    R *app = (R *)smem;
    R *aqq = app + half;
    C<R> *apq = (C<R> *)(aqq + half + (half & 1));   // an even count of R before it
    __shared__ double red[32];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    using E = typename std::conditional<CPLX, C<R>, R>::type;
    void *W = Wg, *V = Vg;
    if (staged) {
        E *ws = (E *)(smem + pair_bytes<R, CPLX>(n)), *vs = ws + (size_t)m * n;
        for (size_t k = threadIdx.x; k < (size_t)m * n; k += blockDim.x) {
            const int i = (int)(k / n), c = (int)(k - (size_t)i * n);
            ws[(size_t)c * m + i] = ((const E *)Wg)[k];
        }
        for (size_t k = threadIdx.x; k < (size_t)n * n; k += blockDim.x) {
            const int i = (int)(k / n), c = (int)(k - (size_t)i * n);
            vs[(size_t)c * n + i] = ((const E *)Vg)[k];
        }
        W = ws;
        V = vs;
        __syncthreads();
    }
    R off = R(0);
    for (int r = r0; r < r1; ++r) {
        for (int k = warp; k < half; k += nw) {
            int p, q;
            rr_pair(r, k, np, p, q);
            if (q >= n) continue;                      // dropped pair
            R sp = 0, sq = 0, cr = 0, ci = 0;
            for (int i = lane; i < m; i += 32) {
                const C<R> x = ld<R, CPLX>(W, at(staged, i, p, m, n)), y = ld<R, CPLX>(W, at(staged, i, q, m, n));
                sp += x.re * x.re + x.im * x.im;
                sq += y.re * y.re + y.im * y.im;
                cr += x.re * y.re + x.im * y.im;
                ci += x.re * y.im - x.im * y.re;
            }
            sp = wsum(sp); sq = wsum(sq); cr = wsum(cr); ci = wsum(ci);
            if (lane == 0) { app[k] = sp; aqq[k] = sq; apq[k] = C<R>{cr, ci}; }
        }
        __syncthreads();
        R mx = R(0);
        for (int k = lane; k < half; k += 32) {
            int p, q;
            rr_pair(r, k, np, p, q);
            if (q < n) mx = fmax(mx, fmax(app[k], aqq[k]));
        }
        const R floor_ = eps<R>() * eps<R>() * wmax(mx);
        for (int k = warp; k < half; k += nw) {
            int p, q;
            rr_pair(r, k, np, p, q);
            if (q >= n) continue;
            const R ap = app[k], aq = aqq[k];
            const C<R> g = apq[k];
            const R ag = hyp(g.re, g.im);
            const R ratio = ag / fmax(sqrt(ap) * sqrt(aq), tiny<R>());
            if (!(ratio > tol && fmin(ap, aq) > floor_)) continue;
            off = fmax(off, ratio);
            const R tau = (aq - ap) / (R(2) * ag);
            const R t = tau == R(0) ? R(1) : copysign(R(1), tau) / (fabs(tau) + hyp(tau, R(1)));
            const R c = rs(R(1) + t * t);
            const R tc = t * c;
            const C<R> s{tc * (g.re / ag), tc * (g.im / ag)};
            for (int pass = 0; pass < 2; ++pass) {
                void *X = pass == 0 ? W : V;
                const int rows = pass == 0 ? m : n;
                for (int i = lane; i < rows; i += 32) {
                    const size_t ip = at(staged, i, p, rows, n), iq = at(staged, i, q, rows, n);
                    const C<R> x = ld<R, CPLX>(X, ip), y = ld<R, CPLX>(X, iq);
                    st<R, CPLX>(X, ip,
                                C<R>{c * x.re - (s.re * y.re + s.im * y.im), c * x.im - (s.re * y.im - s.im * y.re)});
                    st<R, CPLX>(X, iq,
                                C<R>{(s.re * x.re - s.im * x.im) + c * y.re, (s.re * x.im + s.im * x.re) + c * y.im});
                }
            }
        }
        __syncthreads();
    }
    if (staged) {
        const E *ws = (const E *)W, *vs = (const E *)V;
        for (size_t k = threadIdx.x; k < (size_t)m * n; k += blockDim.x) {
            const int i = (int)(k / n), c = (int)(k - (size_t)i * n);
            ((E *)Wg)[k] = ws[(size_t)c * m + i];
        }
        for (size_t k = threadIdx.x; k < (size_t)n * n; k += blockDim.x) {
            const int i = (int)(k / n), c = (int)(k - (size_t)i * n);
            ((E *)Vg)[k] = vs[(size_t)c * n + i];
        }
    }
    const R o = wmax(off);
    if (lane == 0) red[warp] = (double)o;
    __syncthreads();
    if (threadIdx.x == 0) {
        double b = *off_out;
        for (int w = 0; w < nw; ++w) b = fmax(b, red[w]);
        *off_out = b;
    }
}

template <typename R, bool CPLX>
static int launch(void *W, void *V, int m, int n, int r0, int r1, double tol, double *off, cudaStream_t st) {
    const size_t esz = CPLX ? sizeof(C<R>) : sizeof(R);
    const size_t base = pair_bytes<R, CPLX>(n), work = ((size_t)m * n + (size_t)n * n) * esz;
    const bool staged = base + work <= 227 * 1024;
    const size_t smem = staged ? base + work : base;
    auto kern = rounds_kernel<R, CPLX>;
    if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
        return JB_ECUDA;
    kern<<<1, kThreads, smem, st>>>(W, V, m, n, r0, r1, (R)tol, off, staged ? 1 : 0);
    return cudaGetLastError() == cudaSuccess ? JB_OK : JB_ECUDA;
}

}  // namespace lab
}  // namespace jb

extern "C" {

int jb_jacobi_rounds(void *W, void *V, int32_t dtype, int32_t m, int32_t n, int32_t round_begin, int32_t round_end,
                     double tol, double *off, void *stream) {
    if (!W || !V || !off || n < 1 || m < n || n > 8192 || !(tol > 0)) return JB_EINVAL;
    const int np = n + (n & 1);
    if (round_begin < 0 || round_end < round_begin || round_end > np - 1) return JB_EINVAL;
    if (round_end == round_begin) return JB_OK;
    cudaStream_t st = (cudaStream_t)stream;
    switch (dtype) {
        case 0: return jb::lab::launch<float, false>(W, V, m, n, round_begin, round_end, tol, off, st);
        case 1: return jb::lab::launch<double, false>(W, V, m, n, round_begin, round_end, tol, off, st);
        case 2: return jb::lab::launch<float, true>(W, V, m, n, round_begin, round_end, tol, off, st);
        case 3: return jb::lab::launch<double, true>(W, V, m, n, round_begin, round_end, tol, off, st);
        default: return JB_EINVAL;
    }
}

}  // extern "C"
