// jb_device.cuh - per-CTA building blocks of the batched one-sided Jacobi SVD.
//
// One CTA owns one matrix at a time.  The matrix is held as its TALL view
// (mt >= nt; a wide input is loaded transposed, svdbench/standalone/
// solvers.py:224-230) in a column-major work area W (mt x np, np = nt rounded
// up to even with a zero column, primitives.py:320-323) and V (np x np).  The
// work area lives in shared memory when it fits, else in a per-CTA slice of
// global workspace; the code below only sees generic pointers.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <math.h>
#include "jacobi_b200.h"

namespace jb {

constexpr unsigned FULL = 0xffffffffu;

template <typename T> struct Lim;
template <> struct Lim<float> {
    __device__ static float eps() { return 1.1920928955078125e-07f; }   // 2^-23
    __device__ static float tiny() { return 1.1754943508222875e-38f; }  // 2^-126
};
template <> struct Lim<double> {
    __device__ static double eps() { return 2.220446049250313e-16; }    // 2^-52
    __device__ static double tiny() { return 2.2250738585072014e-308; } // 2^-1022
};

__device__ __forceinline__ float  dsqrt(float x)  { return sqrtf(x); }
__device__ __forceinline__ double dsqrt(double x) { return sqrt(x); }
__device__ __forceinline__ float  dhypot(float a, float b)   { return hypotf(a, b); }
__device__ __forceinline__ double dhypot(double a, double b) { return hypot(a, b); }
__device__ __forceinline__ float  dabs(float x)  { return fabsf(x); }
__device__ __forceinline__ double dabs(double x) { return fabs(x); }
__device__ __forceinline__ float  dfma(float a, float b, float c)    { return fmaf(a, b, c); }
__device__ __forceinline__ double dfma(double a, double b, double c) { return fma(a, b, c); }
__device__ __forceinline__ float  dscale(float x, int e)  { return ldexpf(x, e); }
__device__ __forceinline__ double dscale(double x, int e) { return ldexp(x, e); }

template <typename T>
__device__ __forceinline__ T warp_max(T v) {
#pragma unroll
    for (int o = 16; o; o >>= 1) v = fmax(v, __shfl_xor_sync(FULL, v, o));
    return v;
}
template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
    for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(FULL, v, o);
    return v;
}

// Auxiliary per-CTA arrays, always in shared memory.
struct Aux {
    double *app, *aqq, *apq;  // per pair of the current round (np/2 each)
    double *sig;              // column norms / sorted singular values (np)
    double *vec;              // scratch vector (max(mt, np))
    double *tau;              // Householder scalars (np)
    int *perm;                // sorted position -> physical column (np)
    double *red;              // 64 reduction slots
    int *flag;                // 4 ints: [0] non-finite, [1] null-fail, [2] argmax idx
};

__device__ __forceinline__ int nwarps() { return (blockDim.x + 31) >> 5; }

// Maximum over the CTA; every thread gets the result.  Two barriers.
template <typename T>
__device__ T block_max(T v, double *red) {
    v = warp_max(v);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = (double)v;
    __syncthreads();
    double r = red[0];
    for (int w = 1; w < nwarps(); ++w) r = fmax(r, red[w]);
    __syncthreads();
    return (T)r;
}

template <typename T>
__device__ T block_sum(T v, double *red) {
    v = warp_sum(v);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = (double)v;
    __syncthreads();
    double r = 0;
    for (int w = 0; w < nwarps(); ++w) r += red[w];
    __syncthreads();
    return (T)r;
}

// Pair k of round r of the circle-method tournament on np players
// (primitives.py:309-313): position 0 is fixed, positions 1..np-1 rotate one
// step right per round, pair k joins positions k and np-1-k.
__device__ __forceinline__ void rr_pair(int r, int k, int np, int &p, int &q) {
    auto player = [&](int pos) { return pos == 0 ? 0 : 1 + ((pos - 1 - r) % (np - 1) + (np - 1)) % (np - 1); };
    int a = player(k), b = player(np - 1 - k);
    p = a < b ? a : b;
    q = a < b ? b : a;
}

// Problem geometry of one matrix (tall view).
struct Geo {
    int m, n;        // input shape (row-major)
    int mt, nt, np;  // tall view, padded even width
    bool wide;
    int rank, flags;
    int ncp;         // physical columns of W (np, or np + mt - nt with full bases)
    int ldw, ldv;    // leading dimensions (elements)
};

__device__ __forceinline__ Geo make_geo(int m, int n, int rank, int flags) {
    Geo g;
    g.m = m; g.n = n;
    g.wide = m < n;
    g.mt = g.wide ? n : m;
    g.nt = g.wide ? m : n;
    g.np = g.nt + (g.nt & 1);
    g.rank = rank; g.flags = flags;
    g.ncp = (flags & JB_FULL_MATRICES) ? g.np + (g.mt - g.nt) : g.np;
    g.ldw = g.mt | 1;  // odd stride spreads columns over banks
    g.ldv = g.np | 1;
    return g;
}

// Pass 1 over A: non-finite flag and exponent e with max|a| = f 2^e,
// f in [0.5, 1) (0 for a zero matrix).  Scaling by 2^-e is exact, unlike the
// reference's division by max|a| in the input precision (solvers.py:294-295);
// both only guard the sums of squares against overflow and underflow.
template <typename TI>
__device__ int scan_input(const TI *A, int count, Aux &ax, bool &bad) {
    double amax = 0.0;
    int nonfinite = 0;
    for (int i = threadIdx.x; i < count; i += blockDim.x) {
        double x = (double)A[i];
        if (!isfinite(x)) nonfinite = 1;
        else amax = fmax(amax, fabs(x));
    }
    nonfinite = __syncthreads_or(nonfinite);
    amax = block_max(amax, ax.red);
    bad = nonfinite != 0;
    int e = 0;
    if (amax > 0.0) frexp(amax, &e);
    return e;
}

// W[:, j] = (tall view of A)[:, j] * 2^-e for j < nt; padded and extra
// columns are zero.
template <typename T, typename TI>
__device__ void load_tall(const TI *A, const Geo &g, int e, T *W) {
    const int total = g.m * g.n;
    for (int idx = threadIdx.x; idx < total; idx += blockDim.x) {
        int r = idx / g.n, c = idx - r * g.n;     // input row r, column c
        int i = g.wide ? c : r, j = g.wide ? r : c;  // tall coordinates
        W[(size_t)j * g.ldw + i] = dscale((T)A[idx], -e);
    }
    for (int j = g.nt; j < g.ncp; ++j)
        for (int i = threadIdx.x; i < g.mt; i += blockDim.x) W[(size_t)j * g.ldw + i] = T(0);
}

template <typename T>
__device__ void set_identity(T *V, int np, int ldv) {
    for (int idx = threadIdx.x; idx < np * np; idx += blockDim.x) {
        int j = idx / np, i = idx - j * np;
        V[(size_t)j * ldv + i] = (i == j) ? T(1) : T(0);
    }
}

// Lanes per pair: largest power of two <= 32 that still gives every pair of
// a round its own lane group, at least 1.
__device__ __forceinline__ int group_size(int npairs) {
    int G = 32;
    while (G > 1 && npairs * G > (int)blockDim.x) G >>= 1;
    return G;
}

// Round-robin sweeps of one-sided Jacobi (primitives.py:328-355), one CTA.
// Returns the number of sweeps run; *converged tells whether off <= tol was
// reached.  Per round: phase 1 forms app, aqq, apq of every pair (group
// reductions) and the round's max column norm for the null-column floor
// (primitives.py:337); phase 2 applies the rotations (primitives.py:340-351).
template <typename T>
__device__ int sweeps(T *W, T *V, const Geo &g, T tol, int max_sweeps, Aux &ax, bool &converged) {
    const int np = g.np, mt = g.mt, npairs = np >> 1;
    const int G = group_size(npairs);
    const int ngroups = blockDim.x / G;
    const int gid = threadIdx.x / G, gl = threadIdx.x % G;
    const T eps2 = Lim<T>::eps() * Lim<T>::eps();
    converged = false;
    int sweep = 0;
    for (sweep = 1; sweep <= max_sweeps; ++sweep) {
        T off = T(0);
        for (int r = 0; r < np - 1; ++r) {
            T mymax = T(0);
            for (int base = 0; base < npairs; base += ngroups) {
                const int k = base + gid;
                const bool valid = k < npairs && gid < ngroups;
                T app = 0, aqq = 0, apq = 0;
                if (valid) {
                    int p, q;
                    rr_pair(r, k, np, p, q);
                    const T *wp = W + (size_t)p * g.ldw, *wq = W + (size_t)q * g.ldw;
                    for (int i = gl; i < mt; i += G) {
                        T x = wp[i], y = wq[i];
                        app = dfma(x, x, app);
                        aqq = dfma(y, y, aqq);
                        apq = dfma(x, y, apq);
                    }
                }
                for (int o = G >> 1; o; o >>= 1) {
                    app += __shfl_xor_sync(FULL, app, o);
                    aqq += __shfl_xor_sync(FULL, aqq, o);
                    apq += __shfl_xor_sync(FULL, apq, o);
                }
                if (valid) {
                    if (gl == 0) { ax.app[k] = app; ax.aqq[k] = aqq; ax.apq[k] = apq; }
                    mymax = fmax(mymax, fmax(app, aqq));
                }
            }
            mymax = warp_max(mymax);
            if ((threadIdx.x & 31) == 0) ax.red[threadIdx.x >> 5] = (double)mymax;
            __syncthreads();
            double rmax = ax.red[0];
            for (int w = 1; w < nwarps(); ++w) rmax = fmax(rmax, ax.red[w]);
            const T floor_ = eps2 * (T)rmax;
            for (int k = gid; k < npairs && gid < ngroups; k += ngroups) {
                const T app = (T)ax.app[k], aqq = (T)ax.aqq[k], apq = (T)ax.apq[k];
                const T den = dsqrt(app) * dsqrt(aqq);
                const T aapq = dabs(apq);
                const T ratio = aapq / fmax(den, Lim<T>::tiny());
                const bool active = ratio > tol && fmin(app, aqq) > floor_;
                if (!active) continue;
                off = fmax(off, ratio);
                const T tau = (aqq - app) / (T(2) * aapq);
                T t = T(1);
                if (tau != T(0)) t = copysign(T(1), tau) / (dabs(tau) + dhypot(tau, T(1)));
                const T c = T(1) / dsqrt(T(1) + t * t);
                T s = t * c;
                if (apq < T(0)) s = -s;
                int p, q;
                rr_pair(r, k, np, p, q);
                T *wp = W + (size_t)p * g.ldw, *wq = W + (size_t)q * g.ldw;
                for (int i = gl; i < mt; i += G) {
                    T x = wp[i], y = wq[i];
                    wp[i] = dfma(c, x, -s * y);
                    wq[i] = dfma(s, x, c * y);
                }
                T *vp = V + (size_t)p * g.ldv, *vq = V + (size_t)q * g.ldv;
                for (int i = gl; i < np; i += G) {
                    T x = vp[i], y = vq[i];
                    vp[i] = dfma(c, x, -s * y);
                    vq[i] = dfma(s, x, c * y);
                }
            }
            __syncthreads();
        }
        off = block_max(off, ax.red);
        if (off <= tol) { converged = true; break; }
    }
    return converged ? sweep : max_sweeps;
}

// Householder QR of the np x np matrix Q (column-major, ld ldq) in place,
// then Q is overwritten by the explicit orthonormal factor with its columns
// signed so that Q ~ input when the input is nearly orthogonal.  Follows
// householder_vec/qr of primitives.py:41-89 (xLARFG: beta = -sign(alpha)
// ||x||, backward accumulation).  `tmp` holds np x np doubles.
__device__ void householder_orthonormalize(double *Q, int np, int ldq, double *tmp, int ldt, Aux &ax) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = nwarps();
    double *beta_sign = ax.sig;  // reuse: sign(R_jj)
    for (int j = 0; j < np; ++j) {
        double *x = Q + (size_t)j * ldq;
        double part = 0.0;
        for (int i = j + 1 + threadIdx.x; i < np; i += blockDim.x) part = fma(x[i], x[i], part);
        const double xnorm = sqrt(block_sum(part, ax.red));
        const double alpha = x[j];
        const bool trivial = xnorm == 0.0;
        double beta = trivial ? alpha : -copysign(1.0, alpha == 0.0 ? 1.0 : alpha) * hypot(alpha, xnorm);
        const double tau = trivial ? 0.0 : (beta - alpha) / (beta != 0.0 ? beta : 1.0);
        const double denom = trivial ? 1.0 : alpha - beta;
        __syncthreads();
        for (int i = j + 1 + threadIdx.x; i < np; i += blockDim.x) x[i] = trivial ? 0.0 : x[i] / denom;
        if (threadIdx.x == 0) { ax.tau[j] = tau; beta_sign[j] = beta < 0.0 ? -1.0 : 1.0; x[j] = beta; }
        __syncthreads();
        // Apply (I - tau v v^T) to columns j+1.. of rows j.. ; v[0] = 1.
        for (int c = j + 1 + warp; c < np; c += nw) {
            double *y = Q + (size_t)c * ldq;
            double w = 0.0;
            for (int i = j + lane; i < np; i += 32) w = fma(i == j ? 1.0 : x[i], y[i], w);
            w = warp_sum(w) * tau;
            for (int i = j + lane; i < np; i += 32) y[i] -= w * (i == j ? 1.0 : x[i]);
        }
        __syncthreads();
    }
    // Backward accumulation into tmp: tmp = H_0 ... H_{np-1} I.
    for (int idx = threadIdx.x; idx < np * np; idx += blockDim.x) {
        int c = idx / np, i = idx - c * np;
        tmp[(size_t)c * ldt + i] = (i == c) ? 1.0 : 0.0;
    }
    __syncthreads();
    for (int j = np - 1; j >= 0; --j) {
        const double *v = Q + (size_t)j * ldq;
        const double tau = ax.tau[j];
        for (int c = j + warp; c < np; c += nw) {
            double *y = tmp + (size_t)c * ldt;
            double w = 0.0;
            for (int i = j + lane; i < np; i += 32) w = fma(i == j ? 1.0 : v[i], y[i], w);
            w = warp_sum(w) * tau;
            for (int i = j + lane; i < np; i += 32) y[i] -= w * (i == j ? 1.0 : v[i]);
        }
        __syncthreads();
    }
    for (int idx = threadIdx.x; idx < np * np; idx += blockDim.x) {
        int c = idx / np, i = idx - c * np;
        Q[(size_t)c * ldq + i] = tmp[(size_t)c * ldt + i] * beta_sign[c];
    }
    __syncthreads();
}

// Column norms, stable descending order, cut, U = W / sigma, null-space
// completion (primitives.py:356-366 and :430-467, complete_basis for full
// bases) and the output writes of svd() (solvers.py:299-310).
//   W: mt x ncp physical columns; sorted position r < nt lives in physical
//   column perm[r], full-basis positions r >= nt in column np + (r - nt).
template <typename T, typename TO>
__device__ int epilogue(T *W, T *V, const Geo &g, int e, TO *U_out, TO *S_out, TO *Vh_out, Aux &ax) {
    const int mt = g.mt, nt = g.nt, np = g.np;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = nwarps();
    const bool full = (g.flags & JB_FULL_MATRICES) != 0;
    const bool want_vec = (g.flags & JB_VALUES_ONLY) == 0;
    // sigma_j = ||W[:, j]|| (primitives.py:356)
    for (int j = warp; j < nt; j += nw) {
        const T *w = W + (size_t)j * g.ldw;
        T acc = 0;
        for (int i = lane; i < mt; i += 32) acc = dfma(w[i], w[i], acc);
        acc = warp_sum(acc);
        if (lane == 0) ax.sig[j] = (double)dsqrt(acc);
    }
    __syncthreads();
    // Stable descending sort by rank counting (primitives.py:359-361).
    for (int j = threadIdx.x; j < nt; j += blockDim.x) {
        const double sj = ax.sig[j];
        int rnk = 0;
        for (int i = 0; i < nt; ++i) {
            const double si = ax.sig[i];
            rnk += (si > sj) || (si == sj && i < j);
        }
        ax.perm[rnk] = j;
    }
    __syncthreads();
    // cut = eps * max(m, n_padded) * sigma_1 (primitives.py:362; the
    // reference's n is the padded width there).
    const T smax = (T)ax.sig[ax.perm[0]];
    const int npref = nt + (nt & 1);
    const T cut = Lim<T>::eps() * (T)(mt > npref ? mt : npref) * smax;
    // Normalise kept columns in place, zero the others (primitives.py:364, :436).
    int any_missing = 0;
    for (int r = warp; r < nt; r += nw) {
        const int j = ax.perm[r];
        const T sj = (T)ax.sig[j];
        T *w = W + (size_t)j * g.ldw;
        const bool keep = sj > cut;
        for (int i = lane; i < mt; i += 32) w[i] = keep ? w[i] / sj : T(0);
        if (!keep) any_missing = 1;
    }
    // Zero the padding column (never rotated, already zero) and extra columns.
    any_missing = __syncthreads_or(any_missing) || (full && mt > nt);
    const int kcols = full ? mt : nt;  // sorted positions of the U basis
    if (any_missing && want_vec) {
        // complete_null_columns: sequential over sorted positions.
        for (int r = 0; r < kcols; ++r) {
            bool missing;
            int col;
            if (r < nt) {
                col = ax.perm[r];
                missing = !((T)ax.sig[col] > cut);
            } else {
                col = np + (r - nt);
                missing = true;
            }
            if (!missing) continue;
            // leverage_i = 1 - sum_c |U[i, c]|^2 ; idx = first argmax.
            double best = -1e300;
            int bidx = 0;
            for (int i = threadIdx.x; i < mt; i += blockDim.x) {
                T acc = 0;
                for (int c = 0; c < g.ncp; ++c) { T u = W[(size_t)c * g.ldw + i]; acc = dfma(u, u, acc); }
                const double lev = (double)(T(1) - acc);
                if (lev > best) { best = lev; bidx = i; }
            }
            // Warp argmax with first-index tie break.
            for (int o = 16; o; o >>= 1) {
                double ob = __shfl_xor_sync(FULL, best, o);
                int oi = __shfl_xor_sync(FULL, bidx, o);
                if (ob > best || (ob == best && oi < bidx)) { best = ob; bidx = oi; }
            }
            if (lane == 0) { ax.red[warp] = best; ax.vec[warp] = (double)bidx; }
            __syncthreads();
            if (threadIdx.x == 0) {
                double b = ax.red[0];
                int bi = (int)ax.vec[0];
                for (int w = 1; w < nw; ++w) {
                    const double ob = ax.red[w];
                    const int oi = (int)ax.vec[w];
                    if (ob > b || (ob == b && oi < bi)) { b = ob; bi = oi; }
                }
                ax.flag[2] = bi;
            }
            __syncthreads();
            const int idx = ax.flag[2];
            // v = e_idx, stored in physical column `col` (currently zero).
            T *v = W + (size_t)col * g.ldw;
            for (int i = threadIdx.x; i < mt; i += blockDim.x) v[i] = (i == idx) ? T(1) : T(0);
            __syncthreads();
            for (int pass = 0; pass < 2; ++pass) {
                // y = U^T v over all physical columns (v's own column is
                // included by the reference too: it holds zeros there, here
                // it holds v, so skip it to keep the same arithmetic).
                for (int c = warp; c < g.ncp; c += nw) {
                    T acc = 0;
                    if (c != col) {
                        const T *u = W + (size_t)c * g.ldw;
                        for (int i = lane; i < mt; i += 32) acc = dfma(u[i], v[i], acc);
                        acc = warp_sum(acc);
                    }
                    if (lane == 0) ax.vec[c] = (double)acc;
                }
                __syncthreads();
                for (int i = threadIdx.x; i < mt; i += blockDim.x) {
                    T acc = 0;
                    for (int c = 0; c < g.ncp; ++c)
                        if (c != col) acc = dfma(W[(size_t)c * g.ldw + i], (T)ax.vec[c], acc);
                    v[i] -= acc;
                }
                __syncthreads();
            }
            T part = 0;
            for (int i = threadIdx.x; i < mt; i += blockDim.x) part = dfma(v[i], v[i], part);
            const T len = dsqrt(block_sum(part, ax.red));
            if (len < T(10) * Lim<T>::eps()) {
                if (threadIdx.x == 0) ax.flag[1] = 1;
            }
            const T inv = fmax(len, Lim<T>::tiny());
            for (int i = threadIdx.x; i < mt; i += blockDim.x) v[i] = v[i] / inv;
            __syncthreads();
        }
    }
    __syncthreads();
    // Outputs.  S: sorted sigma * 2^e, cut values zeroed (primitives.py:366).
    int nonfinite = 0;
    for (int r = threadIdx.x; r < g.rank; r += blockDim.x) {
        const int j = ax.perm[r];
        const T sj = (T)ax.sig[j];
        const T val = sj > cut ? dscale(sj, e) : T(0);
        const TO o = (TO)val;
        if (!isfinite((double)o)) nonfinite = 1;
        S_out[r] = o;
    }
    if (want_vec) {
        const int ucols = full ? g.m : g.rank;   // output U is m x ucols
        const int vrows = full ? g.n : g.rank;   // output Vh is vrows x n
        if (!g.wide) {
            // U_out[i, r] = U_t[i, r]; Vh_out[r, i] = V[i, perm[r]].
            for (int idx = threadIdx.x; idx < mt * ucols; idx += blockDim.x) {
                const int i = idx / ucols, r = idx - i * ucols;
                const int col = r < nt ? ax.perm[r] : np + (r - nt);
                const TO o = (TO)W[(size_t)col * g.ldw + i];
                if (!isfinite((double)o)) nonfinite = 1;
                U_out[idx] = o;
            }
            for (int idx = threadIdx.x; idx < vrows * nt; idx += blockDim.x) {
                const int r = idx / nt, i = idx - r * nt;
                const TO o = (TO)V[(size_t)ax.perm[r] * g.ldv + i];
                if (!isfinite((double)o)) nonfinite = 1;
                Vh_out[idx] = o;
            }
        } else {
            // A = V_t S U_t^T: U_out (m = nt rows) = V_t, Vh_out (n = mt cols) = U_t^T.
            for (int idx = threadIdx.x; idx < nt * ucols; idx += blockDim.x) {
                const int i = idx / ucols, r = idx - i * ucols;
                const TO o = (TO)V[(size_t)ax.perm[r] * g.ldv + i];
                if (!isfinite((double)o)) nonfinite = 1;
                U_out[idx] = o;
            }
            for (int idx = threadIdx.x; idx < vrows * mt; idx += blockDim.x) {
                const int r = idx / mt, i = idx - r * mt;
                const int col = r < nt ? ax.perm[r] : np + (r - nt);
                const TO o = (TO)W[(size_t)col * g.ldw + i];
                if (!isfinite((double)o)) nonfinite = 1;
                Vh_out[idx] = o;
            }
        }
    }
    nonfinite = __syncthreads_or(nonfinite);
    if (ax.flag[1]) return JB_ST_NULL_FAILED;
    return nonfinite ? JB_ST_NONFINITE_OUT : JB_ST_OK;
}

}  // namespace jb
