// jb_gram64.cuh - the FP64 phase of the mixed solve for large tiles (one
// matrix of up to 256 x 128 in its tall view per CTA).
//
// The FP32 sweeps (rb32_kernel_t, large tile) leave V with every pair ratio of
// W = A V below ~1e-2 after the last rotating sweep.  This phase:
//   V <- V (3I - V^T V) / 2           (Newton-Schulz, V orthogonal in FP64)
//   W  = A_t V                         (A_t: the exactly scaled tall view)
//   G  = W^T W                         (FP64)
//   Jacobi sweeps on G (G <- J^T G J)  until a sweep finds no active pair --
//      the reference's test |g_pq| / sqrt(g_pp g_qq) > tol on the Gram of
//      the current W (primitives.py:334-338, 352-353); J are the one-sided
//      rotations of the columns of W (primitives.py:340-347), applied to G
//      from both sides, and their product is kept as D = Q - I in FP32 (the
//      rotations here are small, so D carries FP64-level accuracy of Q)
//   W <- W (I + D), V <- V (I + D)
// then the common epilogue.  Every product above is a staged FP64 GEMM; the
// sweeps touch only the n x n Gram in shared memory instead of the m x n
// columns of W, which for these shapes do not fit in shared memory in FP64.
#pragma once
#include "jb_device.cuh"

namespace jb {

constexpr int kTG = 1024;      // threads of the Gram kernel
constexpr int kGemmKC = 8;     // K chunk staged per step

// C (M x N) = alpha * op(A) B + beta * C, all column-major FP64 except B
// (TB).  op(A) = A (A: M x K, lda) or A^T (A stored K x M, lda).  stage:
// kGemmKC * (M + N) doubles of shared memory.  4 x 4 outputs per thread and
// pass; every thread takes part (barriers inside).
template <bool TRANS_A, typename TB>
__device__ void gemm64(const double *A, int lda, const TB *B, int ldb, double *C, int ldc, int M, int N, int K,
                       double alpha, double beta, double *stage) {
    const int tm = (M + 3) >> 2, tn = (N + 3) >> 2, tiles = tm * tn;
    double *As = stage;                      // [kc][M]
    double *Bs = stage + kGemmKC * M;        // [kc][N]
    for (int t0 = 0; t0 < tiles; t0 += blockDim.x) {
        const int t = t0 + threadIdx.x;
        const bool own = t < tiles;
        const int i0 = own ? (t % tm) * 4 : 0, j0 = own ? (t / tm) * 4 : 0;
        double acc[4][4];
#pragma unroll
        for (int x = 0; x < 4; ++x)
#pragma unroll
            for (int y = 0; y < 4; ++y) acc[x][y] = 0.0;
        for (int k0 = 0; k0 < K; k0 += kGemmKC) {
            const int kc = min(kGemmKC, K - k0);
            __syncthreads();
            for (int idx = threadIdx.x; idx < kc * M; idx += blockDim.x) {
                if (TRANS_A) {                       // A^T(i, k) = A[i * lda + k]: k fastest
                    const int i = idx / kc, k = idx - i * kc;
                    As[k * M + i] = A[(size_t)i * lda + k0 + k];
                } else {                             // A(i, k) = A[k * lda + i]: i fastest
                    const int k = idx / M, i = idx - k * M;
                    As[k * M + i] = A[(size_t)(k0 + k) * lda + i];
                }
            }
            for (int idx = threadIdx.x; idx < kc * N; idx += blockDim.x) {
                const int j = idx / kc, k = idx - j * kc;
                Bs[k * N + j] = (double)B[(size_t)j * ldb + k0 + k];
            }
            __syncthreads();
            if (own) {
                for (int k = 0; k < kc; ++k) {
                    double a[4], b[4];
#pragma unroll
                    for (int x = 0; x < 4; ++x) {
                        a[x] = i0 + x < M ? As[k * M + i0 + x] : 0.0;
                        b[x] = j0 + x < N ? Bs[k * N + j0 + x] : 0.0;
                    }
#pragma unroll
                    for (int x = 0; x < 4; ++x)
#pragma unroll
                        for (int y = 0; y < 4; ++y) acc[x][y] = fma(a[x], b[y], acc[x][y]);
                }
            }
        }
        if (own) {
#pragma unroll
            for (int y = 0; y < 4; ++y) {
                const int j = j0 + y;
                if (j >= N) continue;
#pragma unroll
                for (int x = 0; x < 4; ++x) {
                    const int i = i0 + x;
                    if (i >= M) continue;
                    double *c = C + (size_t)j * ldc + i;
                    *c = beta != 0.0 ? fma(alpha, acc[x][y], beta * *c) : alpha * acc[x][y];
                }
            }
        }
    }
    __syncthreads();
}

// Shared memory of the Gram phase after the aux area, for a padded width np:
// G (np^2 FP64) | D (np^2 FP32) | c/s (np FP64) | pairs (np) | round-robin
// table ((np - 1) np).  The GEMM staging (kGemmKC (mt + np) FP64) lives in D
// before the sweeps and in G after them, so both regions are at least that
// large (gram64_regions).
__host__ __device__ inline void gram64_regions(int np, int mt, size_t &g, size_t &dd) {
    const size_t st = (size_t)kGemmKC * (mt + np) * 8;
    g = (size_t)np * np * 8;
    dd = (size_t)np * np * 4;
    g = ((g > st ? g : st) + 15) & ~(size_t)15;
    dd = ((dd > st ? dd : st) + 15) & ~(size_t)15;
}
__host__ __device__ inline size_t gram64_smem(int np, int mt) {
    size_t g, dd;
    gram64_regions(np, mt, g, dd);
    const size_t rr = (size_t)np * 8 + (size_t)np + (size_t)(np > 1 ? np - 1 : 1) * np;
    return g + dd + rr + 64;
}

// Jacobi on the n x n Gram G (FP64, column-major in shared memory) with D =
// Q - I (FP32) accumulated; round-robin pairs (primitives.py:309-313), the
// reference's active test and rotation.  Returns the sweeps taken (the last
// one found no active pair) or max_sweeps + 1 when it did not converge.
__device__ int gram_sweeps(double *G, float *D, int n, double tol, int max_sweeps, unsigned char *sched,
                           unsigned char *pq, double *cs, int *any_flag) {
    const int half = n / 2;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    for (int i = threadIdx.x; i < (n - 1) * n; i += blockDim.x) {
        const int r = i / n, pos = i - r * n;
        sched[i] = (unsigned char)circ(pos, r, n);
    }
    for (int i = threadIdx.x; i < n * n; i += blockDim.x) D[i] = 0.f;
    __syncthreads();
    double gmax = 0.0;
    for (int i = 0; i < n; ++i) gmax = fmax(gmax, G[(size_t)i * n + i]);
    const double floor_ = Lim<double>::eps() * Lim<double>::eps() * gmax;
    const double tol2 = tol * tol;
    for (int sweep = 1; sweep <= max_sweeps; ++sweep) {
        __syncthreads();
        if (threadIdx.x == 0) *any_flag = 0;
        for (int r = 0; r < n - 1; ++r) {
            __syncthreads();
            for (int t = threadIdx.x; t < half; t += blockDim.x) {
                int p = sched[r * n + t], q = sched[r * n + n - 1 - t];
                if (p > q) { const int x = p; p = q; q = x; }
                const double app = G[(size_t)p * n + p], aqq = G[(size_t)q * n + q], apq = G[(size_t)q * n + p];
                double c = 1.0, s = 0.0;
                if (apq * apq > tol2 * app * aqq && fmin(app, aqq) > floor_) {
                    const double d = aqq - app;
                    const double tt = copysign(2.0 * fabs(apq), d) / (fabs(d) + sqrt(d * d + 4.0 * apq * apq));
                    c = 1.0 / sqrt(1.0 + tt * tt);
                    s = tt * c;
                    if (apq < 0.0) s = -s;
                    *any_flag = 1;
                }
                cs[t] = c;
                cs[half + t] = s;
                pq[t] = (unsigned char)p;
                pq[half + t] = (unsigned char)q;
            }
            __syncthreads();
            // G <- J^T G J (2 x 2 blocks: row pair a, column pair b)
            for (int b = warp; b < half; b += nw) {
                const int u = pq[b], v = pq[half + b];
                const double cb = cs[b], sb = cs[half + b];
                double *cu = G + (size_t)u * n, *cv = G + (size_t)v * n;
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
                // D <- D J + (J - I): columns u, v rotated, then the rotation's
                // own deviation from I (c - 1 = -s^2 / (1 + c), exact for small s)
                if (cb != 1.0 || sb != 0.0) {
                    const float fc = (float)cb, fs = (float)sb;
                    float *du = D + (size_t)u * n, *dv = D + (size_t)v * n;
                    for (int i = lane; i < n; i += 32) {
                        const float x = du[i], y = dv[i];
                        du[i] = fc * x - fs * y;
                        dv[i] = fs * x + fc * y;
                    }
                    __syncwarp();
                    if (lane == 0) {
                        const float cm1 = (float)(-sb * sb / (1.0 + cb));
                        du[u] += cm1;
                        du[v] += -fs;
                        dv[u] += fs;
                        dv[v] += cm1;
                    }
                    __syncwarp();
                }
            }
        }
        __syncthreads();
        if (!*any_flag) return sweep;
    }
    return max_sweeps + 1;
}

}  // namespace jb
