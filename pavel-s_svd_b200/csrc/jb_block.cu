// jb_block.cu - the non-GEMM kernels of the blocked one-sided Jacobi SVD
// (svdbench/standalone/solvers.py:30-68, block_jacobi).
//
// Block pairs live in "slots": slot k of a round holds the 2b columns of its
// pair (block i, then block j, i < j) as 2b rows of length L (columns of W
// are rows of W^T), in hi/lo BF16 parts that feed the tensor-core products.
//   jb_block_eig_f64   FP64 eigen-solve of every slot's Gram (2b x 2b):
//                      the rotation vv of the reference's inner Jacobi
//                      (solvers.py:48), written as vv^T in hi/lo BF16.
//   jb_rows_scatter    FP32 rows -> hi/lo BF16 rows at mapped positions
//                      (moves rotated blocks into the next round's slots).
//   jb_rows_combine    hi + lo BF16 rows -> FP32 rows at mapped positions.
//   jb_block_finish    sigma = column norms (FP64), descending order, cut,
//                      U = W / sigma, Vh (solvers.py:61-66 with
//                      _finish_columns :18-21).
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>
#include <math.h>
#include "jacobi_b200.h"

namespace jb {
namespace blk {

__device__ __forceinline__ double warp_sum_d(double v) {
    for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

__device__ __forceinline__ int circ(int pos, int r, int n) {
    if (pos == 0) return 0;
    int x = (pos - 1 - r) % (n - 1);
    if (x < 0) x += n - 1;
    return 1 + x;
}

constexpr int kEigThreads = 512;

// Shared-memory bytes of eig_kernel for a 2b = n slot.
__host__ __device__ inline size_t eig_smem_bytes(int n) {
    return (size_t)n * n * 8            // G, FP64
           + (size_t)n * n * 4          // Q, FP32
           + (size_t)2 * n * 8          // c/s of two rounds
           + (size_t)n * 4              // permutation
           + (size_t)(n - 1) * n        // round-robin table
           + (size_t)2 * n              // pairs of two rounds
           + 16;
}

// Q columns u, v <- [u, v] J for the column pairs b = b0, b0 + bstep, ...
__device__ __forceinline__ void rotate_q(float *Q, const unsigned char *pq, const double *cs, int n, int half, int b0,
                                         int bstep, int lane) {
    for (int b = b0; b < half; b += bstep) {
        const int u = pq[b], v = pq[half + b];
        const float fc = (float)cs[b], fs = (float)cs[half + b];
        float *qu = Q + u * n, *qv = Q + v * n;
        for (int i = lane; i < n; i += 32) {
            const float xu = qu[i], xv = qv[i];
            qu[i] = fc * xu - fs * xv;
            qv[i] = fs * xu + fc * xv;
        }
    }
}

// One CTA per slot.  G (n x n, FP64, symmetric, column-major) is rotated as
// G <- J^T G J with the one-sided Jacobi rotation of columns p, q of the slot
// (app = g_pp, aqq = g_qq, apq = g_pq; primitives.py:334-347), the pairs of a
// round in parallel (round-robin order, primitives.py:309-313), Q <- Q J
// accumulated (FP32), until no pair is active or `sweeps` sweeps.  The off
// value of the slot is the largest |g_pq| / sqrt(g_pp g_qq) over its active
// pairs of live columns (g_pp and g_qq above live_floor) in the first sweep;
// dmax is the slot's largest g_pp.
//
// Per round r: warp 0 computes the rotations of round r while the other
// warps apply round r - 1's rotations to Q (c/s and pairs double-buffered);
// one barrier; all warps rotate G with round r; one barrier.  The angle
// t = tan(theta) is formed in FP32 from exponent-scaled FP64 inputs (an
// angle error of ~1e-7 leaves |g_pq| 1e-7 of itself, which the next sweep
// removes); c = 1 / sqrt(1 + t^2) and s = t c are FP64, so every applied J
// is orthogonal to FP64 accuracy.
__global__ void __launch_bounds__(kEigThreads) eig_kernel(const float *Gin, __nv_bfloat16 *Qt_hi,
                                                          __nv_bfloat16 *Qt_lo, __nv_bfloat16 *Qt_lo2,
                                                          float *off_out, float *dmax_out, int *sweeps_out, int n,
                                                          int max_sweeps, double tol, const double *live_floor_ptr) {
    extern __shared__ __align__(16) unsigned char smem[];
    double *G = (double *)smem;                         // n x n, G[col * n + row]
    float *Q = (float *)(G + (size_t)n * n);             // n x n, Q[col * n + row]
    double *csb = (double *)(Q + (size_t)n * n);         // [2][c[half], s[half]] (n even: 8-byte aligned)
    int *perm = (int *)(csb + 2 * n);                    // n
    unsigned char *sched = (unsigned char *)(perm + n);  // (n - 1) x n players
    unsigned char *pqb = sched + (size_t)(n - 1) * n;    // [2][p[half], q[half]]
    __shared__ int s_any;
    __shared__ double s_red[32];
    __shared__ double s_first_off;
    const int k = blockIdx.x;
    const double live_floor = live_floor_ptr ? *live_floor_ptr : 0.0;
    const int half = n / 2;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nwarps = blockDim.x >> 5;
    const float *g_in = Gin + (size_t)k * n * n;
    for (int i = threadIdx.x; i < n * n; i += blockDim.x) {
        const int c = i / n, r = i - c * n;
        // symmetrise (the tensor-core Gram is symmetric up to rounding)
        G[i] = 0.5 * ((double)g_in[i] + (double)g_in[(size_t)r * n + c]);
        Q[i] = (r == c) ? 1.f : 0.f;
    }
    for (int i = threadIdx.x; i < (n - 1) * n; i += blockDim.x) {
        const int r = i / n, pos = i - r * n;
        sched[i] = (unsigned char)circ(pos, r, n);
    }
    if (threadIdx.x == 0) s_first_off = 0.0;
    __syncthreads();
    double dmax = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) dmax = fmax(dmax, G[(size_t)i * n + i]);
    for (int o = 16; o; o >>= 1) dmax = fmax(dmax, __shfl_xor_sync(0xffffffffu, dmax, o));
    if (lane == 0) s_red[warp] = dmax;
    __syncthreads();
    double gmax = 0.0;
    for (int w = 0; w < nwarps; ++w) gmax = fmax(gmax, s_red[w]);
    const double floor_ = 2.220446049250313e-16 * 2.220446049250313e-16 * gmax;
    const double tol2 = tol * tol;
    int sweep = 0;
    for (sweep = 1; sweep <= max_sweeps; ++sweep) {
        __syncthreads();                                 // s_any readers of the last sweep are done
        if (threadIdx.x == 0) s_any = 0;
        // largest ratio^2 of the sweep as num / den (one division at the end)
        double offn = 0.0, offd = 1.0;
        for (int r = 0; r < n - 1; ++r) {
            const int buf = r & 1;
            double *cs = csb + buf * n;
            unsigned char *pq = pqb + buf * n;
            __syncthreads();                             // G of round r - 1 complete
            if (warp == 0) {
                for (int t = lane; t < half; t += 32) {
                    int p = sched[r * n + t], q = sched[r * n + n - 1 - t];
                    if (p > q) { const int x = p; p = q; q = x; }
                    const double app = G[p * n + p], aqq = G[q * n + q], apq = G[q * n + p];
                    double c = 1.0, sn = 0.0;
                    const double prod = app * aqq, apq2 = apq * apq;
                    if (apq2 > tol2 * prod && fmin(app, aqq) > floor_) {
                        // off over live columns only (norm^2 above live_floor),
                        // like the reference's convergence check (solvers.py:55-57)
                        if (fmin(app, aqq) > live_floor && apq2 * offd > offn * prod) { offn = apq2; offd = prod; }
                        const double d = aqq - app, a2 = 2.0 * fabs(apq);
                        // exact power-of-two scaling of (d, 2|apq|) into [1, 2) for the FP32 angle
                        const int ex = (__double2hiint(fmax(fabs(d), a2)) >> 20) & 0x7ff;
                        const double sc = __hiloint2double((2046 - ex) << 20, 0);
                        const float df = fabsf((float)(d * sc)), af = (float)(a2 * sc);
                        const float tf = __fdividef(af, df + sqrtf(df * df + af * af));
                        const double tt = d < 0.0 ? -(double)tf : (double)tf;
                        c = rsqrt(1.0 + tt * tt);
                        sn = tt * c;
                        if (apq < 0.0) sn = -sn;
                        s_any = 1;
                    }
                    cs[t] = c;
                    cs[half + t] = sn;
                    pq[t] = (unsigned char)p;
                    pq[half + t] = (unsigned char)q;
                }
            } else if (r > 0) {
                rotate_q(Q, pqb + (buf ^ 1) * n, csb + (buf ^ 1) * n, n, half, warp - 1, nwarps - 1, lane);
            }
            __syncthreads();
            // G <- J^T G J: warp w takes column pairs b = w, w + nwarps, ...,
            // its lanes the row pairs a (one 2 x 2 block per (a, b)).
            for (int b = warp; b < half; b += nwarps) {
                const int u = pq[b], v = pq[half + b];
                const double cb = cs[b], sb = cs[half + b];
                double *cu = G + u * n, *cv = G + v * n;
                for (int a = lane; a < half; a += 32) {
                    const int p = pq[a], q = pq[half + a];
                    const double ca = cs[a], sa = cs[half + a];
                    const double gpu = cu[p], gqu = cu[q], gpv = cv[p], gqv = cv[q];
                    // rows: [p; q] <- J_a^T [p; q] with J = [[c, s], [-s, c]] acting on columns (p, q)
                    const double rpu = ca * gpu - sa * gqu, rqu = sa * gpu + ca * gqu;
                    const double rpv = ca * gpv - sa * gqv, rqv = sa * gpv + ca * gqv;
                    // columns: [u, v] <- [u, v] J_b
                    cu[p] = cb * rpu - sb * rpv;
                    cv[p] = sb * rpu + cb * rpv;
                    cu[q] = cb * rqu - sb * rqv;
                    cv[q] = sb * rqu + cb * rqv;
                }
            }
        }
        // the last round's Q rotation, all warps
        rotate_q(Q, pqb + ((n - 2) & 1) * n, csb + ((n - 2) & 1) * n, n, half, warp, nwarps, lane);
        if (sweep == 1 && warp == 0) {
            for (int o = 16; o; o >>= 1) {
                const double on = __shfl_xor_sync(0xffffffffu, offn, o), od = __shfl_xor_sync(0xffffffffu, offd, o);
                if (on * offd > offn * od) { offn = on; offd = od; }
            }
            if (lane == 0) s_first_off = sqrt(offn / offd);
        }
        __syncthreads();
        if (!s_any) break;
    }
    __syncthreads();
    // Eigenvalues descending (stable), Q^T rows in that order.
    for (int j = threadIdx.x; j < n; j += blockDim.x) {
        const double dj = G[(size_t)j * n + j];
        int rk = 0;
        for (int i = 0; i < n; ++i) {
            const double di = G[(size_t)i * n + i];
            rk += (di > dj) || (di == dj && i < j);
        }
        perm[rk] = j;
    }
    __syncthreads();
    __nv_bfloat16 *qh = Qt_hi + (size_t)k * n * n, *ql = Qt_lo + (size_t)k * n * n;
    for (int t = threadIdx.x; t < n * n; t += blockDim.x) {
        const int rrow = t / n, i = t - rrow * n;       // Q^T row rrow = column perm[rrow] of Q
        const float x = Q[(size_t)perm[rrow] * n + i];
        const __nv_bfloat16 h = __float2bfloat16_rn(x);
        qh[t] = h;
        const float rem = x - __bfloat162float(h);
        const __nv_bfloat16 l = __float2bfloat16_rn(rem);
        ql[t] = l;
        if (Qt_lo2) Qt_lo2[(size_t)k * n * n + t] = __float2bfloat16_rn(rem - __bfloat162float(l));
    }
    if (threadIdx.x == 0) {
        if (off_out) off_out[k] = (float)s_first_off;
        if (dmax_out) dmax_out[k] = (float)gmax;
        if (sweeps_out) sweeps_out[k] = sweep > max_sweeps ? max_sweeps : sweep;
    }
}

// Register-resident variant of eig_kernel for n = 32 * RPT (64 or 128), the
// slot widths of b = 32 and b = 64.  Same rotations and outputs; the pairs of
// a sweep follow the odd-even ordering instead of the round robin: round r
// pairs adjacent positions (2t + r % 2, 2t + r % 2 + 1) and every rotation
// also swaps its two positions (J P), so after n rounds each pair of columns
// has met exactly once (the swaps reverse the order).  With positions fixed,
// G and Q stay in registers: lane l holds rows RPT l .. RPT l + RPT - 1 and
// warp w columns CB w .. CB w + CB - 1 (CB even: 4, 8 or 16 columns per warp,
// n / CB warps; the outputs do not depend on CB).  Row pairs that straddle two lanes use warp
// shuffles, column pairs that straddle two warps (odd rounds) one exchange
// through shared memory.  Per round: warp 0 forms the angles from the
// diagonal d and superdiagonal e (published in shared memory by their
// owners), one barrier, rotations, (odd rounds: boundary exchange, one
// barrier), new d / e, one barrier.
// DQ (deferred Q): Q is not accumulated here.  The angle threads record every
// applied (c, s) as FP32 pairs, cs_out[(k * max_sweeps + sweep) * n + r][p]
// by the pair's first position p, and the kernel writes the eigenvalues'
// sorted position of every column (pos_out[k * n + j]); q_apply_kernel then
// forms Q^T from them on other SMs, so this latency-bound kernel issues
// about a quarter fewer instructions per round.
template <int RPT, int CB, typename TG, bool DQ = false>
__global__ void __launch_bounds__(RPT * 1024 / CB) eig_reg_kernel(const float *Gin, __nv_bfloat16 *Qt_hi,
                                                            __nv_bfloat16 *Qt_lo, __nv_bfloat16 *Qt_lo2,
                                                            float *off_out, float *dmax_out, int *sweeps_out,
                                                            int max_sweeps, double tol, const double *live_floor_ptr,
                                                            float2 *cs_out, int *pos_out) {
    constexpr int n = 32 * RPT;
    constexpr int NW = n / CB;                 // warps
    static_assert(CB % 2 == 0 && NW >= RPT / 2, "columns per warp");
    extern __shared__ __align__(16) unsigned char smem[];
    TG *sd = (TG *)smem;               // d[x] = G[x][x]
    TG *se = sd + n;                       // e[x] = G[x][x + 1]
    TG *sc = se + n;                       // c of the pair starting at position p, at cs_at(p)
    TG *ss = sc + n;                       // s of the pair starting at position p, at cs_at(p)
    TG *bg = ss + n;                       // [NW][2][RPT][32] boundary columns of G (first, last), lane-major
    float *bq = (float *)(bg + (size_t)NW * 2 * n);  // [NW][2][RPT][32] boundary columns of Q, lane-major
    float *Qs = bq + (size_t)NW * 2 * n;       // n x n, Q[col * n + row] (write-out)
    int *perm = (int *)(Qs + (size_t)n * n);   // n
    __shared__ int s_any;
    __shared__ double s_first_off;
    __shared__ double s_red[NW];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int r0 = lane * RPT, c0 = warp * CB;
    // Shared-memory slots of per-row data, lane-major: row x = RPT l + i (lane l's i-th row) at
    // 32 i + l, so that the 32 lanes reading "their" i-th row hit 32 consecutive words instead of
    // one bank RPT-fold; a warp-uniform row is a broadcast either way.
    auto cs_at = [](int x) { return (x % RPT) * 32 + x / RPT; };
    auto bnd_at = [](int w, int side, int i, int l) { return ((w * 2 + side) * RPT + i) * 32 + l; };
    const int k = blockIdx.x;
    const double live_floor = live_floor_ptr ? *live_floor_ptr : 0.0;
    const float *g_in = Gin + (size_t)k * n * n;

    TG g[RPT][CB];
    float q[RPT][CB];
#pragma unroll
    for (int i = 0; i < RPT; ++i)
#pragma unroll
        for (int j = 0; j < CB; ++j) {
            const int r = r0 + i, c = c0 + j;
            // symmetrise (the tensor-core Gram is symmetric up to rounding)
            g[i][j] = (TG)(0.5 * ((double)g_in[(size_t)r * n + c] + (double)g_in[(size_t)c * n + r]));
            q[i][j] = (r == c) ? 1.f : 0.f;
        }
    auto publish_de = [&]() {
#pragma unroll
        for (int i = 0; i < RPT; ++i) {
            const int x = r0 + i;
#pragma unroll
            for (int j = 0; j < CB; ++j) {
                if (c0 + j == x) sd[x] = g[i][j];
                if (c0 + j == x + 1) se[x] = g[i][j];
            }
        }
    };
    publish_de();
    if (threadIdx.x == 0) s_first_off = 0.0;
    __syncthreads();
    double dm = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) dm = fmax(dm, (double)sd[i]);
    for (int o = 16; o; o >>= 1) dm = fmax(dm, __shfl_xor_sync(0xffffffffu, dm, o));
    if (lane == 0) s_red[warp] = dm;
    __syncthreads();
    double gmax = 0.0;
#pragma unroll
    for (int w = 0; w < NW; ++w) gmax = fmax(gmax, s_red[w]);
    // eps of the arithmetic squared times the largest diagonal: the active floor
    constexpr double eps_g = sizeof(TG) == 8 ? 2.220446049250313e-16 : 1.1920928955078125e-07;
    const double floor_ = eps_g * eps_g * gmax;
    const double tol2 = tol * tol;
    int sweep = 0;
    for (sweep = 1; sweep <= max_sweeps; ++sweep) {
        if (threadIdx.x == 0) s_any = 0;
        double offn = 0.0, offd = 1.0;
        for (int r = 0; r < n; ++r) {
            const int par = r & 1;
            __syncthreads();                   // d / e of the previous round published; s_any reset
            if (warp < RPT / 2) {                 // one pair per lane
                {
                    const int t = warp * 32 + lane;
                    if (t >= n / 2 - par) goto angles_done;
                    const int p = 2 * t + par;
                    const double app = sd[p], aqq = sd[p + 1], apq = se[p];
                    TG c = 1, sn = 0;
                    const double prod = app * aqq, apq2 = apq * apq;
                    if (apq2 > tol2 * prod && fmin(app, aqq) > floor_) {
                        // off over live columns only (solvers.py:55-57)
                        if (fmin(app, aqq) > live_floor && apq2 * offd > offn * prod) { offn = apq2; offd = prod; }
                        if constexpr (sizeof(TG) == 8) {
                            const double d = aqq - app, a2 = 2.0 * fabs(apq);
                            const int ex = (__double2hiint(fmax(fabs(d), a2)) >> 20) & 0x7ff;
                            const double scl = __hiloint2double((2046 - ex) << 20, 0);
                            const float df = fabsf((float)(d * scl)), af = (float)(a2 * scl);
                            const float tf = __fdividef(af, df + sqrtf(df * df + af * af));
                            const double tt = d < 0.0 ? -(double)tf : (double)tf;
                            // c = 1 / sqrt(1 + t^2): FP32 estimate and one Newton step in FP64
                            const double x = 1.0 + tt * tt;
                            const double c0 = (double)rsqrtf(1.f + tf * tf);
                            c = c0 * (1.5 - 0.5 * x * c0 * c0);
                            sn = tt * c;
                        } else {
                            // FP32 G (the two-part stage): the same angle, all in FP32
                            const float d = (float)(aqq - app), a2 = 2.f * fabsf((float)apq);
                            const float tf = __fdividef(a2, fabsf(d) + sqrtf(d * d + a2 * a2));
                            const float tt = d < 0.f ? -tf : tf;
                            c = rsqrtf(1.f + tt * tt);
                            sn = tt * c;
                        }
                        if (apq < 0.0) sn = -sn;
                        s_any = 1;
                    }
                    sc[cs_at(p)] = c;
                    ss[cs_at(p)] = sn;
                    if constexpr (DQ)
                        cs_out[(((size_t)k * max_sweeps + (sweep - 1)) * n + r) * n + p] = make_float2((float)c, (float)sn);
                }
            angles_done:;
            }
            __syncthreads();
            // Rows (J^T from the left, then the swap): (x_p, x_q) <- (s x_p + c x_q, c x_p - s x_q).
            if (par == 0) {
#pragma unroll
                for (int i = 0; i < RPT; i += 2) {
                    const TG c = sc[32 * i + lane], sn = ss[32 * i + lane];       // pair at row r0 + i
#pragma unroll
                    for (int j = 0; j < CB; ++j) {
                        const TG x = g[i][j], y = g[i + 1][j];
                        g[i][j] = sn * x + c * y;
                        g[i + 1][j] = c * x - sn * y;
                    }
                }
            } else {
                const bool has_up = lane > 0, has_down = lane < 31;
                // pairs at rows r0 - 1 (lane - 1's last row) and r0 + RPT - 1 (this lane's last row)
                const TG cu = has_up ? sc[32 * (RPT - 1) + lane - 1] : (TG)1,
                         su = has_up ? ss[32 * (RPT - 1) + lane - 1] : (TG)0;
                const TG cd = has_down ? sc[32 * (RPT - 1) + lane] : (TG)1,
                         sdn = has_down ? ss[32 * (RPT - 1) + lane] : (TG)0;
#pragma unroll
                for (int j = 0; j < CB; ++j) {
                    const TG up = __shfl_up_sync(0xffffffffu, g[RPT - 1][j], 1);   // row r0 - 1
                    const TG dn = __shfl_down_sync(0xffffffffu, g[0][j], 1);       // row r0 + RPT
                    const TG first = g[0][j], last = g[RPT - 1][j];
                    if (has_up) g[0][j] = cu * up - su * first;                         // second of pair (r0 - 1, r0)
                    if (has_down) g[RPT - 1][j] = sdn * last + cd * dn;                 // first of pair (r0 + RPT - 1, r0 + RPT)
                }
#pragma unroll
                for (int i = 1; i + 1 < RPT; i += 2) {
                    const TG c = sc[32 * i + lane], sn = ss[32 * i + lane];       // pair at row r0 + i
#pragma unroll
                    for (int j = 0; j < CB; ++j) {
                        const TG x = g[i][j], y = g[i + 1][j];
                        g[i][j] = sn * x + c * y;
                        g[i + 1][j] = c * x - sn * y;
                    }
                }
            }
            // Columns (J from the right, then the swap), G and Q alike.
            if (par == 0) {
#pragma unroll
                for (int j = 0; j < CB; j += 2) {
                    const TG c = sc[cs_at(c0 + j)], sn = ss[cs_at(c0 + j)];
                    const float fc = (float)c, fs = (float)sn;
#pragma unroll
                    for (int i = 0; i < RPT; ++i) {
                        const TG x = g[i][j], y = g[i][j + 1];
                        g[i][j] = sn * x + c * y;
                        g[i][j + 1] = c * x - sn * y;
                        if constexpr (!DQ) {
                            const float u = q[i][j], v = q[i][j + 1];
                            q[i][j] = fs * u + fc * v;
                            q[i][j + 1] = fc * u - fs * v;
                        }
                    }
                }
            } else {
                // publish this warp's first and last columns (after the row rotation)
#pragma unroll
                for (int i = 0; i < RPT; ++i) {
                    bg[bnd_at(warp, 0, i, lane)] = g[i][0];
                    bg[bnd_at(warp, 1, i, lane)] = g[i][CB - 1];
                    if constexpr (!DQ) {
                        bq[bnd_at(warp, 0, i, lane)] = q[i][0];
                        bq[bnd_at(warp, 1, i, lane)] = q[i][CB - 1];
                    }
                }
                __syncthreads();
                const bool has_left = warp > 0, has_right = warp < NW - 1;
                const TG cl = has_left ? sc[cs_at(c0 - 1)] : (TG)1, sl = has_left ? ss[cs_at(c0 - 1)] : (TG)0;
                const TG cr = has_right ? sc[cs_at(c0 + CB - 1)] : (TG)1,
                         sr = has_right ? ss[cs_at(c0 + CB - 1)] : (TG)0;
#pragma unroll
                for (int i = 0; i < RPT; ++i) {
                    if (has_left) {                // pair (c0 - 1, c0): this warp holds the second
                        const TG x = bg[bnd_at(warp - 1, 1, i, lane)];
                        g[i][0] = cl * x - sl * g[i][0];
                        if constexpr (!DQ) {
                            const float u = bq[bnd_at(warp - 1, 1, i, lane)];
                            q[i][0] = (float)cl * u - (float)sl * q[i][0];
                        }
                    }
                    if (has_right) {               // pair (c0 + CB - 1, c0 + CB): this warp holds the first
                        const TG y = bg[bnd_at(warp + 1, 0, i, lane)];
                        g[i][CB - 1] = sr * g[i][CB - 1] + cr * y;
                        if constexpr (!DQ) {
                            const float v = bq[bnd_at(warp + 1, 0, i, lane)];
                            q[i][CB - 1] = (float)sr * q[i][CB - 1] + (float)cr * v;
                        }
                    }
                }
#pragma unroll
                for (int j = 1; j + 1 < CB; j += 2) {
                    const TG c = sc[cs_at(c0 + j)], sn = ss[cs_at(c0 + j)];
                    const float fc = (float)c, fs = (float)sn;
#pragma unroll
                    for (int i = 0; i < RPT; ++i) {
                        const TG x = g[i][j], y = g[i][j + 1];
                        g[i][j] = sn * x + c * y;
                        g[i][j + 1] = c * x - sn * y;
                        if constexpr (!DQ) {
                            const float u = q[i][j], v = q[i][j + 1];
                            q[i][j] = fs * u + fc * v;
                            q[i][j + 1] = fc * u - fs * v;
                        }
                    }
                }
            }
            publish_de();
        }
        if (sweep == 1 && warp < RPT / 2) {
            for (int o = 16; o; o >>= 1) {
                const double on = __shfl_xor_sync(0xffffffffu, offn, o), od = __shfl_xor_sync(0xffffffffu, offd, o);
                if (on * offd > offn * od) { offn = on; offd = od; }
            }
            if (lane == 0) s_red[warp] = sqrt(offn / offd);
        }
        __syncthreads();
        if (sweep == 1 && threadIdx.x == 0) {
            double o = 0.0;
#pragma unroll
            for (int w = 0; w < RPT / 2; ++w) o = fmax(o, s_red[w]);
            s_first_off = o;
        }
        const int any = s_any;
        __syncthreads();                       // everyone has read s_any before it is reset
        if (!any) break;
    }
    // Q to shared memory (column-major) for the sorted write-out.
    if constexpr (!DQ) {
#pragma unroll
        for (int i = 0; i < RPT; ++i)
#pragma unroll
            for (int j = 0; j < CB; ++j) Qs[(size_t)(c0 + j) * n + r0 + i] = q[i][j];
    }
    __syncthreads();
    // Eigenvalues descending (stable), Q^T rows in that order.
    for (int j = threadIdx.x; j < n; j += blockDim.x) {
        const double dj = sd[j];
        int rk = 0;
        for (int i = 0; i < n; ++i) {
            const double di = sd[i];
            rk += (di > dj) || (di == dj && i < j);
        }
        perm[rk] = j;
        if constexpr (DQ) pos_out[(size_t)k * n + j] = rk;
    }
    __syncthreads();
    __nv_bfloat16 *qh = Qt_hi + (size_t)k * n * n, *ql = Qt_lo + (size_t)k * n * n;
    for (int t = threadIdx.x; t < (DQ ? 0 : n * n); t += blockDim.x) {
        const int rrow = t / n, i = t - rrow * n;       // Q^T row rrow = column perm[rrow] of Q
        const float x = Qs[(size_t)perm[rrow] * n + i];
        const __nv_bfloat16 h = __float2bfloat16_rn(x);
        qh[t] = h;
        const float rem = x - __bfloat162float(h);
        const __nv_bfloat16 l = __float2bfloat16_rn(rem);
        ql[t] = l;
        if (Qt_lo2) Qt_lo2[(size_t)k * n * n + t] = __float2bfloat16_rn(rem - __bfloat162float(l));
    }
    if (threadIdx.x == 0) {
        if (off_out) off_out[k] = (float)s_first_off;
        if (dmax_out) dmax_out[k] = (float)gmax;
        if (sweeps_out) sweeps_out[k] = sweep > max_sweeps ? max_sweeps : sweep;
    }
}

// Q^T of every slot from the rotations eig_reg_kernel<..., DQ = true>
// recorded.  Warp (k, i) forms row i of Q = prod_r J_r P_r with the same FP32
// column updates the register kernel applies to its Q tiles (lane l holds
// columns RPT l .. RPT l + RPT - 1; in odd rounds the pairs that straddle two
// lanes take the neighbour's value by a shuffle), then writes it as column i
// of Q^T in eigenvalue order (row pos[j] for column j), as hi / lo (/ lo2)
// BF16 parts.  Rows are independent, so the whole grid works at once.
template <int RPT>
__global__ void __launch_bounds__(256) q_apply_kernel(const float2 *cs, const int *sweeps, const int *pos,
                                                      __nv_bfloat16 *Qt_hi, __nv_bfloat16 *Qt_lo,
                                                      __nv_bfloat16 *Qt_lo2, int pairs, int max_sweeps) {
    constexpr int n = 32 * RPT;
    const int64_t gw = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (gw >= (int64_t)pairs * n) return;                  // whole warps
    const int k = (int)(gw / n), i = (int)(gw - (int64_t)k * n);
    const int c0 = lane * RPT;
    float q[RPT];
#pragma unroll
    for (int e = 0; e < RPT; ++e) q[e] = (c0 + e == i) ? 1.f : 0.f;
    int ns = sweeps[k];
    if (ns > max_sweeps) ns = max_sweeps;
    const float2 *ck = cs + (size_t)k * max_sweeps * n * n;
    for (int rr = 0; rr < ns * n; ++rr) {
        const float2 *c_r = ck + (size_t)rr * n;
        if ((rr & 1) == 0) {
#pragma unroll
            for (int e = 0; e < RPT; e += 2) {
                const float2 t = c_r[c0 + e];
                const float u = q[e], v = q[e + 1];
                q[e] = t.y * u + t.x * v;
                q[e + 1] = t.x * u - t.y * v;
            }
        } else {
            const bool has_up = lane > 0, has_down = lane < 31;
            const float2 tu = has_up ? c_r[c0 - 1] : make_float2(1.f, 0.f);
            const float2 td = has_down ? c_r[c0 + RPT - 1] : make_float2(1.f, 0.f);
            const float up = __shfl_up_sync(0xffffffffu, q[RPT - 1], 1);    // column c0 - 1
            const float dn = __shfl_down_sync(0xffffffffu, q[0], 1);        // column c0 + RPT
            const float first = q[0], last = q[RPT - 1];
            if (has_up) q[0] = tu.x * up - tu.y * first;                      // second of (c0 - 1, c0)
            if (has_down) q[RPT - 1] = td.y * last + td.x * dn;               // first of (c0 + RPT - 1, c0 + RPT)
#pragma unroll
            for (int e = 1; e + 1 < RPT; e += 2) {
                const float2 t = c_r[c0 + e];
                const float u = q[e], v = q[e + 1];
                q[e] = t.y * u + t.x * v;
                q[e + 1] = t.x * u - t.y * v;
            }
        }
    }
#pragma unroll
    for (int e = 0; e < RPT; ++e) {
        const size_t t = (size_t)k * n * n + (size_t)pos[(size_t)k * n + c0 + e] * n + i;
        const float x = q[e];
        const __nv_bfloat16 h = __float2bfloat16_rn(x);
        Qt_hi[t] = h;
        const float rem = x - __bfloat162float(h);
        const __nv_bfloat16 l = __float2bfloat16_rn(rem);
        Qt_lo[t] = l;
        if (Qt_lo2) Qt_lo2[t] = __float2bfloat16_rn(rem - __bfloat162float(l));
    }
}

__host__ inline size_t eig_reg_smem_bytes(int n, int cb) {   // sized for FP64 G (enough for FP32)
    const int nw = n / cb;
    return (size_t)4 * n * 8 + (size_t)nw * 2 * n * 8 + (size_t)nw * 2 * n * 4 + (size_t)n * n * 4 + (size_t)n * 4 +
           16;
}

// dst row map[r] <- src row r (length L), split into hi / lo BF16.
__global__ void scatter_kernel(const float *src, const int *map, __nv_bfloat16 *hi, __nv_bfloat16 *lo,
                               __nv_bfloat16 *lo2, float *f32, int64_t rows, int64_t L) {
    for (int64_t r = blockIdx.y; r < rows; r += gridDim.y) {
        const int64_t d = map ? map[r] : r;
        for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < L; i += (int64_t)gridDim.x * blockDim.x) {
            const float v = src[r * L + i];
            const __nv_bfloat16 h = __float2bfloat16_rn(v);
            if (hi) hi[d * L + i] = h;
            const float rem = v - __bfloat162float(h);
            const __nv_bfloat16 l = __float2bfloat16_rn(rem);
            if (lo) lo[d * L + i] = l;
            if (lo2) lo2[d * L + i] = __float2bfloat16_rn(rem - __bfloat162float(l));
            if (f32) f32[d * L + i] = v;
        }
    }
}

__global__ void combine_kernel(const __nv_bfloat16 *hi, const __nv_bfloat16 *lo, const __nv_bfloat16 *lo2,
                               const int *map, float *dst, int64_t rows, int64_t L) {
    for (int64_t r = blockIdx.y; r < rows; r += gridDim.y) {
        const int64_t d = map ? map[r] : r;
        for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < L; i += (int64_t)gridDim.x * blockDim.x)
            dst[d * L + i] = __bfloat162float(hi[r * L + i]) + (lo ? __bfloat162float(lo[r * L + i]) : 0.f) +
                             (lo2 ? __bfloat162float(lo2[r * L + i]) : 0.f);
    }
}

// sigma_j = ||Wt row j|| * 2^e (FP64 sums), one warp per row.
__global__ void norms_kernel(const float *Wt, double *sig, int64_t n, int64_t m) {
    const int64_t row = blockIdx.x * (int64_t)(blockDim.x >> 5) + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (row >= n) return;
    double acc = 0.0;
    for (int64_t i = lane; i < m; i += 32) {
        const double x = Wt[row * m + i];
        acc = fma(x, x, acc);
    }
    acc = warp_sum_d(acc);
    if (lane == 0) sig[row] = sqrt(acc);
}

// Stable descending rank of every sigma (n^2 comparisons, n <= a few 1000).
__global__ void rank_kernel(const double *sig, int *perm, int n) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    const double sj = sig[j];
    int rk = 0;
    for (int i = 0; i < n; ++i) {
        const double si = sig[i];
        rk += (si > sj) || (si == sj && i < j);
    }
    perm[rk] = j;
}

// Outputs: S[r] (cut below eps32 max(m, n_even) sigma_1), U[:, r] = W_perm[r] /
// sigma (kept columns; cut columns of nonzero norm are normalised the same
// way), Vh[r, :] = Vt[perm[r], :].
__global__ void finish_kernel(const float *Wt, const float *Vt, const double *sig, const int *perm, float *U,
                              float *S, float *Vh, int64_t m, int64_t n, int rank, int e, int cutw) {
    const double smax = sig[perm[0]];
    const double cut = 1.1920928955078125e-07 * (double)cutw * smax;
    const int64_t total_u = m * rank, total_v = (int64_t)rank * n;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total_u + total_v + rank;
         t += (int64_t)gridDim.x * blockDim.x) {
        if (t < total_u) {
            const int64_t i = t / rank, r = t - i * rank;
            const int j = perm[r];
            const double sj = sig[j];
            U[t] = U ? (float)(sj > 0.0 ? Wt[(int64_t)j * m + i] / sj : 0.0) : 0.f;
        } else if (t < total_u + total_v) {
            const int64_t q = t - total_u, r = q / n, c = q - r * n;
            Vh[q] = Vt[(int64_t)perm[r] * n + c];
        } else {
            const int r = (int)(t - total_u - total_v);
            const double sj = sig[perm[r]];
            S[r] = (float)(sj > cut ? ldexp(sj, e) : 0.0);
        }
    }
}


// C (M x N, f32) = A (M x K) * B (N x K)^T with FP32 inputs (row-major, K
// contiguous) and FP64 accumulation: every product of two floats is exact in
// FP64, so C carries FP64 accuracy until its final rounding.  128 x 128
// tiles, K steps of 8, 256 threads with 8 x 8 outputs each.
__global__ void __launch_bounds__(256) gemm_f64acc_kernel(const float *A, const float *B, float *C, int64_t M,
                                                          int64_t N, int64_t K, int64_t lda, int64_t ldb,
                                                          int64_t ldc) {
    __shared__ double As[8][128];
    __shared__ double Bs[8][128];
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
    const int64_t m0 = (int64_t)blockIdx.y * 128, n0 = (int64_t)blockIdx.x * 128;
    double acc[8][8];
#pragma unroll
    for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int j = 0; j < 8; ++j) acc[i][j] = 0.0;
    const int lr = threadIdx.x >> 1, lk = (threadIdx.x & 1) * 4;
    for (int64_t k0 = 0; k0 < K; k0 += 8) {
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int64_t ka = k0 + lk + q;
            const int64_t ra = m0 + lr, rb = n0 + lr;
            As[lk + q][lr] = (ra < M && ka < K) ? (double)A[ra * lda + ka] : 0.0;
            Bs[lk + q][lr] = (rb < N && ka < K) ? (double)B[rb * ldb + ka] : 0.0;
        }
        __syncthreads();
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            double a[8], b[8];
#pragma unroll
            for (int i = 0; i < 8; ++i) a[i] = As[k][ty + 16 * i];
#pragma unroll
            for (int j = 0; j < 8; ++j) b[j] = Bs[k][tx + 16 * j];
#pragma unroll
            for (int i = 0; i < 8; ++i)
#pragma unroll
                for (int j = 0; j < 8; ++j) acc[i][j] = fma(a[i], b[j], acc[i][j]);
        }
        __syncthreads();
    }
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        const int64_t r = m0 + ty + 16 * i;
        if (r >= M) continue;
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            const int64_t c = n0 + tx + 16 * j;
            if (c < N) C[r * ldc + c] = (float)acc[i][j];
        }
    }
}

// The same product for 16-byte aligned rows (A, B 16-byte aligned; lda, ldb
// and K multiples of 4): the next 16-deep K slice is fetched with float4
// loads into registers while the current slice's FMAs run, then stored as
// FP64 into the other half of a double-buffered shared tile, so each slice
// costs one barrier and no exposed global latency.  Thread (ty, tx) owns rows
// 2 ty + 32 i + {0, 1} and columns 2 tx + 32 j + {0, 1} (i, j < 4): its
// operands are double2 loads from shared memory.
constexpr int kF64KC = 16;
constexpr size_t kF64AccSmem = 2 * 2 * kF64KC * 128 * sizeof(double);   // [A, B][2][16][128]

__global__ void __launch_bounds__(256) gemm_f64acc_vec_kernel(const float *A, const float *B, float *C, int64_t M,
                                                              int64_t N, int64_t K, int64_t lda, int64_t ldb,
                                                              int64_t ldc, int m_fast) {
    extern __shared__ __align__(16) double f64acc_smem[];
    double *As = f64acc_smem;                      // As[buf][k][row] at (buf * kF64KC + k) * 128 + row
    double *Bs = f64acc_smem + 2 * kF64KC * 128;
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
    // m_fast: consecutive CTAs take consecutive row tiles of C, so the tile of
    // B (the larger operand) they share is read from DRAM once
    const int64_t m0 = (int64_t)(m_fast ? blockIdx.x : blockIdx.y) * 128,
                  n0 = (int64_t)(m_fast ? blockIdx.y : blockIdx.x) * 128;
    // loader: row lrow of the tile, K offsets lk and lk + 8 of the slice
    const int lrow = threadIdx.x & 127, lk = (threadIdx.x >> 7) * 4;
    const bool arow = m0 + lrow < M, brow = n0 + lrow < N;
    const float *ap = A + (arow ? (m0 + lrow) * lda : 0), *bp = B + (brow ? (n0 + lrow) * ldb : 0);
    float4 pa[2], pb[2];
    auto fetch = [&](int64_t k0) {
#pragma unroll
        for (int l = 0; l < 2; ++l) {
            const int64_t ka = k0 + lk + 8 * l;
            const bool kin = ka < K;               // K % 4 == 0: a float4 is wholly in or out
            pa[l] = (arow && kin) ? *(const float4 *)(ap + ka) : make_float4(0.f, 0.f, 0.f, 0.f);
            pb[l] = (brow && kin) ? *(const float4 *)(bp + ka) : make_float4(0.f, 0.f, 0.f, 0.f);
        }
    };
    auto stash = [&](int buf) {
#pragma unroll
        for (int l = 0; l < 2; ++l) {
            double *a = As + ((size_t)buf * kF64KC + lk + 8 * l) * 128 + lrow;
            double *b = Bs + ((size_t)buf * kF64KC + lk + 8 * l) * 128 + lrow;
            a[0] = pa[l].x; a[128] = pa[l].y; a[256] = pa[l].z; a[384] = pa[l].w;
            b[0] = pb[l].x; b[128] = pb[l].y; b[256] = pb[l].z; b[384] = pb[l].w;
        }
    };
    double acc[8][8];
#pragma unroll
    for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int j = 0; j < 8; ++j) acc[i][j] = 0.0;
    const int64_t nk = (K + kF64KC - 1) / kF64KC;
    fetch(0);
    stash(0);
    __syncthreads();
    for (int64_t kb = 0; kb < nk; ++kb) {
        const int buf = (int)(kb & 1);
        if (kb + 1 < nk) fetch((kb + 1) * kF64KC);
        const double *a_s = As + (size_t)buf * kF64KC * 128, *b_s = Bs + (size_t)buf * kF64KC * 128;
#pragma unroll
        for (int k = 0; k < kF64KC; ++k) {
            double a[8], b[8];
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                const double2 x = *(const double2 *)(a_s + k * 128 + 2 * ty + 32 * i);
                const double2 y = *(const double2 *)(b_s + k * 128 + 2 * tx + 32 * i);
                a[2 * i] = x.x; a[2 * i + 1] = x.y;
                b[2 * i] = y.x; b[2 * i + 1] = y.y;
            }
#pragma unroll
            for (int i = 0; i < 8; ++i)
#pragma unroll
                for (int j = 0; j < 8; ++j) acc[i][j] = fma(a[i], b[j], acc[i][j]);
        }
        // The other half was last read in the previous slice, before its barrier.
        if (kb + 1 < nk) stash(buf ^ 1);
        __syncthreads();
    }
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        const int64_t r = m0 + 2 * ty + 32 * (i >> 1) + (i & 1);
        if (r >= M) continue;
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            const int64_t c = n0 + 2 * tx + 32 * (j >> 1) + (j & 1);
            if (c < N) C[r * ldc + c] = (float)acc[i][j];
        }
    }
}

// Workspace of the deferred-Q form: the recorded (c, s) of every round and
// the sorted positions, per slot.
__host__ inline size_t eig_dq_cs_bytes(int64_t pairs, int n, int max_sweeps) {
    return ((size_t)pairs * max_sweeps * n * n * sizeof(float2) + 255) & ~(size_t)255;
}
__host__ inline size_t eig_dq_bytes(int64_t pairs, int n, int max_sweeps) {
    return eig_dq_cs_bytes(pairs, n, max_sweeps) + (((size_t)pairs * n * 4 + 255) & ~(size_t)255);
}

template <int RPT, int CB, typename TG>
static int launch_eig_reg(const float *G, void *Qt_hi, void *Qt_lo, void *Qt_lo2, float *off, float *dmax,
                          int32_t *sweeps, int64_t pairs, int32_t max_sweeps, double tol, const double *live_floor,
                          unsigned char *dq_ws, cudaStream_t st) {
    constexpr int n = 32 * RPT;
    const size_t smem = eig_reg_smem_bytes(n, CB);
    if (!dq_ws) {
        auto kern = eig_reg_kernel<RPT, CB, TG>;
        if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
            return JB_ECUDA;
        kern<<<(unsigned)pairs, 32 * (n / CB), smem, st>>>(G, (__nv_bfloat16 *)Qt_hi, (__nv_bfloat16 *)Qt_lo,
                                                          (__nv_bfloat16 *)Qt_lo2, off, dmax, sweeps, max_sweeps, tol,
                                                          live_floor, nullptr, nullptr);
        return cudaGetLastError() == cudaSuccess ? JB_OK : JB_ECUDA;
    }
    float2 *cs = (float2 *)dq_ws;
    int *pos = (int *)(dq_ws + eig_dq_cs_bytes(pairs, n, max_sweeps));
    auto kern = eig_reg_kernel<RPT, CB, TG, true>;
    if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
        return JB_ECUDA;
    kern<<<(unsigned)pairs, 32 * (n / CB), smem, st>>>(G, (__nv_bfloat16 *)Qt_hi, (__nv_bfloat16 *)Qt_lo,
                                                      (__nv_bfloat16 *)Qt_lo2, off, dmax, sweeps, max_sweeps, tol,
                                                      live_floor, cs, pos);
    if (cudaGetLastError() != cudaSuccess) return JB_ECUDA;
    const int64_t warps = pairs * n;
    q_apply_kernel<RPT><<<(unsigned)((warps + 7) / 8), 256, 0, st>>>(cs, sweeps, pos, (__nv_bfloat16 *)Qt_hi,
                                                                     (__nv_bfloat16 *)Qt_lo, (__nv_bfloat16 *)Qt_lo2,
                                                                     (int)pairs, max_sweeps);
    return cudaGetLastError() == cudaSuccess ? JB_OK : JB_ECUDA;
}

template <typename TG>
static int dispatch_eig_reg(int n, int cb, const float *G, void *Qt_hi, void *Qt_lo, void *Qt_lo2, float *off,
                            float *dmax, int32_t *sweeps, int64_t pairs, int32_t max_sweeps, double tol,
                            const double *live_floor, unsigned char *dq_ws, cudaStream_t st) {
#define JB_EIG_CASE(NN, RPT, CBV)                                                                               \
    if (n == NN && cb == CBV)                                                                                   \
        return launch_eig_reg<RPT, CBV, TG>(G, Qt_hi, Qt_lo, Qt_lo2, off, dmax, sweeps, pairs, max_sweeps, tol, \
                                            live_floor, dq_ws, st);
    JB_EIG_CASE(64, 2, 4)
    JB_EIG_CASE(64, 2, 8)
    JB_EIG_CASE(64, 2, 16)
    JB_EIG_CASE(128, 4, 4)
    JB_EIG_CASE(128, 4, 8)
    JB_EIG_CASE(128, 4, 16)
#undef JB_EIG_CASE
    return JB_EINVAL;
}

}  // namespace blk
}  // namespace jb

using namespace jb::blk;

extern "C" {

size_t jb_block_eig_workspace_bytes(int64_t pairs, int32_t n, int32_t max_sweeps) {
    if (pairs < 1 || n < 2 || max_sweeps < 1) return 0;
    return eig_dq_bytes(pairs, n, max_sweeps);
}

int jb_block_eig_ws(const float *G, void *Qt_hi, void *Qt_lo, void *Qt_lo2, float *off, float *dmax,
                    int32_t *sweeps, int64_t pairs, int32_t n, int32_t max_sweeps, double tol,
                    const double *live_floor, int32_t variant, void *workspace, size_t workspace_bytes,
                    void *stream) {
    const bool dq = (variant & JB_EIG_DEFER_Q) != 0;
    variant &= ~JB_EIG_DEFER_Q;
    const int lay = variant & ~JB_EIG_FP32;
    if (!G || !Qt_hi || !Qt_lo || pairs < 1 || n < 2 || (n & 1) || max_sweeps < 1 ||
        !(lay == 0 || lay == 1 || lay == 4 || lay == 8 || lay == 16) || (variant & ~(JB_EIG_FP32 | 31)) ||
        ((variant & JB_EIG_FP32) && !((n == 64 || n == 128) && lay != 1)) ||
        (dq && !((n == 64 || n == 128) && lay != 1)))
        return JB_EINVAL;
    if (dq && (!workspace || workspace_bytes < eig_dq_bytes(pairs, n, max_sweeps))) return JB_EWORKSPACE;
    cudaStream_t st = (cudaStream_t)stream;
    const bool g32 = (variant & JB_EIG_FP32) != 0;
    const int layout = variant & ~JB_EIG_FP32;
    unsigned char *dq_ws = dq ? (unsigned char *)workspace : nullptr;
    if ((n == 64 || n == 128) && layout != 1) {
        const int cb = layout == 0 ? 8 : layout;
        return g32 ? dispatch_eig_reg<float>(n, cb, G, Qt_hi, Qt_lo, Qt_lo2, off, dmax, sweeps, pairs, max_sweeps,
                                             tol, live_floor, dq_ws, st)
                   : dispatch_eig_reg<double>(n, cb, G, Qt_hi, Qt_lo, Qt_lo2, off, dmax, sweeps, pairs, max_sweeps,
                                              tol, live_floor, dq_ws, st);
    }
    if (n > 256) return JB_ETOOBIG;                  // players are stored as bytes
    const size_t smem = eig_smem_bytes(n);
    if (smem > 227 * 1024) return JB_ETOOBIG;
    if (cudaFuncSetAttribute(eig_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
        return JB_ECUDA;
    eig_kernel<<<(unsigned)pairs, kEigThreads, smem, st>>>(G, (__nv_bfloat16 *)Qt_hi, (__nv_bfloat16 *)Qt_lo,
                                                           (__nv_bfloat16 *)Qt_lo2, off, dmax, sweeps, n, max_sweeps,
                                                           tol, live_floor);
    return cudaGetLastError() == cudaSuccess ? JB_OK : JB_ECUDA;
}

int jb_block_eig_f64_ex(const float *G, void *Qt_hi, void *Qt_lo, void *Qt_lo2, float *off, float *dmax,
                        int32_t *sweeps, int64_t pairs, int32_t n, int32_t max_sweeps, double tol,
                        const double *live_floor, int32_t variant, void *stream) {
    if (variant & JB_EIG_DEFER_Q) return JB_EWORKSPACE;  // the deferred-Q form needs jb_block_eig_ws
    return jb_block_eig_ws(G, Qt_hi, Qt_lo, Qt_lo2, off, dmax, sweeps, pairs, n, max_sweeps, tol, live_floor, variant,
                           nullptr, 0, stream);
}

int jb_block_eig_f64(const float *G, void *Qt_hi, void *Qt_lo, void *Qt_lo2, float *off, float *dmax,
                     int32_t *sweeps, int64_t pairs, int32_t n, int32_t max_sweeps, double tol, const double *live_floor,
                     void *stream) {
    return jb_block_eig_f64_ex(G, Qt_hi, Qt_lo, Qt_lo2, off, dmax, sweeps, pairs, n, max_sweeps, tol, live_floor, 0,
                               stream);
}

int jb_rows_scatter(const float *src, const int32_t *map, void *hi, void *lo, void *lo2, float *f32, int64_t rows,
                    int64_t L, void *stream) {
    if (!src || rows < 1 || L < 1 || (!hi && !f32)) return JB_EINVAL;
    dim3 grid((unsigned)((L + 255) / 256 > 64 ? 64 : (L + 255) / 256), (unsigned)(rows > 65535 ? 65535 : rows));
    scatter_kernel<<<grid, 256, 0, (cudaStream_t)stream>>>(src, map, (__nv_bfloat16 *)hi, (__nv_bfloat16 *)lo,
                                                           (__nv_bfloat16 *)lo2, f32, rows, L);
    return cudaGetLastError() == cudaSuccess ? JB_OK : JB_ECUDA;
}

int jb_rows_combine(const void *hi, const void *lo, const void *lo2, const int32_t *map, float *dst, int64_t rows,
                    int64_t L, void *stream) {
    if (!hi || !dst || rows < 1 || L < 1) return JB_EINVAL;
    dim3 grid((unsigned)((L + 255) / 256 > 64 ? 64 : (L + 255) / 256), (unsigned)(rows > 65535 ? 65535 : rows));
    combine_kernel<<<grid, 256, 0, (cudaStream_t)stream>>>((const __nv_bfloat16 *)hi, (const __nv_bfloat16 *)lo,
                                                           (const __nv_bfloat16 *)lo2, map, dst, rows, L);
    return cudaGetLastError() == cudaSuccess ? JB_OK : JB_ECUDA;
}

int jb_block_finish(const float *Wt, const float *Vt, float *U, float *S, float *Vh, double *sig, int32_t *perm,
                    int64_t m, int64_t n, int32_t rank, int32_t e, int32_t cut_width, void *stream) {
    if (!Wt || !Vt || !S || !Vh || !U || !sig || !perm || m < 1 || n < 1 || rank < 1 || rank > n) return JB_EINVAL;
    cudaStream_t st = (cudaStream_t)stream;
    norms_kernel<<<(unsigned)((n + 7) / 8), 256, 0, st>>>(Wt, sig, n, m);
    rank_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(sig, perm, (int)n);
    const int64_t total = m * rank + (int64_t)rank * n + rank;
    int64_t blocks = (total + 255) / 256;
    if (blocks > 148 * 32) blocks = 148 * 32;
    finish_kernel<<<(unsigned)blocks, 256, 0, st>>>(Wt, Vt, sig, perm, U, S, Vh, m, n, rank, e, cut_width);
    return cudaGetLastError() == cudaSuccess ? JB_OK : JB_ECUDA;
}

int jb_gemm_f64acc(const float *A, const float *B, float *C, int64_t M, int64_t N, int64_t K, int64_t lda,
                   int64_t ldb, int64_t ldc, void *stream) {
    if (!A || !B || !C || M < 1 || N < 1 || K < 1 || lda < K || ldb < K || ldc < N) return JB_EINVAL;
    if ((M + 127) / 128 > 65535) return JB_ETOOBIG;
    dim3 grid((unsigned)((N + 127) / 128), (unsigned)((M + 127) / 128));
    const bool vec = ((uintptr_t)A & 15) == 0 && ((uintptr_t)B & 15) == 0 && lda % 4 == 0 && ldb % 4 == 0 &&
                     K % 4 == 0;
    if (vec) {
        const int m_fast = N > M && (N + 127) / 128 <= 65535;
        if (m_fast) grid = dim3((unsigned)((M + 127) / 128), (unsigned)((N + 127) / 128));
        if (cudaFuncSetAttribute(gemm_f64acc_vec_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)kF64AccSmem) != cudaSuccess)
            return JB_ECUDA;
        gemm_f64acc_vec_kernel<<<grid, 256, kF64AccSmem, (cudaStream_t)stream>>>(A, B, C, M, N, K, lda, ldb, ldc,
                                                                                   m_fast);
    } else {
        gemm_f64acc_kernel<<<grid, 256, 0, (cudaStream_t)stream>>>(A, B, C, M, N, K, lda, ldb, ldc);
    }
    return cudaGetLastError() == cudaSuccess ? JB_OK : JB_ECUDA;
}

}  // extern "C"
