// jb_regblock.cuh - register-resident block-cyclic one-sided Jacobi sweeps.
//
// The tall work matrix W (mt x npb, column-major in shared memory, 32*R rows
// per column, rows >= mt zero) and V (npb x npb, 32*RV rows per column) are
// split into nb = npb / B blocks of B columns.  Warp w of the CTA holds the two
// blocks at positions (w, nb-1-w) of a circle-method tournament over blocks
// in registers: lane l owns rows l, l+32, ... of all 2B columns.  A sweep is
//   * an intra step: the B-1 circle rounds inside each held block, and
//   * nb-1 block rounds: each warp meets its block pair with B "shift"
//     rounds (x_i, y_(i+j) mod B), i.e. all B^2 cross pairs,
// so every column pair is rotated exactly once per sweep, as in the
// reference's round-robin sweep (primitives.py:328-351) but with a block
// ordering: B disjoint pairs per warp step, their 3B dot products reduced
// together across the warp, and one CTA barrier per block round instead of
// two per pair round.  Blocks move between warps through shared memory.
//
// The rotation, the active test and the convergence test (no active pair in
// a sweep <=> off <= tol) are the reference's (primitives.py:334-355); the
// rotation is evaluated in an algebraically equal form (rot_params).  The null-column floor
// eps^2 * max ||w_j||^2 uses the column norms at the start of each sweep
// (the reference takes the maximum inside each round: they differ only for
// columns whose squared norm is within a factor n of eps^2 max).
#pragma once
#include "jb_device.cuh"

namespace jb {

template <int N> struct Log2 { static constexpr int value = 1 + Log2<N / 2>::value; };
template <> struct Log2<1> { static constexpr int value = 0; };

__device__ __forceinline__ int circ(int pos, int r, int n) {
    if (pos == 0) return 0;
    int x = (pos - 1 - r) % (n - 1);
    if (x < 0) x += n - 1;
    return 1 + x;
}

template <typename T, int B, int R, int RV>
struct Tile {
    T w[2 * B][R];
    T v[2 * B][RV];
    T nrm[2 * B];   // column norms squared (norm-update sweeps, intra steps), same on every lane
    T nx, ny;       // norm-update cross steps: the squared norms of the lane group's pair (x_i, y_i)
};

// Warp reduce-scatter of NV (power of two <= 32) values: afterwards x[0] on
// lane l holds the full warp sum of value index l >> (5 - log2 NV).
template <typename T, int NV>
__device__ __forceinline__ void reduce_scatter(T (&x)[NV], int lane) {
    constexpr int L = Log2<NV>::value;
#pragma unroll
    for (int s = 0; s < L; ++s) {
        const int h = NV >> (s + 1);
        const int o = 16 >> s;
        const bool up = (lane & o) != 0;
#pragma unroll
        for (int k = 0; k < h; ++k) {
            const T send = up ? x[k] : x[k + h];
            const T keep = up ? x[k + h] : x[k];
            x[k] = keep + __shfl_xor_sync(FULL, send, o);
        }
    }
#pragma unroll
    for (int o = 16 >> L; o >= 1; o >>= 1) x[0] += __shfl_xor_sync(FULL, x[0], o);
}

// Rotation of one pair from its Gram entries: the reference's rotation
// (primitives.py:334-347) in an algebraically equal form with one square
// root and one division.  With d = aqq - app, tau = d / (2|apq|) and
//   t = sign(tau) / (|tau| + hypot(tau, 1)) = sign(d) 2|apq| / (|d| + sqrt(d^2 + 4 apq^2)),
// c = 1/sqrt(1 + t^2), s = t c sign(apq); t = 1 when d = 0, as in the
// reference.  The active test ratio = |apq| / sqrt(app aqq) > tol is taken
// on squares.  Inputs are scaled (max |a| < 1), so d^2 + 4 apq^2 cannot
// overflow, and active pairs keep apq^2 far above the underflow range.
// Returns bit 0: active; bit 1: ratio > sqrt(tol) / 2 (the confirmation
// heuristic of rb_sweeps); bit 2: ratio > the phase exit ratio (ex2 its
// square).  Inactive pairs get c = 1, s = 0.
template <typename T>
__device__ __forceinline__ int rot_params(T app, T aqq, T apq, T tol2, T big2, T ex2, T floor_, T &c, T &s,
                                          T *shift = nullptr);

// FP32: t from approximate reciprocal / reciprocal square root (an error of
// a few ulp in t only leaves |apq| a few ulp of itself), c = 1/sqrt(1+t^2)
// refined by one Newton step so that c^2 + s^2 = 1 to ~1 ulp: every applied
// rotation stays orthogonal at FP32 precision.
// shift (optional): t |apq|, the change of the two squared column norms
// (app' = app - shift, aqq' = aqq + shift); 0 for an inactive pair.
template <>
__device__ __forceinline__ int rot_params<float>(float app, float aqq, float apq, float tol2, float big2, float ex2,
                                                 float floor_, float &c, float &s, float *shift) {
    c = 1.f;
    s = 0.f;
    if (shift) *shift = 0.f;
    const float apq2 = apq * apq;
    const float prod = app * aqq;
    const bool active = apq2 > tol2 * prod && fminf(app, aqq) > floor_;
    if (!active) return 0;
    const float d = aqq - app;
    const float h = fmaf(d, d, 4.f * apq2);
    const float sq = h * rsqrtf(h);                       // sqrt(h), h > 0 for an active pair
    const float t = copysignf(__fdividef(2.f * fabsf(apq), fabsf(d) + sq), d);
    const float x = fmaf(t, t, 1.f);
    const float c0 = rsqrtf(x);
    c = c0 * fmaf(-0.5f * x, c0 * c0, 1.5f);
    s = t * c;
    if (apq < 0.f) s = -s;
    if (shift) *shift = t * fabsf(apq);
    return 1 | (apq2 > big2 * prod ? 2 : 0) | (apq2 > ex2 * prod ? 4 : 0);
}

// FP64: the angle in FP32 from exponent-scaled (d, 2|apq|) -- exact power of
// two scaling into [1, 2), so no FP32 overflow or underflow -- and
// c = 1/sqrt(1+t^2), s = t c in FP64 (FP32 estimate + one Newton step), so
// every applied rotation is orthogonal to FP64 precision.
template <>
__device__ __forceinline__ int rot_params<double>(double app, double aqq, double apq, double tol2, double big2,
                                                  double ex2, double floor_, double &c, double &s, double *) {
    c = 1.0;
    s = 0.0;
    const double apq2 = apq * apq;
    const double prod = app * aqq;
    const bool active = apq2 > tol2 * prod && fmin(app, aqq) > floor_;
    if (!active) return 0;
    const double d = aqq - app, a2 = 2.0 * fabs(apq);
    const int ex = (__double2hiint(fmax(fabs(d), a2)) >> 20) & 0x7ff;
    const double scl = __hiloint2double((2046 - ex) << 20, 0);
    const float df = fabsf((float)(d * scl)), af = (float)(a2 * scl);
    const float hf = fmaf(df, df, af * af);
    const float tf = __fdividef(af, df + hf * rsqrtf(hf));
    const double t = d < 0.0 ? -(double)tf : (double)tf;
    const double x = fma(t, t, 1.0);
    const double c0 = (double)rsqrtf((float)x);
    c = c0 * fma(-0.5 * x, c0 * c0, 1.5);
    s = t * c;
    if (apq < 0.0) s = -s;
    return 1 | (apq2 > big2 * prod ? 2 : 0) | (apq2 > ex2 * prod ? 4 : 0);
}

// FP64 at the reference's precision (the float64 solve, tol 10 eps): the same
// rotation with t and c accurate to FP64 rounding, so that one rotation
// leaves the pair orthogonal to rounding level as the reference's FP64
// arithmetic does (an FP32 angle leaves a ratio ~1e-7 of the one it removed,
// near 10 eps in the last rotating sweep, and costs a sweep).  With the
// exponent-scaled dd = |d| scl, aa = 2|apq| scl (max of the two in [1, 2)),
// t is the positive root of g(t) = aa t^2 + 2 dd t - aa: the FP32 estimate,
// then two Newton steps t -= g(t) / g'(t) with g'/2 = aa t + dd >= 1/2
// inverted once in FP32 (each step multiplies the error by ~1e-7; g(t) is
// evaluated to rounding of its largest term, ~aa, so small angles keep
// their relative accuracy); c = 1/sqrt(1 + t^2) from the FP32 estimate and
// two Newton steps.
__device__ __forceinline__ int rot_params_exact(double app, double aqq, double apq, double tol2, double big2,
                                                double ex2, double floor_, double &c, double &s) {
    c = 1.0;
    s = 0.0;
    const double apq2 = apq * apq;
    const double prod = app * aqq;
    const bool active = apq2 > tol2 * prod && fmin(app, aqq) > floor_;
    if (!active) return 0;
    const double d = aqq - app, a2 = 2.0 * fabs(apq);
    const int ex = (__double2hiint(fmax(fabs(d), a2)) >> 20) & 0x7ff;
    const double scl = __hiloint2double((2046 - ex) << 20, 0);
    const double dd = fabs(d) * scl, aa = a2 * scl;
    const float df = (float)dd, af = (float)aa;
    const float hf = fmaf(df, df, af * af);
    double t = (double)__fdividef(af, df + hf * rsqrtf(hf));
    const double r = 0.5 * (double)__frcp_rn((float)fma(aa, t, dd));
#pragma unroll
    for (int k = 0; k < 2; ++k) t -= fma(aa * t, t, fma(2.0 * dd, t, -aa)) * r;
    if (d < 0.0) t = -t;
    const double x = fma(t, t, 1.0), hx = -0.5 * x;
    double c0 = (double)rsqrtf((float)x);
#pragma unroll
    for (int k = 0; k < 2; ++k) c0 *= fma(hx, c0 * c0, 1.5);
    c = c0;
    s = t * c;
    if (apq < 0.0) s = -s;
    return 1 | (apq2 > big2 * prod ? 2 : 0) | (apq2 > ex2 * prod ? 4 : 0);
}

// Packed FP32 (two rows per instruction, the sm_100 float2 intrinsics, so
// that the compiler sees the operations and keeps operand pairs in register
// pairs): a += x * y for (a0, a1), and the rotation pair
// (x, y) <- (c x - s y, s x + c y) for two rows at once, with the packed
// (c, c), (s, s), (-s, -s) built once per pair by the caller.
__device__ __forceinline__ void fma2(float &a0, float &a1, float x0, float x1, float y0, float y1) {
    const float2 r = __ffma2_rn(make_float2(x0, x1), make_float2(y0, y1), make_float2(a0, a1));
    a0 = r.x;
    a1 = r.y;
}
struct Rot2 {
    float2 c, s, ns;
    __device__ __forceinline__ Rot2(float c_, float s_)
        : c(make_float2(c_, c_)), s(make_float2(s_, s_)), ns(make_float2(-s_, -s_)) {}
};
__device__ __forceinline__ void rot2(float &x0, float &x1, float &y0, float &y1, const Rot2 &g) {
    const float2 x = make_float2(x0, x1), y = make_float2(y0, y1);
    const float2 t1 = __ffma2_rn(g.c, x, __fmul2_rn(g.ns, y));   // c x - s y
    const float2 t2 = __ffma2_rn(g.s, x, __fmul2_rn(g.c, y));    // s x + c y
    x0 = t1.x;
    x1 = t1.y;
    y0 = t2.x;
    y1 = t2.y;
}

// Register column of the first / second member of pair i in a step.
// CROSS steps pair x_i with y_i; INTRA steps pair positions (k, B-1-k) of
// each held block.
template <bool INTRA, int B>
__device__ __forceinline__ constexpr int pair_p(int i) {
    return INTRA ? (i < B / 2 ? i : B + (i - B / 2)) : i;
}
template <bool INTRA, int B>
__device__ __forceinline__ constexpr int pair_q(int i) {
    return INTRA ? (i < B / 2 ? B - 1 - i : 2 * B - 1 - (i - B / 2)) : B + i;
}

// One step: B disjoint pairs; ORs the pairs' rot_params flags into fl.
// FP32 tiles work on row pairs with packed instructions; rows >= nr of a
// lane are zero in the tile (tile_io), so a pair past nr adds nothing and
// stays zero.
template <bool INTRA, typename T, int B, int R, int RV>
__device__ __forceinline__ void step(Tile<T, B, R, RV> &t, T tol2, T big2, T ex2, T floor_, int &fl, bool rotate,
                                     int lane, int nr, int nv) {
    constexpr int LB = Log2<B>::value;
    constexpr bool PACK = sizeof(T) == 4 && R % 2 == 0 && RV % 2 == 0;
    T pa[B], pb[B], pc[B];
#pragma unroll
    for (int i = 0; i < B; ++i) {
        const int p = pair_p<INTRA, B>(i), q = pair_q<INTRA, B>(i);
        if constexpr (PACK) {
            float a0 = 0.f, a1 = 0.f, b0 = 0.f, b1 = 0.f, c0 = 0.f, c1 = 0.f;
#pragma unroll
            for (int r = 0; r < R; r += 2) {
                if (r < nr) {
                    const float x0 = t.w[p][r], x1 = t.w[p][r + 1], y0 = t.w[q][r], y1 = t.w[q][r + 1];
                    fma2(a0, a1, x0, x1, x0, x1);
                    fma2(b0, b1, y0, y1, y0, y1);
                    fma2(c0, c1, x0, x1, y0, y1);
                }
            }
            pa[i] = a0 + a1; pb[i] = b0 + b1; pc[i] = c0 + c1;
        } else {
            T a = 0, b = 0, c = 0;
#pragma unroll
            for (int r = 0; r < R; ++r) {
                if (r < nr) {
                    const T x = t.w[p][r], y = t.w[q][r];
                    a = dfma(x, x, a);
                    b = dfma(y, y, b);
                    c = dfma(x, y, c);
                }
            }
            pa[i] = a; pb[i] = b; pc[i] = c;
        }
    }
    reduce_scatter<T, B>(pa, lane);
    reduce_scatter<T, B>(pb, lane);
    reduce_scatter<T, B>(pc, lane);
    T c, s;
    int f;
    if constexpr (sizeof(T) == 8) f = rot_params_exact(pa[0], pb[0], pc[0], tol2, big2, ex2, floor_, c, s);
    else f = rot_params<T>(pa[0], pb[0], pc[0], tol2, big2, ex2, floor_, c, s);
    fl |= f;
    if (!rotate || !__any_sync(FULL, f != 0)) return;
#pragma unroll
    for (int i = 0; i < B; ++i) {
        const int src = i << (5 - LB);
        const T ci = __shfl_sync(FULL, c, src), si = __shfl_sync(FULL, s, src);
        const int p = pair_p<INTRA, B>(i), q = pair_q<INTRA, B>(i);
        if constexpr (PACK) {
            const Rot2 g((float)ci, (float)si);
#pragma unroll
            for (int r = 0; r < R; r += 2)
                if (r < nr) rot2(t.w[p][r], t.w[p][r + 1], t.w[q][r], t.w[q][r + 1], g);
#pragma unroll
            for (int r = 0; r < RV; r += 2)
                if (r < nv) rot2(t.v[p][r], t.v[p][r + 1], t.v[q][r], t.v[q][r + 1], g);
        } else {
#pragma unroll
            for (int r = 0; r < R; ++r) {
                if (r < nr) {
                    const T x = t.w[p][r], y = t.w[q][r];
                    t.w[p][r] = dfma(ci, x, -si * y);
                    t.w[q][r] = dfma(si, x, ci * y);
                }
            }
#pragma unroll
            for (int r = 0; r < RV; ++r) {
                if (r < nv) {
                    const T x = t.v[p][r], y = t.v[q][r];
                    t.v[p][r] = dfma(ci, x, -si * y);
                    t.v[q][r] = dfma(si, x, ci * y);
                }
            }
        }
    }
}

// Norm-update step: the squared column norms come from the tile instead of
// two more dot products, and each rotation updates them as it changes them;
// only w_p^T w_q is reduced across the warp.  FP32 (packed tiles):
// app - t|apq|, aqq + t|apq|.  FP64: the expansion c^2 app - 2cs apq + s^2 aqq
// (and its mirror) with the applied c and s, exact whatever the accuracy of
// the angle.  INTRA steps read and update the replicated t.nrm (every lane
// holds all 2B norms: the updated pair norms are broadcast).  CROSS steps
// pair x_i with y_i in lane group i, which holds just those two norms
// (t.nx, t.ny) and updates them itself, so they cost no broadcast; shift_y
// passes ny on to the neighbouring group.
template <bool INTRA, typename T, int B, int R, int RV>
__device__ __forceinline__ void step_upd(Tile<T, B, R, RV> &t, T tol2, T big2, T ex2, T floor_, int &fl,
                                         bool rotate, int lane, int nr, int nv) {
    constexpr int LB = Log2<B>::value;
    constexpr bool PACK = sizeof(T) == 4 && R % 2 == 0 && RV % 2 == 0;
    static_assert(PACK || sizeof(T) == 8, "norm-update steps: FP32 packed tiles or FP64");
    T pc[B];
#pragma unroll
    for (int i = 0; i < B; ++i) {
        const int p = pair_p<INTRA, B>(i), q = pair_q<INTRA, B>(i);
        if constexpr (PACK) {
            float c0 = 0.f, c1 = 0.f;
#pragma unroll
            for (int r = 0; r < R; r += 2)
                if (r < nr) fma2(c0, c1, t.w[p][r], t.w[p][r + 1], t.w[q][r], t.w[q][r + 1]);
            pc[i] = c0 + c1;
        } else {
            T c = 0;
#pragma unroll
            for (int r = 0; r < R; ++r)
                if (r < nr) c = dfma(t.w[p][r], t.w[q][r], c);
            pc[i] = c;
        }
    }
    reduce_scatter<T, B>(pc, lane);
    // this lane's pair (lane >> (5 - LB)): its two norms
    T app, aqq;
    if constexpr (INTRA) {
        const int li = lane >> (5 - LB);
        app = t.nrm[pair_p<INTRA, B>(0)];
        aqq = t.nrm[pair_q<INTRA, B>(0)];
#pragma unroll
        for (int i = 1; i < B; ++i)
            if (li == i) { app = t.nrm[pair_p<INTRA, B>(i)]; aqq = t.nrm[pair_q<INTRA, B>(i)]; }
    } else {
        app = t.nx;
        aqq = t.ny;
    }
    T c, s, sh;
    const int f = rot_params<T>(app, aqq, pc[0], tol2, big2, ex2, floor_, c, s, &sh);
    fl |= f;
    if (!rotate || !__any_sync(FULL, f != 0)) return;
    T np_, nq_;
    if constexpr (PACK) {
        np_ = app - sh;
        nq_ = aqq + sh;
    } else {
        const T cc = c * c, ss = s * s, x2 = T(2) * c * s * pc[0];
        np_ = dfma(cc, app, dfma(ss, aqq, -x2));
        nq_ = dfma(ss, app, dfma(cc, aqq, x2));
    }
    if constexpr (!INTRA) {
        t.nx = np_;
        t.ny = nq_;
    }
#pragma unroll
    for (int i = 0; i < B; ++i) {
        const int src = i << (5 - LB);
        const T ci = __shfl_sync(FULL, c, src), si = __shfl_sync(FULL, s, src);
        const int p = pair_p<INTRA, B>(i), q = pair_q<INTRA, B>(i);
        if constexpr (INTRA) {
            t.nrm[p] = __shfl_sync(FULL, np_, src);
            t.nrm[q] = __shfl_sync(FULL, nq_, src);
        }
        if constexpr (PACK) {
            const Rot2 g((float)ci, (float)si);
#pragma unroll
            for (int r = 0; r < R; r += 2)
                if (r < nr) rot2(t.w[p][r], t.w[p][r + 1], t.w[q][r], t.w[q][r + 1], g);
#pragma unroll
            for (int r = 0; r < RV; r += 2)
                if (r < nv) rot2(t.v[p][r], t.v[p][r + 1], t.v[q][r], t.v[q][r + 1], g);
        } else {
#pragma unroll
            for (int r = 0; r < R; ++r) {
                if (r < nr) {
                    const T x = t.w[p][r], y = t.w[q][r];
                    t.w[p][r] = dfma(ci, x, -si * y);
                    t.w[q][r] = dfma(si, x, ci * y);
                }
            }
#pragma unroll
            for (int r = 0; r < RV; ++r) {
                if (r < nv) {
                    const T x = t.v[p][r], y = t.v[q][r];
                    t.v[p][r] = dfma(ci, x, -si * y);
                    t.v[q][r] = dfma(si, x, ci * y);
                }
            }
        }
    }
}

// Cross-step norms from / to the replicated form: lane group i takes the
// norms of x_i (column i of the tile) and y_i (column B + i).
template <typename T, int B, int R, int RV>
__device__ __forceinline__ void norms_to_pairs(Tile<T, B, R, RV> &t, int lane) {
    constexpr int LB = Log2<B>::value;
    const int li = lane >> (5 - LB);
    t.nx = t.nrm[0];
    t.ny = t.nrm[B];
#pragma unroll
    for (int i = 1; i < B; ++i)
        if (li == i) { t.nx = t.nrm[i]; t.ny = t.nrm[B + i]; }
}

// y_i <- y_(i+1) (cyclic): the next CROSS step pairs x_i with the old y_(i+1).
// Norm-update sweeps: lane group i takes the norm of y_(i+1) from group i + 1.
template <int UPD, typename T, int B, int R, int RV>
__device__ __forceinline__ void shift_y(Tile<T, B, R, RV> &t, int lane) {
    if constexpr (UPD != 0) {
        constexpr int LB = Log2<B>::value;
        t.ny = __shfl_sync(FULL, t.ny, (lane + (32 >> LB)) & 31);
    }
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const T f = t.w[B][r];
#pragma unroll
        for (int i = 0; i < B - 1; ++i) t.w[B + i][r] = t.w[B + i + 1][r];
        t.w[2 * B - 1][r] = f;
    }
#pragma unroll
    for (int r = 0; r < RV; ++r) {
        const T f = t.v[B][r];
#pragma unroll
        for (int i = 0; i < B - 1; ++i) t.v[B + i][r] = t.v[B + i + 1][r];
        t.v[2 * B - 1][r] = f;
    }
}

// Circle rotation inside both blocks: positions 1..B-1 move one step right.
template <int UPD, typename T, int B, int R, int RV>
__device__ __forceinline__ void circle_shift(Tile<T, B, R, RV> &t) {
#pragma unroll
    for (int half = 0; half < 2; ++half) {
        const int o = half * B;
        if constexpr (UPD != 0) {
            const T last = t.nrm[o + B - 1];
#pragma unroll
            for (int i = B - 1; i >= 2; --i) t.nrm[o + i] = t.nrm[o + i - 1];
            t.nrm[o + 1] = last;
        }
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const T last = t.w[o + B - 1][r];
#pragma unroll
            for (int i = B - 1; i >= 2; --i) t.w[o + i][r] = t.w[o + i - 1][r];
            t.w[o + 1][r] = last;
        }
#pragma unroll
        for (int r = 0; r < RV; ++r) {
            const T last = t.v[o + B - 1][r];
#pragma unroll
            for (int i = B - 1; i >= 2; --i) t.v[o + i][r] = t.v[o + i - 1][r];
            t.v[o + 1][r] = last;
        }
    }
}

template <typename T, int B, int R, int RV>
__device__ __forceinline__ void tile_io(Tile<T, B, R, RV> &t, T *W, int ldw, T *V, int ldv, int X, int Y, int lane,
                                        bool store, int nr, int nv) {
#pragma unroll
    for (int c = 0; c < 2 * B; ++c) {
        const int col = (c < B ? X * B + c : Y * B + (c - B));
        T *w = W + (size_t)col * ldw + lane;
        T *v = V + (size_t)col * ldv + lane;
#pragma unroll
        for (int r = 0; r < R; ++r) {
            if (r < nr) {
                if (store) w[32 * r] = t.w[c][r];
                else t.w[c][r] = w[32 * r];
            } else if (!store) {
                t.w[c][r] = T(0);
            }
        }
#pragma unroll
        for (int r = 0; r < RV; ++r) {
            if (r < nv) {
                if (store) v[32 * r] = t.v[c][r];
                else t.v[c][r] = v[32 * r];
            } else if (!store) {
                t.v[c][r] = T(0);
            }
        }
    }
}

// The tile through the exchange area between block rounds (FP32, R a
// multiple of 4, RV of 2): lane-major, so that a lane's R rows of a W column
// are one 16-byte access and its RV rows of a V column one 8-byte access,
// instead of R + RV scalar accesses per column in the column-major W / V.
// Area: W part npb x 32 x R floats, then V part npb x 32 x RV floats.
template <typename T, int B, int R, int RV>
__device__ __forceinline__ void tile_x(Tile<T, B, R, RV> &t, T *xw, int npb, int X, int Y, int lane, bool store) {
    static_assert(sizeof(T) == 4 && R % 4 == 0 && RV % 2 == 0, "exchange area: FP32 tiles, R % 4 == 0, RV % 2 == 0");
    T *xv = xw + (size_t)npb * 32 * R;
#pragma unroll
    for (int c = 0; c < 2 * B; ++c) {
        const int col = (c < B ? X * B + c : Y * B + (c - B));
        float4 *pw = (float4 *)(xw + ((size_t)col * 32 + lane) * R);
        float2 *pv = (float2 *)(xv + ((size_t)col * 32 + lane) * RV);
#pragma unroll
        for (int k = 0; k < R / 4; ++k) {
            if (store) {
                pw[k] = make_float4(t.w[c][4 * k], t.w[c][4 * k + 1], t.w[c][4 * k + 2], t.w[c][4 * k + 3]);
            } else {
                const float4 v = pw[k];
                t.w[c][4 * k] = v.x; t.w[c][4 * k + 1] = v.y; t.w[c][4 * k + 2] = v.z; t.w[c][4 * k + 3] = v.w;
            }
        }
#pragma unroll
        for (int k = 0; k < RV / 2; ++k) {
            if (store) {
                pv[k] = make_float2(t.v[c][2 * k], t.v[c][2 * k + 1]);
            } else {
                const float2 v = pv[k];
                t.v[c][2 * k] = v.x; t.v[c][2 * k + 1] = v.y;
            }
        }
    }
}

// Bytes of the exchange area for npb columns: the tiles, then one float per
// column for the squared norms of the norm-update sweeps.
__host__ __device__ inline size_t xchg_bytes(int npb, int R, int RV) {
    return (size_t)npb * (32 * (R + RV) + 1) * 4;
}

// Squared column norms of the tile's 2B columns, reduced across the warp:
// afterwards nrm[0] on lane l is column l >> (5 - log2 2B)'s norm.
template <typename T, int B, int R, int RV>
__device__ __forceinline__ void tile_col_norms(const Tile<T, B, R, RV> &t, T (&nrm)[2 * B], int lane, int nr) {
#pragma unroll
    for (int c = 0; c < 2 * B; ++c) {
        T a = 0;
#pragma unroll
        for (int r = 0; r < R; ++r)
            if (r < nr) a = dfma(t.w[c][r], t.w[c][r], a);
        nrm[c] = a;
    }
    reduce_scatter<T, 2 * B>(nrm, lane);
}

// Norm-update sweeps: every lane gets all 2B exact norms of the tile.
template <typename T, int B, int R, int RV>
__device__ __forceinline__ void spread_norms(Tile<T, B, R, RV> &t, T n0) {
    constexpr int LB2 = Log2<2 * B>::value;
#pragma unroll
    for (int c = 0; c < 2 * B; ++c) t.nrm[c] = __shfl_sync(FULL, n0, c << (5 - LB2));
}

// The measuring sweep as one Gram pass: every pair ratio |w_p^T w_q| /
// (||w_p|| ||w_q||) of the current W (shared memory, column-major, ldw = 32 nr
// rows per lane) tested as rot_params tests it, without rotating.  A sweep
// with no rotation measures exactly these ratios (primitives.py:334-339), so
// "no active pair" here is the reference's convergence test (:352-353) at a
// fraction of a sweep's latency: 4 x 4 tiles of W^T W per warp, lanes over
// rows, one warp reduce-scatter per tile.  colnorm: npb doubles of shared
// memory.  All threads of the CTA call it; returns nonzero if a pair is active.
template <typename T>
__device__ int gram_check(const T *W, int ldw, int npb, int nr, T tol2, T floor_, double *colnorm) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = nwarps();
    for (int c = warp; c < npb; c += nw) {
        const T *w = W + (size_t)c * ldw + lane;
        T a = 0;
        for (int r = 0; r < nr; ++r) a = dfma(w[32 * r], w[32 * r], a);
        a = warp_sum(a);
        if (lane == 0) colnorm[c] = (double)a;
    }
    __syncthreads();
    const int nbk = npb >> 2;                      // 4-column blocks
    const int ntile = nbk * (nbk + 1) / 2;         // blocks bp <= bq
    int active = 0;
    for (int t = warp; t < ntile; t += nw) {
        int bp = 0, rem = t;                       // t -> (bp, bq), row-major upper triangle
        while (rem >= nbk - bp) { rem -= nbk - bp; ++bp; }
        const int bq = bp + rem;
        T acc[16];
#pragma unroll
        for (int v = 0; v < 16; ++v) acc[v] = 0;
        for (int r = 0; r < nr; ++r) {
            T x[4], y[4];
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                x[k] = W[(size_t)(4 * bp + k) * ldw + lane + 32 * r];
                y[k] = W[(size_t)(4 * bq + k) * ldw + lane + 32 * r];
            }
#pragma unroll
            for (int a = 0; a < 4; ++a)
#pragma unroll
                for (int b = 0; b < 4; ++b) acc[4 * a + b] = dfma(x[a], y[b], acc[4 * a + b]);
        }
        reduce_scatter<T, 16>(acc, lane);
        const int v = lane >> 1, a = v >> 2, b = v & 3;
        const int p = 4 * bp + a, q = 4 * bq + b;
        if (p < q) {
            const T app = (T)colnorm[p], aqq = (T)colnorm[q], apq = acc[0];
            if (apq * apq > tol2 * app * aqq && fmin(app, aqq) > floor_) active = 1;
        }
    }
    return __syncthreads_or(active);
}

// Sweeps over W/V in shared memory until off <= tol or max_sweeps.  nb blocks
// (even), of which the first `live` hold real columns; blocks >= live are
// zero and their pairs are skipped.  All threads of the CTA call this; warps
// >= nb/2 only take part in the barriers.  `red` needs 2*32 doubles.
// confirm: after a rotating sweep whose off is already below sqrt(tol)/2,
// run the next sweep without rotations; when it confirms off <= tol the
// reference would have rotated nothing in that sweep either.
// nr = ldw / 32 and nv = ldv / 32 are the rows per lane actually used
// (<= R, RV): one instantiation serves every matrix up to 32R x 32RV.
// exit_ratio > 0 (the first phase of the mixed solve): also stop after the
// first sweep whose largest ratio is <= exit_ratio -- the rotations of that
// sweep leave ~exit_ratio^2, below what FP32 sweeps resolve, and the FP64
// phase that follows takes it from there (converged is then set).
// colnorm (npb doubles of shared memory, or NULL): when given, a measuring
// sweep is replaced by gram_check.
// UPD: norm-update steps (step_upd); the norms are recomputed exactly at every
// sweep start, and then
//   UPD == 1: recomputed whenever a warp loads a new block pair from W / V,
//             so the updates accumulate over one block round at most; with
//             the exchange area (xbuf) carried with the tiles instead, so
//             they accumulate over a sweep (FP32 preconditioning sweeps);
//   UPD == 2: carried with the columns through colnorm (npb doubles of shared
//             memory) between block rounds, so they accumulate over a sweep
//             (FP64: the updates round like the dot products they replace).
// xbuf (FP32 tiles, or NULL): the exchange area (tile_x) that carries the
// tiles between block rounds; W and V are then read at the start and written
// at the end and before each Gram pass only, every layout change separated
// from the last access of the other layout by a CTA barrier.
template <typename T, int B, int R, int RV, int UPD = 0>
__device__ int rb_sweeps(T *W, int ldw, T *V, int ldv, int nb, int live, T tol, int max_sweeps, bool confirm,
                         double *red, bool &converged, T exit_ratio = T(0), double *colnorm = nullptr,
                         T *xbuf = nullptr) {
    const int nr = ldw >> 5, nv = ldv >> 5;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    constexpr int LB = Log2<B>::value;
    const int li = lane >> (5 - LB);   // the lane's pair in the cross steps
    const int nw = nwarps();
    const bool act = warp < nb / 2;
    Tile<T, B, R, RV> t;
    int rr = 0;
    int X = act ? circ(warp, 0, nb) : 0, Y = act ? circ(nb - 1 - warp, 0, nb) : 0;
    if (act) tile_io(t, W, ldw, V, ldv, X, Y, lane, false, nr, nv);
    bool measure = false, measure_allowed = confirm;
    const T tol2 = tol * tol, big2 = tol / T(4);  // ratio > tol, ratio > sqrt(tol)/2
    const T ex2 = exit_ratio * exit_ratio;
    converged = false;
    int sweep = 0;
    for (sweep = 1; sweep <= max_sweeps; ++sweep) {
        // Null-column floor from the column norms at the sweep start.
        T nmax = 0;
        if (act) {
            T nrm[2 * B];
            tile_col_norms(t, nrm, lane, nr);
            nmax = warp_max(nrm[0]);
            if constexpr (UPD != 0) spread_norms(t, nrm[0]);
        }
        if (lane == 0) red[warp] = (double)nmax;
        __syncthreads();
        double gm = red[0];
        for (int w = 1; w < nw; ++w) gm = fmax(gm, red[w]);
        const T floor_ = Lim<T>::eps() * Lim<T>::eps() * (T)gm;
        if (measure && colnorm) {
            // the measuring sweep as one Gram pass over the current W
            if (act) tile_io(t, W, ldw, V, ldv, X, Y, lane, true, nr, nv);
            __syncthreads();
            if (!gram_check<T>(W, ldw, nb * B, nr, tol2, floor_, colnorm)) { converged = true; break; }
            measure = false;
            measure_allowed = false;  // a failed confirmation: rotate from now on
            continue;
        }
        const bool rotate = !measure;
        int fl = 0;
        // The step loops are unrolled so that circle_shift / shift_y become
        // register renaming instead of moves.
        if (act && (X < live || Y < live)) {
#pragma unroll
            for (int j = 0; j < B - 1; ++j) {
                if constexpr (UPD != 0) step_upd<true>(t, tol2, big2, ex2, floor_, fl, rotate, lane, nr, nv);
                else step<true>(t, tol2, big2, ex2, floor_, fl, rotate, lane, nr, nv);
                circle_shift<UPD>(t);
            }
        }
        if constexpr (UPD != 0) {
            if (act) norms_to_pairs(t, lane);   // the cross steps keep each pair's norms in its lane group
        }
        for (int br = 0; br < nb - 1; ++br) {
            if (br > 0 || sweep > 1) {
                if (act) {
                    if constexpr (sizeof(T) == 4 && R == 4 && RV == 2) {   // the 128 x 64 tiles
                        if (xbuf) {
                            tile_x(t, xbuf, nb * B, X, Y, lane, true);
                            if constexpr (UPD == 1) {
                                // the updated norms travel with the tiles
                                T *xn = xbuf + (size_t)nb * B * 32 * (R + RV);
                                if ((lane & ((32 >> LB) - 1)) == 0) {
                                    xn[X * B + li] = t.nx;
                                    xn[Y * B + li] = t.ny;
                                }
                            }
                        } else {
                            tile_io(t, W, ldw, V, ldv, X, Y, lane, true, nr, nv);
                        }
                    } else {
                        tile_io(t, W, ldw, V, ldv, X, Y, lane, true, nr, nv);
                    }
                    if constexpr (UPD == 2) {
                        if ((lane & ((32 >> LB) - 1)) == 0) {
                            colnorm[X * B + li] = (double)t.nx;
                            colnorm[Y * B + li] = (double)t.ny;
                        }
                    }
                }
                __syncthreads();
                rr = rr + 1 == nb - 1 ? 0 : rr + 1;
                if (act) {
                    X = circ(warp, rr, nb);
                    Y = circ(nb - 1 - warp, rr, nb);
                    if constexpr (sizeof(T) == 4 && R == 4 && RV == 2) {   // the 128 x 64 tiles
                        if (xbuf) tile_x(t, xbuf, nb * B, X, Y, lane, false);
                        else tile_io(t, W, ldw, V, ldv, X, Y, lane, false, nr, nv);
                    } else {
                        tile_io(t, W, ldw, V, ldv, X, Y, lane, false, nr, nv);
                    }
                    if constexpr (UPD == 1) {
                        if (xbuf) {
                            const T *xn = xbuf + (size_t)nb * B * 32 * (R + RV);
                            t.nx = xn[X * B + li];
                            t.ny = xn[Y * B + li];
                        } else {
                            // nrm[0] on lane l: column l >> (5 - log2 2B) of the tile
                            T nrm[2 * B];
                            tile_col_norms(t, nrm, lane, nr);
                            t.nx = __shfl_sync(FULL, nrm[0], li << (4 - LB));
                            t.ny = __shfl_sync(FULL, nrm[0], (B + li) << (4 - LB));
                        }
                    } else if constexpr (UPD == 2) {
                        t.nx = (T)colnorm[X * B + li];
                        t.ny = (T)colnorm[Y * B + li];
                    }
                }
            }
            if (act && X < live && Y < live) {
#pragma unroll
                for (int j = 0; j < B; ++j) {
                    if constexpr (UPD != 0) step_upd<false>(t, tol2, big2, ex2, floor_, fl, rotate, lane, nr, nv);
                    else step<false>(t, tol2, big2, ex2, floor_, fl, rotate, lane, nr, nv);
                    shift_y<UPD>(t, lane);
                }
            }
        }
        // off <= tol  <=>  no active pair in the sweep (primitives.py:352).
        const int any_active = __syncthreads_or(fl & 1);
        const int any_big = __syncthreads_or(fl & 2);
        const int any_above_exit = __syncthreads_or(fl & 4);
        if (!any_active) { converged = true; break; }
        if (exit_ratio > T(0) && rotate && !any_above_exit) { converged = true; break; }
        if (measure) {
            measure = false;
            measure_allowed = false;  // a failed confirmation: rotate from now on
        } else if (measure_allowed && !any_big) {
            measure = true;
        }
    }
    if (act) tile_io(t, W, ldw, V, ldv, X, Y, lane, true, nr, nv);
    __syncthreads();
    return converged ? sweep : max_sweeps;
}

}  // namespace jb
