// jb_null.cu - null-space completion of U on the GPU
// (svdbench/standalone/primitives.py:430-455, complete_null_columns; used by
// complete_basis :458-467 and by _finish_columns, solvers.py:18-21).
//
// For every matrix of a batch U (batch x m x n, row-major) and its keep mask
// (batch x n bytes): the columns not kept are replaced, in ascending column
// order, by unit vectors orthogonal to all columns before them.  Per missing
// column, as the reference: idx = the first row of largest leftover leverage
// 1 - sum_c |u_ic|^2 (over the kept and the already completed columns),
// v = e_idx projected out against those columns, v / ||v||; ||v|| < 10 eps
// of the dtype fails the matrix (JB_ST_NULL_FAILED, primitives.py:451-452).
//
// B200 form.  The columns that count (kept, then completed ones in the order
// they are made) are packed into a work matrix X (m x a, row stride n), so
// every product reads a contiguous row prefix.  U^H e_idx is row idx of X,
// so the first projection is row-local: v_i = delta_{i,idx} - X_i . conj(X_idx).
// The leverage is kept per row in FP64 and lowered by |v_i|^2 after each new
// column; products accumulate in FP64 (complex: FP64 pairs).
//   * Many matrices (team of one CTA per matrix): the second projection
//     always runs, as in the reference.
//   * Few large matrices: one team of CTAs (about 64 rows each, at most one
//     per SM, cooperative launch) handles one matrix after another.  The
//     first projection's length^2 equals the pivot's leverage (v = P e_idx,
//     P the projector onto the complement), so while that leverage is at
//     least 1/2 a column costs one grid-wide barrier: v is normalised by it
//     directly (Kahan-Parlett "twice is enough": v is then orthogonal to the
//     columns to working accuracy and needs no second projection).  Below
//     1/2 the second projection runs, with the norm reduced over the team.
// Every barrier wait is bounded (about two seconds of globaltimer); a wait
// that runs out marks the team's matrix JB_ST_TIMEOUT and the CTAs return.
#include <cuda_runtime.h>
#include <stdint.h>
#include <math.h>
#include "jacobi_b200.h"

namespace jb {
namespace nul {

constexpr int kThreads = 512;
constexpr int kWarps = kThreads / 32;
constexpr unsigned long long kWaitNs = 2000000000ull;

struct cf { float x, y; };
struct cd { double x, y; };

// Element traits: storage type S, FP64 accumulation type A.
template <typename S> struct Tr;
template <> struct Tr<float> {
    using A = double;
    static constexpr bool cplx = false;
    static constexpr double eps = 1.1920928955078125e-07;
    __device__ static A zero() { return 0.0; }
    __device__ static A ld(const float *p) { return (double)*p; }
    __device__ static A ldcg(const float *p) { return (double)__ldcg(p); }
    __device__ static void st(float *p, A v) { *p = (float)v; }
    __device__ static A fma_(A acc, A x, A y) { return fma(x, y, acc); }
    __device__ static double norm2(A x) { return x * x; }
    __device__ static A scale(A x, double s) { return x * s; }
    __device__ static A sub(A x, A y) { return x - y; }
    __device__ static A add(A x, A y) { return x + y; }
    __device__ static A conj(A x) { return x; }
    __device__ static A ldcgA(const A *p) { return __ldcg(p); }
    __device__ static A unit() { return 1.0; }
    __device__ static A shfl_sum(A v) {
        for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        return v;
    }
};
template <> struct Tr<double> {
    using A = double;
    static constexpr bool cplx = false;
    static constexpr double eps = 2.220446049250313e-16;
    __device__ static A zero() { return 0.0; }
    __device__ static A ld(const double *p) { return *p; }
    __device__ static A ldcg(const double *p) { return __ldcg(p); }
    __device__ static void st(double *p, A v) { *p = v; }
    __device__ static A fma_(A acc, A x, A y) { return fma(x, y, acc); }
    __device__ static double norm2(A x) { return x * x; }
    __device__ static A scale(A x, double s) { return x * s; }
    __device__ static A sub(A x, A y) { return x - y; }
    __device__ static A add(A x, A y) { return x + y; }
    __device__ static A conj(A x) { return x; }
    __device__ static A ldcgA(const A *p) { return __ldcg(p); }
    __device__ static A unit() { return 1.0; }
    __device__ static A shfl_sum(A v) {
        for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        return v;
    }
};
template <typename S, typename R> struct TrC {
    using A = cd;
    static constexpr bool cplx = true;
    __device__ static A zero() { return {0.0, 0.0}; }
    __device__ static A ld(const S *p) { return {(double)p->x, (double)p->y}; }
    __device__ static A ldcg(const S *p) {
        const R *q = (const R *)p;
        return {(double)__ldcg(q), (double)__ldcg(q + 1)};
    }
    __device__ static void st(S *p, A v) { p->x = (R)v.x; p->y = (R)v.y; }
    __device__ static A fma_(A acc, A x, A y) {                          // acc + x * y
        return {fma(x.x, y.x, fma(-x.y, y.y, acc.x)), fma(x.x, y.y, fma(x.y, y.x, acc.y))};
    }
    __device__ static double norm2(A x) { return x.x * x.x + x.y * x.y; }
    __device__ static A scale(A x, double s) { return {x.x * s, x.y * s}; }
    __device__ static A sub(A x, A y) { return {x.x - y.x, x.y - y.y}; }
    __device__ static A add(A x, A y) { return {x.x + y.x, x.y + y.y}; }
    __device__ static A conj(A x) { return {x.x, -x.y}; }
    __device__ static A ldcgA(const A *p) { return {__ldcg(&p->x), __ldcg(&p->y)}; }
    __device__ static A unit() { return {1.0, 0.0}; }
    __device__ static A shfl_sum(A v) {
        for (int o = 16; o; o >>= 1) {
            v.x += __shfl_xor_sync(0xffffffffu, v.x, o);
            v.y += __shfl_xor_sync(0xffffffffu, v.y, o);
        }
        return v;
    }
};
template <> struct Tr<cf> : TrC<cf, float> { static constexpr double eps = 1.1920928955078125e-07; };
template <> struct Tr<cd> : TrC<cd, double> { static constexpr double eps = 2.220446049250313e-16; };

struct Slot {            // one CTA's contribution to a team-wide reduction
    double val;          // norm^2 partial, or the CTA's best leverage
    int64_t idx;         // row of the best leverage (first on ties)
};

struct Params {
    void *U;
    const uint8_t *keep;
    int32_t *status;
    int64_t batch, m, n;
    unsigned char *ws;   // per-team areas of team_bytes each
    size_t team_bytes;
    int G;               // CTAs per team (1: every CTA is a team)
    int always_reorth;
    int blocked;         // team path, real types: the blocked pass may run (block_pass)
};

__device__ __forceinline__ unsigned long long gtimer() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
    return t;
}

// Team-wide barrier.  G == 1: the CTA barrier.  G > 1: a two-level
// generation barrier over the whole (co-resident, cooperative) grid: CTAs
// arrive on the counter of their group of kGroupCTAs, the last of a group on
// the counter of groups, and the last group releases everyone by bumping the
// generation word, so no counter takes more than ~20 contending atomics.
// Waits are bounded; returns false once any CTA of the team gave up.
// bar[0] generation, bar[1] groups arrived, bar[2] error flag, bar[4 + k]
// CTAs of group k arrived (the area is zeroed before the launch).
constexpr int kGroupCTAs = 8;
__device__ __forceinline__ bool team_sync(unsigned *bar, int G) {
    __syncthreads();
    if (G == 1) return true;
    __shared__ int s_ok;
    if (threadIdx.x == 0) {
        volatile unsigned *vgen = bar;
        volatile int *verr = (volatile int *)(bar + 2);
        const unsigned gen = *vgen;
        __threadfence();
        const int grp = blockIdx.x / kGroupCTAs, ngroups = (G + kGroupCTAs - 1) / kGroupCTAs;
        const int gsize = min(kGroupCTAs, G - grp * kGroupCTAs);
        int ok = 1;
        if (atomicAdd(bar + 4 + grp, 1u) == (unsigned)gsize - 1) {
            atomicExch(bar + 4 + grp, 0u);
            __threadfence();
            if (atomicAdd(bar + 1, 1u) == (unsigned)ngroups - 1) {
                atomicExch(bar + 1, 0u);
                __threadfence();
                atomicAdd(bar, 1u);
            }
        }
        const unsigned long long t0 = gtimer();
        while (*vgen == gen) {
            if (gtimer() - t0 > kWaitNs) {
                ok = 0;
                atomicExch((int *)(bar + 2), 1);
                break;
            }
            __nanosleep(32);
        }
        __threadfence();
        s_ok = ok && !*verr;
    }
    __syncthreads();
    return s_ok != 0;
}

// Best (largest val, then smallest idx) of the CTA's candidates; result in
// thread 0.  `red` holds kWarps slots.
__device__ __forceinline__ Slot cta_argmax(double best, int64_t bidx, Slot *red) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int o = 16; o; o >>= 1) {
        const double ob = __shfl_xor_sync(0xffffffffu, best, o);
        const int64_t oi = __shfl_xor_sync(0xffffffffu, bidx, o);
        if (ob > best || (ob == best && oi < bidx)) { best = ob; bidx = oi; }
    }
    if (lane == 0) red[warp] = {best, bidx};
    __syncthreads();
    Slot s = red[0];
    if (threadIdx.x == 0)
        for (int w = 1; w < kWarps; ++w)
            if (red[w].val > s.val || (red[w].val == s.val && red[w].idx < s.idx)) s = red[w];
    __syncthreads();
    return s;
}

__device__ __forceinline__ double cta_sum(double v, double *red) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (lane == 0) red[warp] = v;
    __syncthreads();
    double s = 0.0;
    if (threadIdx.x == 0)
        for (int w = 0; w < kWarps; ++w) s += red[w];
    __syncthreads();
    return s;
}

// Team-wide reductions over the G slots, read by warp 0 only (one L2 read
// per slot per CTA) and broadcast through shared memory.
__device__ __forceinline__ Slot team_argmax(const Slot *slots, int G, bool team, Slot *s_slot) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (warp == 0) {
        double best = -1e300;
        int64_t bidx = 0;
        for (int q = lane; q < G; q += 32) {
            const double v = team ? __ldcg(&slots[q].val) : slots[q].val;
            const int64_t i = team ? __ldcg(&slots[q].idx) : slots[q].idx;
            if (v > best || (v == best && i < bidx)) { best = v; bidx = i; }
        }
        for (int o = 16; o; o >>= 1) {
            const double ob = __shfl_xor_sync(0xffffffffu, best, o);
            const int64_t oi = __shfl_xor_sync(0xffffffffu, bidx, o);
            if (ob > best || (ob == best && oi < bidx)) { best = ob; bidx = oi; }
        }
        if (lane == 0) *s_slot = {best, bidx};
    }
    __syncthreads();
    const Slot r = *s_slot;
    __syncthreads();
    return r;
}

// Sum of slots[q].val over q < G in a fixed order (the same value in every
// CTA): lane-strided partial sums combined by a fixed butterfly.
__device__ __forceinline__ double team_sum(const Slot *slots, int G, bool team, double *s_val) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (warp == 0) {
        double v = 0.0;
        for (int q = lane; q < G; q += 32) v += team ? __ldcg(&slots[q].val) : slots[q].val;
        for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (lane == 0) *s_val = v;
    }
    __syncthreads();
    const double r = *s_val;
    __syncthreads();
    return r;
}

// Row stride of the packed columns X: a multiple of 16 bytes, so that every
// row starts aligned for 16-byte vector loads.
__host__ __device__ inline int64_t x_stride(int64_t n, int esz) {
    const int64_t v = 16 / esz;
    return (n + v - 1) / v * v;
}

// Blocked pass of the team path (block_pass): the most candidate rows of a
// block, columns per block at most, K chunk of its row products, and the
// most rows a CTA may hold for it (its local sort).
constexpr int kCandMax = 256;
constexpr int kBlk = 32;
constexpr int kKC = 128;
constexpr int kSortMax = 1024;
static_assert(kCandMax % 64 == 0 && kBlk == 32 && kSortMax >= 64, "blocked pass sizes");

// Per-team workspace layout (byte offsets from the team's base).  X, the
// packed columns, and the blocked pass's areas exist only for multi-CTA teams:
// cand (every CTA's best rows), bm (the candidate block of the projector,
// kCandMax^2), bl (kBlk^2 triangular factor), bp (pivot rows), bv (pivot
// leverages), bmeta.
struct Layout {
    size_t x, lev, y, part, cmap, slots, bar, cand, bm, bl, bp, bv, bmeta, total;
};
__host__ __device__ inline size_t al256(size_t b) { return (b + 255) & ~(size_t)255; }
__host__ __device__ inline Layout layout(int64_t m, int64_t n, int esz, int asz, int G) {
    Layout L;
    size_t o = 0;
    const bool team = G > 1;
    L.x = o;     o += team ? al256((size_t)m * x_stride(n, esz) * esz) : 0;
    L.lev = o;   o += al256((size_t)m * 8);
    L.y = o;     o += al256((size_t)n * asz);
    L.part = o;  o += team ? al256((size_t)G * n * asz) : 0;
    L.cmap = o;  o += al256((size_t)n * 4);
    L.slots = o; o += al256((size_t)2 * G * sizeof(Slot));
    L.bar = o;   o += 256;
    L.cand = o;  o += team ? al256((size_t)kCandMax * sizeof(Slot)) : 0;
    L.bm = o;    o += team ? al256((size_t)kCandMax * kCandMax * 8) : 0;
    L.bl = o;    o += team ? al256((size_t)kBlk * kBlk * 8) : 0;
    L.bp = o;    o += team ? al256((size_t)kBlk * 8) : 0;
    L.bv = o;    o += team ? al256((size_t)kBlk * 8) : 0;
    L.bmeta = o; o += team ? 256 : 0;
    L.total = o;
    return L;
}

// Candidates each CTA of a team of G contributes (its best rows) and the
// candidate count padded to whole 64-row tiles: G q <= kCandMax.
__host__ __device__ inline int cand_per_cta(int G) {
    int q = kCandMax / G;
    return q > 64 ? 64 : (q < 1 ? 1 : q);
}
__host__ __device__ inline int cand_count(int G) { return (G * cand_per_cta(G) + 63) & ~63; }

// Dynamic shared memory of the blocked pass: the candidates (row, leverage),
// then the largest of its phases' work areas.
__host__ __device__ constexpr size_t block_smem() {
    constexpr size_t sort = (size_t)kSortMax * 16;
    constexpr size_t chol = (size_t)kCandMax * (kBlk + 1) * 8 + kCandMax * 8 + kBlk * 4 * 2 + 64;
    constexpr size_t rows = (size_t)kBlk * kBlk * 8 + kBlk * 8 * 2 + (size_t)(64 + kBlk) * (kKC + 1) * 8 +
                            (size_t)64 * (kBlk + 1) * 8 + 64 * 8 + kSortMax;
    constexpr size_t w = sort > chol ? (sort > rows ? sort : rows) : (chol > rows ? chol : rows);
    return (size_t)kCandMax * 16 + w;
}

// Rows are processed TPR threads per row, THREADS / TPR rows at a time, so a
// CTA has many independent loads in flight (the products stream X from L2).
constexpr int kTPR = 8;

// sum_k x[k] * (CONJ ? conj(r[k]) : r[k]) over k < na, this thread's share:
// k-chunks sub, sub + TPR, ... of VEC = 16 / sizeof(S) elements (16-byte
// loads when VECTOR: x 16-byte aligned, r in shared memory), four chunks in
// flight, then the scalar tail.
template <typename S, bool VECTOR, bool CONJ>
__device__ __forceinline__ typename Tr<S>::A row_dot(const S *x, const S *r, int na, int sub) {
    using T = Tr<S>;
    using A = typename T::A;
    constexpr int V = VECTOR ? 16 / (int)sizeof(S) : 1;
    union Pack { uint4 u; S s[16 / sizeof(S)]; };
    A acc0 = T::zero(), acc1 = T::zero();
    int k = 0;
    if (VECTOR) {
        const int nv = na / V;
        int j = sub;
        for (; j + 3 * kTPR < nv; j += 4 * kTPR) {
            Pack a[4], b[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                a[u].u = *(const uint4 *)(x + (size_t)(j + u * kTPR) * V);
                b[u].u = *(const uint4 *)(r + (size_t)(j + u * kTPR) * V);
            }
#pragma unroll
            for (int u = 0; u < 4; ++u)
#pragma unroll
                for (int e = 0; e < V; ++e) {
                    const A rv = CONJ ? T::conj(T::ld(&b[u].s[e])) : T::ld(&b[u].s[e]);
                    if (u & 1) acc1 = T::fma_(acc1, T::ld(&a[u].s[e]), rv);
                    else acc0 = T::fma_(acc0, T::ld(&a[u].s[e]), rv);
                }
        }
        for (; j < nv; j += kTPR) {
            Pack a, b;
            a.u = *(const uint4 *)(x + (size_t)j * V);
            b.u = *(const uint4 *)(r + (size_t)j * V);
#pragma unroll
            for (int e = 0; e < V; ++e)
                acc0 = T::fma_(acc0, T::ld(&a.s[e]), CONJ ? T::conj(T::ld(&b.s[e])) : T::ld(&b.s[e]));
        }
        k = nv * V;
    }
#pragma unroll 4
    for (int kk = k + sub; kk < na; kk += kTPR)
        acc1 = T::fma_(acc1, T::ld(x + kk), CONJ ? T::conj(T::ld(r + kk)) : T::ld(r + kk));
    return T::add(acc0, acc1);
}

// Sum over the kTPR consecutive lanes of a row group (all lanes take part).
template <typename A, typename T>
__device__ __forceinline__ A group_sum(A v) {
    for (int o = kTPR / 2; o; o >>= 1) {
        if constexpr (T::cplx) {
            v.x += __shfl_xor_sync(0xffffffffu, v.x, o);
            v.y += __shfl_xor_sync(0xffffffffu, v.y, o);
        } else {
            v += __shfl_xor_sync(0xffffffffu, v, o);
        }
    }
    return v;
}

// Order of the candidate rows: the larger leverage first, then the smaller
// row index (the reference's argmax takes the first of equal values).
__device__ __forceinline__ bool before(double va, int64_t ia, double vb, int64_t ib) {
    return va > vb || (va == vb && ia < ib);
}

// Rows rowA[0..64) (entries of INT64_MAX are zero rows) times rows
// rowB[0..32) of X over its first `a` columns, in FP64: Yb (64 x 32, ld
// kBlk + 1) = X_A X_B^T.  Staged through shared memory in FP64, kKC columns
// at a time, the next chunk's loads in flight (registers) while the current
// one is multiplied: warp w stages rows w + 16 j, lanes the columns.  Each
// thread owns 4 x 4 outputs (rows r + 16 v, four consecutive columns) of one
// quarter of the chunk's columns, the quarters summed at the end.  All
// threads of the CTA call it.
template <typename S>
__device__ void rows_dot(const S *X, int64_t ldx, int a, const int64_t *rowA, const int64_t *rowB, double *Xr,
                         double *Xs, double *Yb) {
    constexpr int LDK = kKC + 1, LDY = kBlk + 1, NW = kThreads / 32;
    constexpr int KC = sizeof(S) == 8 ? kKC / 2 : kKC;     // chunk: FP64 storage keeps half in flight
    constexpr int RA = 64 / NW, RB = kBlk / NW, KL = KC / 32;    // rows per warp, columns per lane
    static_assert(kThreads == 512 && kKC % 32 == 0, "rows_dot layout");
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int kq = tid >> 7, t7 = tid & 127, rr = t7 & 15, cg = t7 >> 4;   // K quarter, row, column group
    const S *pa[RA], *pb[RB];
#pragma unroll
    for (int j = 0; j < RA; ++j) {
        const int64_t row = rowA[warp + NW * j];
        pa[j] = row != INT64_MAX ? X + row * ldx : nullptr;
    }
#pragma unroll
    for (int j = 0; j < RB; ++j) {
        const int64_t row = rowB[warp + NW * j];
        pb[j] = row != INT64_MAX ? X + row * ldx : nullptr;
    }
    S va[RA][KL], vb[RB][KL];                              // the next chunk, in the storage type
    auto fetch = [&](int k0) {
#pragma unroll
        for (int u = 0; u < KL; ++u) {
            const int k = k0 + lane + 32 * u;
            const bool in = k < a;
#pragma unroll
            for (int j = 0; j < RA; ++j) va[j][u] = in && pa[j] ? __ldcg(pa[j] + k) : S(0);
#pragma unroll
            for (int j = 0; j < RB; ++j) vb[j][u] = in && pb[j] ? __ldcg(pb[j] + k) : S(0);
        }
    };
    auto stage = [&]() {
#pragma unroll
        for (int u = 0; u < KL; ++u) {
#pragma unroll
            for (int j = 0; j < RA; ++j) Xr[(warp + NW * j) * LDK + lane + 32 * u] = (double)va[j][u];
#pragma unroll
            for (int j = 0; j < RB; ++j) Xs[(warp + NW * j) * LDK + lane + 32 * u] = (double)vb[j][u];
        }
    };
    double acc[4][4];
#pragma unroll
    for (int v = 0; v < 4; ++v)
#pragma unroll
        for (int u = 0; u < 4; ++u) acc[v][u] = 0.0;
    fetch(0);
    stage();
    __syncthreads();
    for (int k0 = 0; k0 < a; k0 += KC) {
        const int kc = (a - k0) < KC ? (a - k0) : KC;
        const bool more = k0 + KC < a;
        if (more) fetch(k0 + KC);                          // in flight during the products
        for (int k = kq; k < kc; k += 4) {
            double x[4], y[4];
#pragma unroll
            for (int v = 0; v < 4; ++v) x[v] = Xr[(rr + 16 * v) * LDK + k];
#pragma unroll
            for (int u = 0; u < 4; ++u) y[u] = Xs[(4 * cg + u) * LDK + k];
#pragma unroll
            for (int v = 0; v < 4; ++v)
#pragma unroll
                for (int u = 0; u < 4; ++u) acc[v][u] = fma(x[v], y[u], acc[v][u]);
        }
        __syncthreads();
        if (more) {
            stage();
            __syncthreads();
        }
    }
    // the four quarters, summed in a fixed order
    for (int q4 = 0; q4 < 4; ++q4) {
        if (kq == q4)
#pragma unroll
            for (int v = 0; v < 4; ++v)
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    double *y = Yb + (rr + 16 * v) * LDY + 4 * cg + u;
                    *y = q4 ? *y + acc[v][u] : acc[v][u];
                }
        __syncthreads();
    }
}

// This CTA's best q rows by leverage ("before" order: bitonic sort of its
// nrow <= kSortMax rows in `work`), written to out[0..q).
__device__ void publish_best(const double *lev, int64_t r0, int nrow, int q, Slot *out, unsigned char *work) {
    double *kv = (double *)work;
    int64_t *ki = (int64_t *)(work + (size_t)kSortMax * 8);
    const int tid = threadIdx.x;
    int np2 = 64;
    while (np2 < nrow || np2 < q) np2 <<= 1;
    for (int i = tid; i < np2; i += kThreads) {
        kv[i] = i < nrow ? lev[r0 + i] : -1e300;
        ki[i] = i < nrow ? r0 + i : INT64_MAX;
    }
    __syncthreads();
    for (int k = 2; k <= np2; k <<= 1)
        for (int j = k >> 1; j > 0; j >>= 1) {
            for (int i = tid; i < np2; i += kThreads) {
                const int ixj = i ^ j;
                if (ixj > i) {
                    const bool up = (i & k) == 0;
                    const bool sw = up ? before(kv[ixj], ki[ixj], kv[i], ki[i]) : before(kv[i], ki[i], kv[ixj], ki[ixj]);
                    if (sw) {
                        const double tv = kv[i];
                        kv[i] = kv[ixj];
                        kv[ixj] = tv;
                        const int64_t ti = ki[i];
                        ki[i] = ki[ixj];
                        ki[ixj] = ti;
                    }
                }
            }
            __syncthreads();
        }
    for (int i = tid; i < q; i += kThreads) out[i] = {kv[i], ki[i]};
    __syncthreads();
}

// Blocked pass of the team path (real types).  The missing columns are the
// pivoted Cholesky factor of the projector P = I - X X^T onto the complement
// of the packed columns X, pivot = the largest leverage (P's remaining
// diagonal), exactly as the per-column loop builds them: column k =
// P_k e_p / sqrt(lev_p).  A block of up to kBlk columns is built
// speculatively on a candidate set C (every CTA's best rows), then checked:
//   P2  M = P[C, C] (diagonal: the tracked leverages; off-diagonal
//       -X_i . X_j in FP64), shared out over the team in 64 x 32 tiles;
//   P3  CTA 0: the pivoted Cholesky of M, pivot = the best remaining
//       leverage in C, until kBlk columns, the missing columns run out, or
//       the best is below 1/2 (the per-column loop then takes that column,
//       with its second projection);
//   P4  every CTA forms its rows of the block, Y = E_S - X X_S^T and
//       N = Y L_SS^-T (forward substitution with the factor's pivot rows),
//       stores N as the next packed columns, and checks every row outside C
//       step by step: a row whose leverage at step s ranks before the
//       pivot's would have been step s's pivot, so the block keeps only the
//       steps before the first such s (step 0 always stands: the best row of
//       every CTA is in C);
//   P5  the leverages lowered by |N_i|^2 over the kept steps, the slots and
//       the next block's candidates published.
// The kept pivots and columns are, in exact arithmetic, the per-column
// loop's, at four team barriers per block instead of one per column.
// `fresh`: the candidate lists match the current leverages (else P1
// publishes them first).  Returns the columns completed (0: the per-column
// loop takes the next one), or -1 when a barrier wait ran out; `slow` is set
// when the block ended on a leverage below 1/2.
template <typename S>
__device__ int block_pass(const Params &p, const Layout &L, unsigned char *base, S *X, int64_t ldx, double *lev,
                          int a, const uint8_t *keep, int64_t c, int *cmap, Slot *slots, unsigned *bar,
                          unsigned char *smem, int G, int g, int64_t r0, int64_t r1, bool &fresh, bool &slow,
                          Slot *s_red) {
    using T = Tr<S>;
    constexpr unsigned FULL = 0xffffffffu;
    constexpr int LDK = kKC + 1, LDY = kBlk + 1;
    const int64_t n = p.n;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int q = cand_per_cta(G), nc = cand_count(G), nreal = G * q;
    Slot *cand = (Slot *)(base + L.cand);
    double *bm = (double *)(base + L.bm);
    double *bl = (double *)(base + L.bl);
    int64_t *bp = (int64_t *)(base + L.bp);
    double *bpv = (double *)(base + L.bv);
    int *bmeta = (int *)(base + L.bmeta);
    int64_t *cidx = (int64_t *)smem;                       // candidates: row, leverage
    double *cval = (double *)(smem + kCandMax * 8);
    unsigned char *work = smem + kCandMax * 16;
    __shared__ int s_nmiss, s_fail;
    const int nrow = (int)(r1 - r0);
    slow = false;

    if (!fresh) {                                          // P1
        publish_best(lev, r0, nrow, q, cand + (size_t)g * q, work);
        if (!team_sync(bar, G)) return -1;
    }
    fresh = false;
    // P2
    for (int i = tid; i < nc; i += kThreads) {
        cidx[i] = i < nreal ? __ldcg(&cand[i].idx) : INT64_MAX;
        cval[i] = i < nreal ? __ldcg(&cand[i].val) : -1e300;
    }
    __syncthreads();
    {
        double *Xr = (double *)work, *Xs = Xr + 64 * LDK, *Yb = Xs + kBlk * LDK;
        const int tcol = nc / kBlk, tiles = (nc / 64) * tcol;
        for (int tt = g; tt < tiles; tt += G) {
            const int i0 = 64 * (tt / tcol), j0 = kBlk * (tt % tcol);
            rows_dot<S>(X, ldx, a, cidx + i0, cidx + j0, Xr, Xs, Yb);
            for (int e = tid; e < 64 * kBlk; e += kThreads) {
                const int r = e / kBlk, cc = e - r * kBlk, ia = i0 + r, jb = j0 + cc;
                const bool ok = cidx[ia] != INT64_MAX && cidx[jb] != INT64_MAX;
                bm[(size_t)ia * nc + jb] = ia == jb ? (ok ? cval[ia] : 0.0) : (ok ? -Yb[r * LDY + cc] : 0.0);
            }
            __syncthreads();
        }
    }
    if (!team_sync(bar, G)) return -1;

    // P3: CTA 0, the pivoted Cholesky of M
    if (g == 0) {
        constexpr int LDL = kBlk + 1;                      // odd: candidates' rows in different banks
        double *Lc = (double *)work;                       // L[t][s], nc x kBlk (ld LDL)
        double *d = Lc + (size_t)kCandMax * LDL;           // remaining leverage of candidate t
        int *pa = (int *)(d + kCandMax);                   // candidate of pivot s
        int *cols = pa + kBlk;                             // U column of pivot s
        for (int i = tid; i < nc * LDL; i += kThreads) Lc[i] = 0.0;
        for (int i = tid; i < nc; i += kThreads) d[i] = cidx[i] != INT64_MAX ? cval[i] : -1e300;
        if (tid == 0) {
            int k = 0;
            for (int64_t cc = c; cc < n && k < kBlk; ++cc)
                if (!keep[cc]) cols[k++] = (int)cc;
            s_nmiss = k;
        }
        __syncthreads();
        const int nmax = s_nmiss;
        int ns = 0, stop_slow = 0;
        // the best remaining candidate: each warp's best of its 32 (after the
        // step's update), then the warps' bests in shared memory
        __shared__ double s_wv[kWarps];
        __shared__ int64_t s_wi[kWarps];
        __shared__ int s_wa[kWarps];
        auto warp_best = [&]() {
            double bv = -1e300;
            int64_t bi = INT64_MAX;
            int ba = -1;
            for (int t = tid; t < nc; t += kThreads)
                if (d[t] > -1e299 && before(d[t], cidx[t], bv, bi)) { bv = d[t]; bi = cidx[t]; ba = t; }
            for (int o = 16; o; o >>= 1) {
                const double ov = __shfl_xor_sync(FULL, bv, o);
                const int64_t oi = __shfl_xor_sync(FULL, bi, o);
                const int oa = __shfl_xor_sync(FULL, ba, o);
                if (before(ov, oi, bv, bi)) { bv = ov; bi = oi; ba = oa; }
            }
            if (lane == 0) { s_wv[warp] = bv; s_wi[warp] = bi; s_wa[warp] = ba; }
        };
        auto cta_best = [&](double &bv, int &ba) {
            bv = s_wv[0];
            int64_t bi = s_wi[0];
            ba = s_wa[0];
            for (int w = 1; w < kWarps; ++w)
                if (before(s_wv[w], s_wi[w], bv, bi)) { bv = s_wv[w]; bi = s_wi[w]; ba = s_wa[w]; }
        };
        warp_best();
        __syncthreads();
        for (; ns < nmax; ++ns) {
            double bv;
            int pb;
            cta_best(bv, pb);
            if (pb < 0 || bv < 0.5) {
                stop_slow = pb >= 0;
                break;
            }
            const double lpp = sqrt(bv);
            for (int t = tid; t < nc; t += kThreads) {
                if (t == pb) {
                    Lc[t * LDL + ns] = lpp;
                    d[t] = -1e300;                         // pivoted
                } else if (d[t] > -1e299) {
                    const double mt = __ldcg(bm + (size_t)pb * nc + t);   // row pb of M (symmetric), in flight
                    double acc0 = 0.0, acc1 = 0.0;
                    int u = 0;
                    for (; u + 1 < ns; u += 2) {
                        acc0 = fma(Lc[t * LDL + u], Lc[pb * LDL + u], acc0);
                        acc1 = fma(Lc[t * LDL + u + 1], Lc[pb * LDL + u + 1], acc1);
                    }
                    if (u < ns) acc0 = fma(Lc[t * LDL + u], Lc[pb * LDL + u], acc0);
                    const double l = (mt - (acc0 + acc1)) / lpp;
                    Lc[t * LDL + ns] = l;
                    d[t] -= l * l;
                }
            }
            if (tid == 0) {
                pa[ns] = pb;
                bpv[ns] = bv;
            }
            __syncthreads();                               // everyone has read this step's s_w*
            warp_best();                                   // each thread's candidates are its own: no barrier before
            __syncthreads();
        }
        for (int i = tid; i < ns * kBlk; i += kThreads) {
            const int s2 = i / kBlk, t = i - s2 * kBlk;
            bl[i] = t <= s2 ? Lc[pa[s2] * LDL + t] : 0.0;
        }
        for (int i = tid; i < ns; i += kThreads) {
            bp[i] = cidx[pa[i]];
            cmap[a + i] = cols[i];
        }
        if (tid == 0) {
            bmeta[0] = ns;
            bmeta[1] = stop_slow;
            bmeta[2] = ns;                                 // the first failing step (P4), at most ns
        }
    }
    if (!team_sync(bar, G)) return -1;
    const int ns = __ldcg(bmeta);
    if (ns == 0) {
        slow = __ldcg(bmeta + 1) != 0;
        fresh = true;                                      // the leverages did not change
        return 0;
    }

    // P4: this CTA's rows of the block, 64 at a time, and the check
    double *Ls = (double *)work;                           // kBlk x kBlk
    int64_t *Sv = (int64_t *)(Ls + kBlk * kBlk);           // pivot rows
    double *Pv = (double *)(Sv + kBlk);                    // pivot leverages
    double *Xr = Pv + kBlk;                                // 64 x kKC (ld LDK)
    double *Xs = Xr + 64 * LDK;                            // kBlk x kKC (ld LDK)
    double *Yb = Xs + kBlk * LDK;                          // 64 x kBlk (ld LDY)
    int64_t *rowsA = (int64_t *)(Yb + 64 * LDY);           // this chunk's rows
    unsigned char *incand = (unsigned char *)(rowsA + 64); // own rows in C
    for (int i = tid; i < ns * kBlk; i += kThreads) Ls[i] = __ldcg(bl + i);
    for (int i = tid; i < kBlk; i += kThreads) {
        Sv[i] = i < ns ? __ldcg(bp + i) : INT64_MAX;
        Pv[i] = i < ns ? __ldcg(bpv + i) : 0.0;
    }
    for (int i = tid; i < nrow; i += kThreads) incand[i] = 0;
    if (tid == 0) s_fail = ns;
    __syncthreads();
    for (int i = tid; i < nc; i += kThreads)
        if (cidx[i] >= r0 && cidx[i] < r1) incand[cidx[i] - r0] = 1;
    __syncthreads();
    int fail = ns;
    for (int64_t rc = r0; rc < r1; rc += 64) {
        const int nr = (int)((r1 - rc) < 64 ? (r1 - rc) : 64);
        if (tid < 64) rowsA[tid] = tid < nr ? rc + tid : INT64_MAX;
        __syncthreads();
        rows_dot<S>(X, ldx, a, rowsA, Sv, Xr, Xs, Yb);
        if (tid < nr) {
            const int64_t i = rc + tid;
            double *yr = Yb + tid * LDY;
            const bool check = !incand[i - r0];
            double lv = lev[i];
            for (int s2 = 0; s2 < ns; ++s2) {
                if (check && s2 < fail && before(lv, i, Pv[s2], Sv[s2])) fail = s2;
                double y0 = (i == Sv[s2] ? 1.0 : 0.0) - yr[s2], y1 = 0.0;
                int t = 0;
                for (; t + 1 < s2; t += 2) {
                    y0 = fma(-yr[t], Ls[s2 * kBlk + t], y0);
                    y1 = fma(-yr[t + 1], Ls[s2 * kBlk + t + 1], y1);
                }
                if (t < s2) y0 = fma(-yr[t], Ls[s2 * kBlk + t], y0);
                const double y = (y0 + y1) / Ls[s2 * kBlk + s2];
                yr[s2] = y;
                const S ys = (S)y;                         // the stored value, as the leverage sees it
                X[i * ldx + a + s2] = ys;
                lv -= (double)ys * (double)ys;
            }
        }
        __syncthreads();
    }
    if (fail < ns) atomicMin(&s_fail, fail);
    __syncthreads();
    if (tid == 0 && s_fail < ns) atomicMin(bmeta + 2, s_fail);
    if (!team_sync(bar, G)) return -1;
    const int kept = __ldcg(bmeta + 2);

    // P5: leverages over the kept steps, slots, the next candidates
    double best = -1e300;
    int64_t bidx = 0;
    for (int64_t i = r0 + tid; i < r1; i += kThreads) {
        double lv = lev[i];
        const S *xi = X + i * ldx + a;
#pragma unroll 8
        for (int s2 = 0; s2 < kept; ++s2) {
            const double x = (double)__ldcg(xi + s2);
            lv -= x * x;
        }
        lev[i] = lv;
        if (lv > best) { best = lv; bidx = i; }
    }
    const Slot sb = cta_argmax(best, bidx, s_red);
    if (tid == 0) slots[g] = sb;
    publish_best(lev, r0, nrow, q, cand + (size_t)g * q, work);
    if (!team_sync(bar, G)) return -1;
    fresh = true;
    slow = kept == ns && __ldcg(bmeta + 1) != 0;
    return kept;
}

// TEAM = false: one CTA per matrix, in place on U (the columns not yet
// completed are zero, so every product runs over all n columns, as the
// reference's u @ (u^H v) does; the new column is excluded from the second
// projection).  TEAM = true: a cooperative team of G CTAs, the kept and
// completed columns packed into X (row stride x_stride(n)), G > 1.
template <typename S, bool TEAM>
__global__ void __launch_bounds__(kThreads, 1) null_kernel(Params p) {
    using T = Tr<S>;
    using A = typename T::A;
    constexpr int kGroups = kThreads / kTPR;
    extern __shared__ __align__(16) unsigned char smem[];
    S *rowc = (S *)smem;                                   // row idx of X; y in the second projection
    __shared__ Slot s_red[kWarps];
    __shared__ double s_dred[kWarps];
    __shared__ int s_flag;
    __shared__ Slot s_piv;
    __shared__ double s_sum;
    const int G = TEAM ? p.G : 1;
    const int g = TEAM ? blockIdx.x : 0;                   // rank in the team
    const int64_t team = TEAM ? 0 : blockIdx.x;
    const int64_t nteams = TEAM ? 1 : gridDim.x;
    const int64_t m = p.m, n = p.n;
    const int64_t ldx = TEAM ? x_stride(n, sizeof(S)) : n;
    const Layout L = layout(m, n, sizeof(S), sizeof(A), G);
    unsigned char *base = p.ws + team * p.team_bytes;
    double *lev = (double *)(base + L.lev);
    A *y = (A *)(base + L.y);
    A *part = (A *)(base + L.part);
    int *cmap = (int *)(base + L.cmap);
    Slot *slots = (Slot *)(base + L.slots);                // [2][G]
    unsigned *bar = (unsigned *)(base + L.bar);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int sub = threadIdx.x % kTPR, grp = threadIdx.x / kTPR;
    const int64_t r0 = m * g / G, r1 = m * (g + 1) / G;   // this CTA's rows
    // cross-CTA data is read through L2 (ld.global.cg): L1 is not coherent
    auto ldx_ = [&](const S *q) -> A { return TEAM ? T::ldcg(q) : T::ld(q); };
    auto ldy = [&](const A *q) -> A { return TEAM ? T::ldcgA(q) : *q; };
    int64_t z = team;
    for (; z < p.batch; z += nteams) {
        S *U = (S *)p.U + z * m * n;
        S *X = TEAM ? (S *)(base + L.x) : U;
        const uint8_t *keep = p.keep + z * n;
        if (warp == 0) {                                   // kept columns in order (cmap), by ballots
            int a = 0, miss = 0;
            for (int64_t c0 = 0; c0 < n; c0 += 32) {
                const int64_t c = c0 + lane;
                const bool in = c < n, kp = in && keep[c] != 0;
                const unsigned bk = __ballot_sync(0xffffffffu, kp);
                if (TEAM && kp) cmap[a + __popc(bk & ((1u << lane) - 1u))] = (int)c;
                a += __popc(bk);
                miss += __popc(__ballot_sync(0xffffffffu, in && !kp));
            }
            if (lane == 0) s_flag = miss ? a : -1;
        }
        __syncthreads();
        const int nkept = s_flag;
        if (nkept < 0) {                                   // nothing to complete
            if (g == 0 && threadIdx.x == 0) p.status[z] = JB_ST_OK;
            __syncthreads();                               // s_flag is rewritten for the next matrix
            continue;
        }
        // Zero U's missing columns (primitives.py:436), pack the kept ones
        // (TEAM), leverage of every row of this CTA in FP64.
        double best = -1e300;
        int64_t bidx = 0;
        for (int64_t i = r0 + warp; i < r1; i += kWarps) {
            S *urow = U + i * n;
            double acc = 0.0;
            for (int64_t c = lane; c < n; c += 32) {
                if (!keep[c]) T::st(urow + c, T::zero());
                else acc += T::norm2(T::ld(urow + c));
            }
            if (TEAM)
                for (int k = lane; k < nkept; k += 32) X[i * ldx + k] = urow[cmap[k]];
            for (int o = 16; o; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
            const double lv = 1.0 - acc;
            if (lane == 0) lev[i] = lv;
            if (lv > best) { best = lv; bidx = i; }         // lanes agree; rows ascend
        }
        Slot sb = cta_argmax(best, bidx, s_red);
        if (threadIdx.x == 0) slots[g] = sb;
        if (!team_sync(bar, G)) goto timeout;
        {
            int a = nkept;                                 // packed columns (TEAM)
            bool failed = false;
            bool blocked = TEAM && !T::cplx && p.blocked;  // block_pass while it applies
            bool fresh = false;                            // its candidate lists are current
            for (int64_t c = 0; c < n; ++c) {
                if (keep[c]) continue;
                if constexpr (TEAM && !T::cplx) {
                    if (blocked) {
                        bool slow = false;
                        const int done = block_pass<S>(p, L, base, X, ldx, lev, a, keep, c, cmap, slots, bar, smem, G,
                                                       g, r0, r1, fresh, slow, s_red);
                        if (done < 0) goto timeout;
                        if (slow) blocked = false;
                        if (done > 0) {
                            a += done;
                            c = __ldcg(&cmap[a - 1]);              // the last column of the block
                            continue;
                        }
                    }
                    fresh = false;                         // the per-column step changes the leverages
                }
                const int na = TEAM ? a : (int)n;          // columns a product runs over
                const int64_t col = TEAM ? a : c;          // where v is built
                // idx = team-wide first argmax of the leverage
                const Slot piv = team_argmax(slots, G, TEAM, &s_piv);
                const int64_t idx = piv.idx;
                // The first projection's length^2 is the pivot's leverage (v = P e_idx
                // with P the projector onto the complement, so |v|^2 = P_idx,idx).  A
                // team that needs no second projection (leverage >= 1/2) normalises
                // by it at once and saves the team-wide norm reduction.
                const bool fast = TEAM && piv.val >= 0.5;
                const double inv_fast = fast ? 1.0 / sqrt(piv.val) : 0.0;
                for (int k = threadIdx.x; k < na; k += kThreads) T::st(rowc + k, ldx_(X + idx * ldx + k));
                __syncthreads();
                // first projection, row-local: v_i = delta - X_i . conj(X_idx)
                // (column col of X is still zero in every row)
                double pn2 = 0.0;
                best = -1e300;
                bidx = 0;
                for (int64_t i0 = r0; i0 < r1; i0 += kGroups) {
                    const int64_t i = i0 + grp;
                    A acc = i < r1 ? row_dot<S, TEAM, true>(X + i * ldx, rowc, na, sub) : T::zero();
                    acc = group_sum<A, T>(acc);
                    if (sub == 0 && i < r1) {
                        const A v = T::sub(i == idx ? T::unit() : T::zero(), acc);
                        if (fast) {
                            T::st(X + i * ldx + col, T::scale(v, inv_fast));
                            const double lv = lev[i] - T::norm2(T::ld(X + i * ldx + col));
                            lev[i] = lv;
                            if (lv > best) { best = lv; bidx = i; }
                        } else {
                            T::st(X + i * ldx + col, v);
                            pn2 += T::norm2(T::ld(X + i * ldx + col));
                        }
                    }
                }
                if (fast) {
                    sb = cta_argmax(best, bidx, s_red);
                    if (threadIdx.x == 0) {
                        slots[g] = sb;
                        if (g == 0) cmap[a] = (int)c;
                    }
                    ++a;
                    if (!team_sync(bar, G)) goto timeout;
                    continue;
                }
                double n2 = cta_sum(pn2, s_dred);
                if (threadIdx.x == 0) slots[G + g].val = n2;
                if (!team_sync(bar, G)) goto timeout;
                n2 = team_sum(slots + G, G, TEAM, &s_sum);
                if (p.always_reorth || n2 < 0.5) {
                    // second projection: y = X^H v (without v's own column), v -= X y
                    A *yout = TEAM ? part + (size_t)g * n : y;
                    for (int k = threadIdx.x; k < na; k += kThreads) {
                        A acc0 = T::zero(), acc1 = T::zero();
                        if (k != col) {
                            int64_t i = r0;
                            for (; i + 1 < r1; i += 2) {
                                acc0 = T::fma_(acc0, T::conj(T::ld(X + i * ldx + k)), T::ld(X + i * ldx + col));
                                acc1 = T::fma_(acc1, T::conj(T::ld(X + (i + 1) * ldx + k)),
                                               T::ld(X + (i + 1) * ldx + col));
                            }
                            if (i < r1) acc0 = T::fma_(acc0, T::conj(T::ld(X + i * ldx + k)), T::ld(X + i * ldx + col));
                        }
                        yout[k] = T::add(acc0, acc1);
                    }
                    if (TEAM) {
                        // every CTA sums the partials of its slice of y
                        if (!team_sync(bar, G)) goto timeout;
                        const int64_t k0 = (int64_t)na * g / G, k1 = (int64_t)na * (g + 1) / G;
                        for (int64_t k = k0 + threadIdx.x; k < k1; k += kThreads) {
                            A acc = T::zero();
                            for (int q = 0; q < G; ++q) acc = T::add(acc, T::ldcgA(part + (size_t)q * n + k));
                            y[k] = acc;
                        }
                    }
                    if (!team_sync(bar, G)) goto timeout;
                    // y in the input precision, as the reference's product (rowc is free again)
                    for (int k = threadIdx.x; k < na; k += kThreads) T::st(rowc + k, ldy(y + k));
                    __syncthreads();
                    double pn2b = 0.0;
                    for (int64_t i0 = r0; i0 < r1; i0 += kGroups) {
                        const int64_t i = i0 + grp;
                        A acc = i < r1 ? row_dot<S, TEAM, false>(X + i * ldx, rowc, na, sub) : T::zero();
                        acc = group_sum<A, T>(acc);
                        if (sub == 0 && i < r1) {
                            T::st(X + i * ldx + col, T::sub(T::ld(X + i * ldx + col), acc));
                            pn2b += T::norm2(T::ld(X + i * ldx + col));
                        }
                    }
                    const double s2 = cta_sum(pn2b, s_dred);
                    if (threadIdx.x == 0) slots[G + g].val = s2;
                    if (!team_sync(bar, G)) goto timeout;
                    n2 = team_sum(slots + G, G, TEAM, &s_sum);
                }
                const double len = sqrt(n2);
                if (len < 10.0 * T::eps) {                 // primitives.py:451-452
                    failed = true;
                    break;
                }
                // normalise, lower the leverage, next argmax
                const double inv = 1.0 / len;
                best = -1e300;
                bidx = 0;
                for (int64_t i = r0 + threadIdx.x; i < r1; i += kThreads) {
                    T::st(X + i * ldx + col, T::scale(T::ld(X + i * ldx + col), inv));
                    const double lv = lev[i] - T::norm2(T::ld(X + i * ldx + col));
                    lev[i] = lv;
                    if (lv > best) { best = lv; bidx = i; }
                }
                sb = cta_argmax(best, bidx, s_red);
                if (threadIdx.x == 0) {
                    slots[g] = sb;
                    if (TEAM && g == 0) cmap[a] = (int)c;
                }
                ++a;
                if (!team_sync(bar, G)) goto timeout;
            }
            if (TEAM)                                      // completed columns back into U
                for (int64_t i = r0 + warp; i < r1; i += kWarps)
                    for (int k = nkept + lane; k < a; k += 32) U[i * n + __ldcg(&cmap[k])] = X[i * ldx + k];
            if (g == 0 && threadIdx.x == 0) p.status[z] = failed ? JB_ST_NULL_FAILED : JB_ST_OK;
            if (!team_sync(bar, G)) goto timeout;
        }
    }
    return;
timeout:
    // a barrier wait ran out: this matrix and the team's later ones fail
    if (threadIdx.x == 0 && g == 0)
        for (; z < p.batch; z += nteams) p.status[z] = JB_ST_TIMEOUT;
}

struct Plan {
    int G, blocked;
    int64_t grid;
    size_t team_bytes, bytes, smem;
};

static int esize(int dtype) { return dtype == 0 ? 4 : dtype == 1 ? 8 : dtype == 2 ? 8 : 16; }

static int dev_sms() {
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return 148;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms < 1) return 148;
    return sms;
}

// One CTA per matrix unless the batch has few large matrices: then one
// cooperative team of up to one CTA per SM (about 64 rows each).
static Plan make_plan(int dtype, int64_t batch, int64_t m, int64_t n) {
    Plan pl;
    const int sms = dev_sms();
    const int esz = esize(dtype), asz = dtype >= 2 ? 16 : 8;
    const bool large = batch * 4 < sms && m * n >= (1 << 16) && m >= 256;
    pl.blocked = 0;
    if (large) {
        int64_t G = m / 64;                         // about 64 rows per CTA
        if (G > sms) G = sms;
        if (G < 2) G = 2;
        pl.G = (int)G;
        pl.grid = G;
        pl.team_bytes = layout(m, n, esz, asz, pl.G).total;
        pl.bytes = pl.team_bytes;
        // real types, at most kSortMax rows per CTA: the blocked pass
        pl.blocked = dtype <= 1 && (m + G - 1) / G <= kSortMax;
    } else {
        pl.G = 1;
        int64_t grid = (int64_t)sms * 4;
        if (grid > batch) grid = batch;
        if (grid < 1) grid = 1;
        pl.grid = grid;
        pl.team_bytes = layout(m, n, esz, asz, 1).total;
        pl.bytes = pl.team_bytes * (size_t)grid;
    }
    pl.smem = (size_t)n * esz;
    if (pl.blocked && pl.smem < block_smem()) pl.smem = block_smem();
    return pl;
}

template <typename S>
static int launch(Params &p, const Plan &pl, cudaStream_t st) {
    p.G = pl.G;
    p.team_bytes = pl.team_bytes;
    p.always_reorth = pl.G == 1;
    p.blocked = pl.blocked;
    if (pl.G == 1) {
        auto kern = null_kernel<S, false>;
        if (pl.smem > 48 * 1024 &&
            cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)pl.smem) != cudaSuccess)
            return JB_ECUDA;
        kern<<<(unsigned)pl.grid, kThreads, pl.smem, st>>>(p);
        return cudaGetLastError() == cudaSuccess ? JB_OK : JB_ECUDA;
    }
    auto kern = null_kernel<S, true>;
    if (pl.smem > 48 * 1024 &&
        cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)pl.smem) != cudaSuccess)
        return JB_ECUDA;
    // the barrier words and the error flag start at zero
    const Layout L = layout(p.m, p.n, sizeof(S), Tr<S>::cplx ? 16 : 8, pl.G);
    if (cudaMemsetAsync(p.ws + L.bar, 0, 256, st) != cudaSuccess) return JB_ECUDA;
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kThreads, pl.smem) != cudaSuccess)
        return JB_ECUDA;
    if ((int64_t)per_sm * dev_sms() < pl.grid) return JB_ETOOBIG;   // every CTA must be resident
    void *args[] = {&p};
    if (cudaLaunchCooperativeKernel((const void *)kern, dim3((unsigned)pl.grid), dim3(kThreads), args, pl.smem,
                                    st) != cudaSuccess)
        return JB_ECUDA;
    return JB_OK;
}

}  // namespace nul
}  // namespace jb

using namespace jb::nul;

extern "C" {

size_t jb_complete_null_workspace_bytes(int32_t dtype, int64_t batch, int64_t m, int64_t n) {
    if (dtype < 0 || dtype > 3 || batch < 0 || m < 1 || n < 1) return 0;
    return make_plan(dtype, batch, m, n).bytes;
}

int jb_complete_null(void *U, const uint8_t *keep, int32_t dtype, int64_t batch, int64_t m, int64_t n,
                     int32_t *status, void *workspace, size_t workspace_bytes, void *stream) {
    if (!U || !keep || !status || dtype < 0 || dtype > 3 || batch < 0 || m < 1 || n < 1) return JB_EINVAL;
    if (n > 8192 || m > ((int64_t)1 << 31) / n) return JB_ETOOBIG;
    if (batch == 0) return JB_OK;
    const Plan pl = make_plan(dtype, batch, m, n);
    if (pl.smem > 227 * 1024) return JB_ETOOBIG;
    if (!workspace || workspace_bytes < pl.bytes) return JB_EWORKSPACE;
    Params p;
    p.U = U;
    p.keep = keep;
    p.status = status;
    p.batch = batch;
    p.m = m;
    p.n = n;
    p.ws = (unsigned char *)workspace;
    cudaStream_t st = (cudaStream_t)stream;
    switch (dtype) {
        case 0: return launch<float>(p, pl, st);
        case 1: return launch<double>(p, pl, st);
        case 2: return launch<cf>(p, pl, st);
        default: return launch<cd>(p, pl, st);
    }
}

}  // extern "C"
