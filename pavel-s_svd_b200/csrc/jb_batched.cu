// jb_batched.cu - persistent batched one-sided Jacobi SVD for sm_100a and
// the C-ABI entry points declared in include/jacobi_b200.h.
//
// One CTA solves one matrix at a time and then takes the next one from a
// work list (an atomic ticket for uneven batches, a grid stride for equal
// shapes), so an uneven batch of thousands of matrices is ONE launch and can
// be captured in a CUDA graph.  Everything of svd(a, 'jacobi') for one matrix
// happens inside the CTA: finiteness scan, exact power-of-two scaling,
// wide->tall transposition, sweeps with per-matrix convergence (no host
// synchronisation), sort, cut, normalisation, null-space completion, full
// bases and the final writes of U, S and Vh.
#include <cuda_runtime.h>
#include <stdint.h>
#include <string.h>
#include <mutex>
#include "jacobi_b200.h"
#include "jb_device.cuh"
#include "jb_regblock.cuh"
#include "jb_gram64.cuh"

namespace jb {

// ---------------------------------------------------------------------------
// Work-area layout, shared by host (sizing) and device (carving).
// ---------------------------------------------------------------------------
__host__ __device__ inline size_t align16(size_t x) { return (x + 15) & ~(size_t)15; }

struct Dims {
    int mt, nt, np, ncp, ldw, ldv;
};

__host__ __device__ inline Dims dims_of(int mt, int nt, int flags) {
    Dims d;
    d.mt = mt; d.nt = nt;
    d.np = nt + (nt & 1);
    d.ncp = (flags & JB_FULL_MATRICES) ? d.np + (mt - nt) : d.np;
    d.ldw = mt | 1;
    d.ldv = d.np | 1;
    return d;
}

// Bytes of the matrix work area (W, V and the mixed-precision aliases).
__host__ __device__ inline size_t region_bytes(const Dims &d, int elem, int precision) {
    if (precision == JB_PREC_MIXED && elem == 4) {
        size_t v64 = align16((size_t)d.ldv * d.np * 8);
        size_t w64 = (size_t)d.ldw * d.ncp * 8;
        size_t w32 = align16((size_t)d.ldw * d.np * 4) + (size_t)d.ldv * d.np * 4;
        size_t q = (size_t)d.ldv * d.np * 8;
        size_t w = w64 > w32 ? w64 : w32;
        w = w > q ? w : q;
        return v64 + align16(w);
    }
    return align16((size_t)d.ldw * d.ncp * elem) + align16((size_t)d.ldv * d.np * elem);
}

__host__ __device__ inline size_t aux_bytes(const Dims &d) {
    const int npairs = d.np / 2;
    const int vecn = (d.mt > d.ncp ? d.mt : d.ncp) + 32;
    return align16((size_t)3 * npairs * 8) + align16((size_t)d.np * 8) + align16((size_t)vecn * 8) +
           align16((size_t)d.np * 8) + align16((size_t)d.np * 4) + align16(64 * 8) + align16(4 * 4);
}

__device__ inline Aux carve_aux(unsigned char *base, const Dims &d) {
    Aux a;
    const int npairs = d.np / 2;
    const int vecn = (d.mt > d.ncp ? d.mt : d.ncp) + 32;
    unsigned char *p = base;
    a.app = (double *)p; a.aqq = a.app + npairs; a.apq = a.aqq + npairs; p += align16((size_t)3 * npairs * 8);
    a.sig = (double *)p; p += align16((size_t)d.np * 8);
    a.vec = (double *)p; p += align16((size_t)vecn * 8);
    a.tau = (double *)p; p += align16((size_t)d.np * 8);
    a.perm = (int *)p; p += align16((size_t)d.np * 4);
    a.red = (double *)p; p += align16(64 * 8);
    a.flag = (int *)p;
    return a;
}

struct Params {
    const void *A;
    void *U, *S, *Vh;
    const jb_matrix_desc *descs;  // NULL: equal shapes (um, un, urank, uflags)
    const int32_t *order;         // NULL: identity order
    int64_t count;
    int32_t um, un, urank, uflags;
    double tol;                   // <= 0: 10 eps(dtype)
    int32_t max_sweeps;
    double tol32;                 // first (FP32) phase of the mixed solve
    int32_t max_sweeps32;
    int32_t *sweeps, *status;
    int *counter;                 // NULL: static grid-stride schedule
    int *counter2;                // ticket of the second (FP64) kernel
    int from_x32;                 // mixed round-robin solve: start from the FP32 V in x32 (large-tile K1)
    float exit_ratio;             // mixed FP32 phase exit ratio (0: kMixedExitRatio, < 0: run to tol)
    unsigned char *gws;           // NULL: work area in shared memory
    size_t gws_stride;
    Dims maxd;                    // sizing of aux / region (largest matrix)
    const float *vstart;          // warm start: nt x nt start V per matrix (x_off), or NULL
    float *x32;                   // mixed scratch (V of the FP32 phase)
    int64_t x_cap;                // floats available at x32
    size_t region_cap;            // bytes of the shared-memory work area
    int cls;                      // 0: every matrix; 1: only nt > kNarrowN; 2: only nt <= kNarrowN
    int xchg;                     // register FP32 kernels: tile exchange area (tile_x) ...
    size_t xchg_off;              // ... at this byte offset in the work area (after W / V; it may share the
                                  //     warm-start staging of A, which is dead once the sweeps start)
};

__device__ inline jb_matrix_desc desc_of(const Params &p, int64_t mat) {
    if (p.descs) return p.descs[mat];
    jb_matrix_desc d;
    d.m = p.um; d.n = p.un; d.rank = p.urank; d.flags = p.uflags;
    const int64_t ucols = (p.uflags & JB_FULL_MATRICES) ? p.um : p.urank;
    const int64_t vrows = (p.uflags & JB_FULL_MATRICES) ? p.un : p.urank;
    d.a_off = mat * (int64_t)p.um * p.un;
    d.u_off = mat * (int64_t)p.um * ucols;
    d.s_off = mat * (int64_t)p.urank;
    d.v_off = mat * vrows * (int64_t)p.un;
    const int64_t nt = p.um < p.un ? p.um : p.un;
    d.x_off = mat * nt * nt;
    return d;
}

// A descriptor is solved only if its work area fits the one the launch was
// sized for (checked on the device: the host cannot read device descriptors).
__device__ inline bool desc_fits(const jb_matrix_desc &d, const Dims &maxd) {
    if (d.m < 1 || d.n < 1) return false;
    const int mt = d.m > d.n ? d.m : d.n, nt = d.m > d.n ? d.n : d.m;
    if (d.rank < 1 || d.rank > nt) return false;
    if ((d.flags & JB_FULL_MATRICES) && d.rank != nt) return false;
    const Dims dd = dims_of(mt, nt, d.flags);
    return mt <= maxd.mt && nt <= maxd.nt && dd.ncp <= maxd.ncp;
}

// Native-precision solve of one matrix (T = input type).
template <typename T>
__device__ int solve_native(const Params &p, const jb_matrix_desc &d, unsigned char *region, Aux &ax,
                            int &nsweeps) {
    const Geo g = make_geo(d.m, d.n, d.rank, d.flags);
    const T *A = (const T *)p.A + d.a_off;
    T *W = (T *)region;
    T *V = (T *)(region + align16((size_t)g.ldw * g.ncp * sizeof(T)));
    bool bad;
    const int e = scan_input(A, g.m * g.n, ax, bad);
    nsweeps = 0;
    if (bad) return JB_ST_NONFINITE_IN;
    load_tall(A, g, e, W);
    set_identity(V, g.np, g.ldv);
    __syncthreads();
    const T tol = p.tol > 0 ? (T)p.tol : T(10) * Lim<T>::eps();
    bool conv;
    nsweeps = sweeps<T>(W, V, g, tol, p.max_sweeps, ax, conv);
    if (!conv) return JB_ST_NOT_CONVERGED;
    T *U = p.U ? (T *)p.U + d.u_off : nullptr;
    T *Vh = p.Vh ? (T *)p.Vh + d.v_off : nullptr;
    return epilogue<T, T>(W, V, g, e, U, (T *)p.S + d.s_off, Vh, ax);
}

// Mixed solve of one f32 matrix: FP32 sweeps, Householder re-orthonormalised
// V in FP64, W = A V in FP64, FP64 sweeps to the same tolerance.
__device__ int solve_mixed(const Params &p, const jb_matrix_desc &d, unsigned char *region, Aux &ax,
                           int &nsweeps) {
    const int k1_sweeps = nsweeps;  // FP32 sweeps of the large-tile kernel (from_x32)
    const Geo g = make_geo(d.m, d.n, d.rank, d.flags);
    const float *A = (const float *)p.A + d.a_off;
    double *V64 = (double *)region;
    double *W64 = (double *)(region + align16((size_t)g.ldv * g.np * 8));
    float *W32 = (float *)W64;
    float *V32 = (float *)((unsigned char *)W64 + align16((size_t)g.ldw * g.np * 4));
    bool bad;
    const int e = scan_input(A, g.m * g.n, ax, bad);
    nsweeps = 0;
    if (bad) return JB_ST_NONFINITE_IN;
    int s1 = 0;
    if (p.from_x32) {
        // the FP32 sweeps ran in the large-tile kernel: V (nt x nt,
        // column-major) in x32, identity on the padding column
        s1 = k1_sweeps;
        const float *x = p.x32 + d.x_off;
        for (int idx = threadIdx.x; idx < g.np * g.np; idx += blockDim.x) {
            const int c = idx / g.np, i = idx - c * g.np;
            V64[(size_t)c * g.ldv + i] = (c < g.nt && i < g.nt) ? (double)x[(size_t)c * g.nt + i] : (c == i ? 1.0 : 0.0);
        }
    } else {
        Geo g32 = g;
        g32.ncp = g.np;
        load_tall(A, g32, e, W32);
        set_identity(V32, g.np, g.ldv);
        __syncthreads();
        const float tol32 = p.tol32 > 0 ? (float)p.tol32 : 10.0f * Lim<float>::eps();
        bool conv32;
        s1 = sweeps<float>(W32, V32, g32, tol32, p.max_sweeps32, ax, conv32);
        for (int idx = threadIdx.x; idx < g.np * g.np; idx += blockDim.x) {
            int c = idx / g.np, i = idx - c * g.np;
            V64[(size_t)c * g.ldv + i] = (double)V32[(size_t)c * g.ldv + i];
        }
    }
    __syncthreads();
    householder_orthonormalize(V64, g.np, g.ldv, W64, g.ldv, ax);
    // W64[:, j] = A_t V64[:, j]  (A_t: scaled tall view of A, zero padding).
    for (int idx = threadIdx.x; idx < g.mt * g.np; idx += blockDim.x) {
        const int j = idx / g.mt, i = idx - j * g.mt;
        const double *v = V64 + (size_t)j * g.ldv;
        double acc = 0.0;
        for (int k = 0; k < g.nt; ++k) {
            const float a = g.wide ? A[(size_t)k * g.n + i] : A[(size_t)i * g.n + k];
            acc = fma(ldexp((double)a, -e), v[k], acc);
        }
        W64[(size_t)j * g.ldw + i] = acc;
    }
    for (int j = g.np; j < g.ncp; ++j)
        for (int i = threadIdx.x; i < g.mt; i += blockDim.x) W64[(size_t)j * g.ldw + i] = 0.0;
    __syncthreads();
    const double tol = p.tol > 0 ? (double)(float)p.tol : (double)(10.0f * Lim<float>::eps());
    bool conv;
    const int s2 = sweeps<double>(W64, V64, g, tol, p.max_sweeps, ax, conv);
    nsweeps = s1 + s2;
    if (!conv) return JB_ST_NOT_CONVERGED;
    float *U = p.U ? (float *)p.U + d.u_off : nullptr;
    float *Vh = p.Vh ? (float *)p.Vh + d.v_off : nullptr;
    return epilogue<double, float>(W64, V64, g, e, U, (float *)p.S + d.s_off, Vh, ax);
}

template <typename T, int PREC>
__global__ void __launch_bounds__(1024, 1) batched_kernel(Params p) {
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ int s_idx;
    Aux ax = carve_aux(smem, p.maxd);
    unsigned char *region = p.gws ? p.gws + (size_t)blockIdx.x * p.gws_stride
                                  : smem + aux_bytes(p.maxd);
    int64_t idx = blockIdx.x;
    for (;;) {
        if (p.counter) {
            if (threadIdx.x == 0) s_idx = atomicAdd(p.counter, 1);
            __syncthreads();
            idx = s_idx;
            __syncthreads();
        }
        if (idx >= p.count) break;
        const int64_t mat = p.order ? (int64_t)p.order[idx] : idx;
        const jb_matrix_desc d = desc_of(p, mat);
        if (threadIdx.x < 4) ax.flag[threadIdx.x] = 0;
        __syncthreads();
        int ns = 0, st;
        int prev = JB_ST_OK;
        if (PREC == JB_PREC_MIXED && p.from_x32) {
            // K1 (large-tile FP32 sweeps) left its status and sweep count
            if (threadIdx.x == 0) { ax.flag[3] = p.status[mat]; ax.flag[2] = p.sweeps[mat]; }
            __syncthreads();
            prev = ax.flag[3];
            ns = ax.flag[2];
            __syncthreads();
            if (threadIdx.x == 0) ax.flag[2] = 0;
            __syncthreads();
        }
        if (prev != JB_ST_OK) st = prev;
        else if (!desc_fits(d, p.maxd)) st = JB_ST_BAD_DESC;
        else if (PREC == JB_PREC_MIXED) st = solve_mixed(p, d, region, ax, ns);
        else st = solve_native<T>(p, d, region, ax, ns);
        if (threadIdx.x == 0) {
            if (p.status) p.status[mat] = st;
            if (p.sweeps) p.sweeps[mat] = ns;
        }
        __syncthreads();
        if (!p.counter) idx += gridDim.x;
    }
}


// ---------------------------------------------------------------------------
// Register-tile path (matrices up to 128 x 64 in their tall view).
// ---------------------------------------------------------------------------
constexpr int kB32 = 4;   // block width of the FP32 sweeps (8 warps for 64 columns)
constexpr int kB32L = 4;  // block width of the large-tile FP32 kernel (16 warps for 128 columns)
// Mixed precision: the FP32 phase ends after the first sweep whose largest
// pair ratio is <= this (quadratic convergence leaves ~1e-4 after it); the
// FP64 phase then converges to the requested tolerance in one rotating sweep
// and one confirming sweep, as it does from a fully converged FP32 phase.
constexpr float kMixedExitRatio = 1e-2f;
// Launch choices jb_svd_uneven_f32_ex accepts in `flags` (an autotuner picks among them).
constexpr int kTuneFlags = JB_ROUND_ROBIN | JB_BLOCK_WIDTH_8 | JB_ONE_SIZE_CLASS;
constexpr int kB64 = 2;   // block width of the FP64 sweeps (16 warps for 64 columns)
constexpr int kT32 = 256, kT64 = 512;  // threads of the two kernels
constexpr int kMaxR = 4;  // rows per lane: mt <= 128
// Size classes of the register path: matrices with nt <= kNarrowN occupy at
// most half of the warps of a CTA (kT32 / kT64), so they run in a second
// launch with CTAs of half the size and twice as many CTAs per SM.
constexpr int kNarrowN = 32;
constexpr int kMaxRV = 2; // V rows per lane: padded width <= 64
// Large-tile FP32 kernel (one matrix up to 256 x 128 per CTA, 16 warps).
constexpr int kT32L = 512, kMaxRL = 8, kMaxRVL = 4;

struct RGeo {
    int R, RV, nb, npb, live, ldw, ldv, ncp;
};

__host__ __device__ inline RGeo rgeo(int mt, int nt, int B, int flags) {
    RGeo r;
    r.R = (mt + 31) / 32;
    r.nb = 2 * ((nt + 2 * B - 1) / (2 * B));
    r.npb = r.nb * B;
    r.RV = (r.npb + 31) / 32;
    r.live = (nt + B - 1) / B;
    r.ldw = 32 * r.R;
    r.ldv = 32 * r.RV;
    r.ncp = (flags & JB_FULL_MATRICES) ? r.npb + (mt - nt) : r.npb;
    return r;
}

__host__ __device__ inline size_t rregion_bytes(const RGeo &r, int elem) {
    return align16((size_t)r.ldw * r.ncp * elem) + align16((size_t)r.ldv * r.npb * elem);
}

// FP64 polish of a float32 matrix: W | V | X1 (npb x npb doubles) | X2
// (npb x npb doubles, or the float32 staging of A, ldw x nt).
__host__ __device__ inline size_t xbytes(const RGeo &r, int nt) {
    const size_t a = (size_t)r.ldw * nt * 4, b = (size_t)r.ldv * r.npb * 8;
    return align16(a > b ? a : b);
}
__host__ __device__ inline size_t rregion_mixed64(const RGeo &r, int nt) {
    return rregion_bytes(r, 8) + align16((size_t)r.ldv * r.npb * 8) + xbytes(r, nt);
}

// Aux sizing for the register path: np -> padded width, mt -> row stride.
__host__ __device__ inline Dims raux_dims(const RGeo &r) {
    Dims d;
    d.mt = r.ldw; d.nt = r.npb; d.np = r.npb; d.ncp = r.ncp; d.ldw = r.ldw; d.ldv = r.ldv;
    return d;
}

// Whether a launch with class filter cls (Params::cls) takes this matrix.
__device__ inline bool class_takes(const jb_matrix_desc &d, int cls) {
    if (cls == 0) return true;
    const bool narrow = (d.m < d.n ? d.m : d.n) <= kNarrowN;
    return cls == 2 ? narrow : !narrow;
}

__device__ inline bool rdesc_fits(const jb_matrix_desc &d, int B, int elem, const Params &p, bool mixed_scratch,
                                  int max_r = kMaxR, int max_rv = kMaxRV) {
    if (d.m < 1 || d.n < 1) return false;
    const int mt = d.m > d.n ? d.m : d.n, nt = d.m > d.n ? d.n : d.m;
    if (d.rank < 1 || d.rank > nt) return false;
    if ((d.flags & JB_FULL_MATRICES) && d.rank != nt) return false;
    const RGeo r = rgeo(mt, nt, B, d.flags);
    if (r.R > max_r || r.RV > max_rv) return false;
    size_t need = (mixed_scratch && elem == 8) ? rregion_mixed64(r, nt) : rregion_bytes(r, elem);
    if (elem == 4 && p.vstart) need += align16((size_t)r.ldw * nt * 4);
    if (need > p.region_cap) return false;
    if (r.ldw > p.maxd.mt || r.npb > p.maxd.np || r.ncp > p.maxd.ncp) return false;
    if (mixed_scratch && (d.x_off < 0 || d.x_off + (int64_t)nt * nt > p.x_cap)) return false;
    return true;
}

template <typename T>
__device__ void zero_fill(T *X, size_t count) {
    for (size_t i = threadIdx.x; i < count; i += blockDim.x) X[i] = T(0);
}

// W = scaled tall view of A (rows < mt, cols < nt); the rest of W and V must
// already be zero.  V = I on the padded width.
template <typename T, typename TI>
__device__ void load_padded(const TI *A, const Geo &g, const RGeo &r, int e, T *W, T *V) {
    const int total = g.m * g.n;
    for (int idx = threadIdx.x; idx < total; idx += blockDim.x) {
        const int row = idx / g.n, col = idx - row * g.n;
        const int i = g.wide ? col : row, j = g.wide ? row : col;
        W[(size_t)j * r.ldw + i] = dscale((T)A[idx], -e);
    }
    for (int j = threadIdx.x; j < r.npb; j += blockDim.x) V[(size_t)j * r.ldv + j] = T(1);
}

// A_t (tall view of A, float, rows < mt) into As (ld x nt, zero-filled).
template <typename TI>
__device__ void load_stage(const TI *A, const Geo &g, int ld, float *As) {
    const int total = g.m * g.n;
    for (int k = threadIdx.x; k < total; k += blockDim.x) {
        const int row = k / g.n, col = k - row * g.n;
        const int i = g.wide ? col : row, j = g.wide ? row : col;
        As[(size_t)j * ld + i] = (float)A[k];
    }
}

template <typename T, int B, int MR = kMaxR, int MRV = kMaxRV, int UPD = 0>
__device__ int rb_dispatch(const RGeo &r, T *W, T *V, T tol, int max_sweeps, bool confirm, double *red,
                           bool &conv, T exit_ratio = T(0), double *colnorm = nullptr, T *xbuf = nullptr) {
    return rb_sweeps<T, B, MR, MRV, UPD>(W, r.ldw, V, r.ldv, r.nb, r.live, tol, max_sweeps, confirm, red, conv,
                                    exit_ratio, colnorm, xbuf);
}

__device__ inline Geo reg_geo(const jb_matrix_desc &d, const RGeo &r) {
    Geo g = make_geo(d.m, d.n, d.rank, d.flags);
    g.np = r.npb;  // physical width (extra full-basis columns follow it)
    g.ncp = r.ncp;
    g.ldw = r.ldw;
    g.ldv = r.ldv;
    return g;
}

__device__ inline bool next_ticket(int *counter, int &s_idx, int64_t &idx) {
    if (threadIdx.x == 0) s_idx = atomicAdd(counter, 1);
    __syncthreads();
    idx = s_idx;
    __syncthreads();
    return true;
}

// C (M x N) = alpha * A (M x K) * B (K x N), column-major, in shared memory;
// M and N multiples of 4.  Each thread owns a 4 x 4 tile of C: rows
// i0, i0 + M/4, i0 + 2M/4, i0 + 3M/4 (consecutive lanes take consecutive i0,
// so every A load and C store of a warp is one contiguous run of shared
// memory, free of bank conflicts) and columns j0 .. j0 + 3 (B loads
// broadcast across the lanes of one j0).
template <typename TA, typename TC = double, typename TB = double>
__device__ void gemm_nn(TC *C, int ldc, const TA *A, int lda, const TB *B, int ldb, int M, int N, int K,
                        TC alpha) {
    const int tm = M >> 2, tn = N >> 2;
    for (int t = threadIdx.x; t < tm * tn; t += blockDim.x) {
        const int i0 = t % tm, j0 = (t / tm) << 2;
        TC acc[4][4];
#pragma unroll
        for (int r = 0; r < 4; ++r)
#pragma unroll
            for (int c = 0; c < 4; ++c) acc[r][c] = TC(0);
        for (int k = 0; k < K; ++k) {
            TC a[4], b[4];
#pragma unroll
            for (int r = 0; r < 4; ++r) a[r] = (TC)A[(size_t)k * lda + i0 + r * tm];
#pragma unroll
            for (int c = 0; c < 4; ++c) b[c] = (TC)B[(size_t)(j0 + c) * ldb + k];
#pragma unroll
            for (int r = 0; r < 4; ++r)
#pragma unroll
                for (int c = 0; c < 4; ++c) acc[r][c] = dfma(a[r], b[c], acc[r][c]);
        }
#pragma unroll
        for (int r = 0; r < 4; ++r)
#pragma unroll
            for (int c = 0; c < 4; ++c) C[(size_t)(j0 + c) * ldc + i0 + r * tm] = alpha * acc[r][c];
    }
}

// T (ld) = transpose of S (ld), n x n, column-major in shared memory.  The
// 32 lanes of a warp take one diagonal of a 32 x 32 block (row i = lane,
// column (lane + s) mod 32), so both the read of S and the write of T hit 32
// different banks instead of one (a column-major stride of ld words).
__device__ inline void transpose_sq(double *T, const double *S, int n, int ld) {
    const int nbk = (n + 31) >> 5;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int job = warp; job < nbk * nbk * 32; job += nw) {
        const int s = job & 31, blk = job >> 5;
        const int i = ((blk % nbk) << 5) + lane, c = ((blk / nbk) << 5) + ((lane + s) & 31);
        if (i < n && c < n) T[(size_t)i * ld + c] = S[(size_t)c * ld + i];
    }
}

// V <- V (3I - V^T V) / 2 (Newton-Schulz step towards the orthogonal polar
// factor of V), n x n with ld; VT, H, Vn: n x n scratch (ld).  Returns
// max |V^T V - I| before the step.
__device__ double polar_step(double *V, int n, int ld, double *VT, double *H, double *Vn, Aux &ax) {
    transpose_sq(VT, V, n, ld);
    __syncthreads();
    gemm_nn<double>(H, ld, VT, ld, V, ld, n, n, n, 1.0);
    __syncthreads();
    double err = 0.0;
    for (int k = threadIdx.x; k < n * n; k += blockDim.x) {
        const int c = k / n, i = k - c * n;
        const double g = H[(size_t)c * ld + i];
        const double e = g - (i == c ? 1.0 : 0.0);
        err = fmax(err, fabs(e));
        H[(size_t)c * ld + i] = (i == c ? 1.0 : 0.0) - 0.5 * e;  // (3I - G) / 2
    }
    err = block_max(err, ax.red);
    gemm_nn<double>(Vn, ld, V, ld, H, ld, n, n, n, 1.0);
    __syncthreads();
    for (int k = threadIdx.x; k < n * n; k += blockDim.x) {
        const int c = k / n, i = k - c * n;
        V[(size_t)c * ld + i] = Vn[(size_t)c * ld + i];
    }
    __syncthreads();
    return err;
}

// Hand-off word from the FP32 to the FP64 launch of the mixed register path:
// bit 30 set, the input's scale exponent e + 1024 in bits 12..22, the FP32
// sweeps in bits 0..11.  A sweep count or exponent out of that range is
// passed as the plain sweep count, and the FP64 launch then scans the input.
__device__ __forceinline__ int pack_handoff(int ns, int e) {
    return (ns >= 0 && ns < 4096 && e > -1024 && e < 1024) ? (1 << 30) | ((e + 1024) << 12) | ns : ns;
}
__device__ __forceinline__ bool unpack_handoff(int w, int &ns, int &e) {
    if (!(w & (1 << 30))) { ns = w; return false; }
    ns = w & 0xfff;
    e = ((w >> 12) & 0x7ff) - 1024;
    return true;
}

// K1: FP32 sweeps.  MIXED: store the FP32 V (nt x nt) in the scratch for K2;
// else run the epilogue and write U, S, Vh.  THREADS / MR / MRV: the CTA size
// and the register tile (rows per lane of W and V); rb32_kernel is the
// 256-thread form for matrices up to 128 x 64, rb32_large_kernel the
// 512-thread form for one matrix up to 256 x 128 per CTA.
template <bool MIXED, int THREADS, int BW, int MR, int MRV>
__global__ void __launch_bounds__(THREADS, (BW == kB32 && MR <= kMaxR) ? 512 / THREADS : 1) rb32_kernel_t(Params p) {
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ int s_idx;
    Aux ax = carve_aux(smem, p.maxd);
    unsigned char *region = smem + aux_bytes(p.maxd);
    float *xbuf = p.xchg ? (float *)(region + p.xchg_off) : nullptr;   // tile exchange area
    for (;;) {
        int64_t idx;
        next_ticket(p.counter, s_idx, idx);
        if (idx >= p.count) break;
        const int64_t mat = p.order ? (int64_t)p.order[idx] : idx;
        const jb_matrix_desc d = desc_of(p, mat);
        if (!class_takes(d, p.cls)) continue;  // the other size class's launch solves it
        if (threadIdx.x < 4) ax.flag[threadIdx.x] = 0;
        __syncthreads();
        int ns = 0, st = JB_ST_OK, e_in = 0;
        if (!rdesc_fits(d, BW, 4, p, MIXED, MR, MRV)) {
            st = JB_ST_BAD_DESC;
        } else {
            const RGeo r = rgeo(d.m > d.n ? d.m : d.n, d.m > d.n ? d.n : d.m, BW, d.flags);
            const Geo g = reg_geo(d, r);
            const float *A = (const float *)p.A + d.a_off;
            float *W = (float *)region;
            float *V = (float *)(region + align16((size_t)r.ldw * r.ncp * 4));
            bool bad;
            const int e = scan_input(A, g.m * g.n, ax, bad);
            e_in = e;
            if (bad) {
                st = JB_ST_NONFINITE_IN;
            } else {
                zero_fill(W, (size_t)r.ldw * r.ncp);
                zero_fill(V, (size_t)r.ldv * r.npb);
                __syncthreads();
                if (!p.vstart) {
                    load_padded(A, g, r, e, W, V);
                } else {
                    // Warm start: V = given start (identity on the padding),
                    // W = A_t V with A_t staged after the work area.
                    float *As = (float *)(region + rregion_bytes(r, 4));
                    const int nt = g.nt;
                    zero_fill(As, (size_t)r.ldw * nt);
                    __syncthreads();
                    load_stage(A, g, r.ldw, As);
                    const float *vs = p.vstart + d.x_off;
                    for (int k = threadIdx.x; k < nt * nt; k += blockDim.x) {
                        const int c = k / nt, i = k - c * nt;
                        V[(size_t)c * r.ldv + i] = vs[k];
                    }
                    for (int j = nt + threadIdx.x; j < r.npb; j += blockDim.x) V[(size_t)j * r.ldv + j] = 1.0f;
                    __syncthreads();
                    gemm_nn<float, float, float>(W, r.ldw, As, r.ldw, V, r.ldv, r.ldw, r.npb, nt, ldexpf(1.0f, -e));
                }
                __syncthreads();
                const float tol = MIXED ? (p.tol32 > 0 ? (float)p.tol32 : 10.0f * Lim<float>::eps())
                                        : (p.tol > 0 ? (float)p.tol : 10.0f * Lim<float>::eps());
                bool conv;
                // MIXED: the FP32 sweeps only precondition the FP64 phase, which
                // decides convergence on exact dot products; they update the
                // column norms instead of recomputing them (rb_sweeps UPD).  Not
                // in the large tile, where the norms would not fit in registers.
                const float exit_ratio =
                    MIXED ? (p.exit_ratio == 0.f ? kMixedExitRatio : fmaxf(p.exit_ratio, 0.f)) : 0.0f;
                ns = rb_dispatch<float, BW, MR, MRV, (MIXED && MR <= kMaxR) ? 1 : 0>(
                    r, W, V, tol, MIXED ? p.max_sweeps32 : p.max_sweeps, true, ax.red, conv, exit_ratio, ax.sig,
                    xbuf);
                if (MIXED) {
                    float *x = p.x32 + d.x_off;
                    const int nt = g.nt;
                    for (int k = threadIdx.x; k < nt * nt; k += blockDim.x) {
                        const int c = k / nt, i = k - c * nt;
                        x[k] = V[(size_t)c * r.ldv + i];
                    }
                } else if (!conv) {
                    st = JB_ST_NOT_CONVERGED;
                } else {
                    float *U = p.U ? (float *)p.U + d.u_off : nullptr;
                    float *Vh = p.Vh ? (float *)p.Vh + d.v_off : nullptr;
                    st = epilogue<float, float>(W, V, g, e, U, (float *)p.S + d.s_off, Vh, ax);
                }
            }
        }
        if (threadIdx.x == 0) {
            if (p.status) p.status[mat] = st;
            // Mixed, register tiles: the FP64 phase (rb64_kernel) takes over a
            // matrix this launch solved; the sweeps word then also carries the
            // input's scale exponent, so that rb64 need not scan the input again.
            if (p.sweeps)
                p.sweeps[mat] = (MIXED && MR <= kMaxR && st == JB_ST_OK) ? pack_handoff(ns, e_in) : ns;
        }
        __syncthreads();
    }
}


// K2: FP64 sweeps.  MIXED (TI = float): start from the FP32 V of K1, made
// orthogonal by Newton-Schulz polar steps to well below the FP32 rounding of
// the outputs (it is orthogonal to ~1e-5 already), with W = A V recomputed
// in FP64 from the exact input;
// native (TI = double): start from V = I.  Runs the epilogue and writes U,
// S, Vh in TI.
template <typename TI, bool MIXED, int THREADS = kT64>
__global__ void __launch_bounds__(THREADS, kT64 / THREADS) rb64_kernel(Params p) {
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ int s_idx;
    Aux ax = carve_aux(smem, p.maxd);
    unsigned char *region = smem + aux_bytes(p.maxd);
    for (;;) {
        int64_t idx;
        next_ticket(MIXED ? p.counter2 : p.counter, s_idx, idx);
        if (idx >= p.count) break;
        const int64_t mat = p.order ? (int64_t)p.order[idx] : idx;
        const jb_matrix_desc d = desc_of(p, mat);
        if (!class_takes(d, p.cls)) continue;  // the other size class's launch solves it
        if (threadIdx.x < 4) ax.flag[threadIdx.x] = 0;
        __syncthreads();
        int prev = JB_ST_OK, s1 = 0, e_k1 = 0;
        bool have_e = false;
        if (MIXED && threadIdx.x == 0) { ax.flag[3] = p.status[mat]; ax.flag[2] = p.sweeps[mat]; }
        __syncthreads();
        if (MIXED) { prev = ax.flag[3]; have_e = unpack_handoff(ax.flag[2], s1, e_k1); }
        __syncthreads();
        if (threadIdx.x == 0) ax.flag[2] = 0;
        __syncthreads();
        if (prev != JB_ST_OK) continue;  // K1 already reported this matrix
        int ns = s1, st = JB_ST_OK;
        if (!rdesc_fits(d, kB64, 8, p, MIXED)) {
            st = JB_ST_BAD_DESC;
        } else {
            const int mt = d.m > d.n ? d.m : d.n, nt = d.m > d.n ? d.n : d.m;
            const RGeo r = rgeo(mt, nt, kB64, d.flags);
            const Geo g = reg_geo(d, r);
            const TI *A = (const TI *)p.A + d.a_off;
            double *W = (double *)region;
            double *V = (double *)(region + align16((size_t)r.ldw * r.ncp * 8));
            bool bad = false;
            // the FP32 launch already checked the input and found its scale
            const int e = have_e ? e_k1 : scan_input(A, g.m * g.n, ax, bad);
            if (bad) {
                st = JB_ST_NONFINITE_IN;
            } else {
                zero_fill(V, (size_t)r.ldv * r.npb);
                if (!MIXED) zero_fill(W, (size_t)r.ldw * r.ncp);
                __syncthreads();
                if (!MIXED) {
                    load_padded(A, g, r, e, W, V);
                } else {
                    double *X1 = (double *)(region + rregion_bytes(r, 8));
                    unsigned char *X2 = region + rregion_bytes(r, 8) + align16((size_t)r.ldv * r.npb * 8);
                    const float *x = p.x32 + d.x_off;
                    for (int k = threadIdx.x; k < nt * nt; k += blockDim.x) {
                        const int c = k / nt, i = k - c * nt;
                        V[(size_t)c * r.ldv + i] = (double)x[k];
                    }
                    for (int j = nt + threadIdx.x; j < r.npb; j += blockDim.x) V[(size_t)j * r.ldv + j] = 1.0;
                    __syncthreads();
                    double err = polar_step(V, r.npb, r.ldv, W, X1, (double *)X2, ax);
                    // One step leaves |V^T V - I| ~ 0.75 err^2: <= 7.5e-9 from err <= 1e-4,
                    // below the FP32 rounding of the outputs; a second step beyond that.
                    if (err > 1e-4 && err < 0.5) err = polar_step(V, r.npb, r.ldv, W, X1, (double *)X2, ax);
                    if (err >= 0.5) {  // not near-orthogonal: restart from V = I
                        for (int k = threadIdx.x; k < r.npb * r.ldv; k += blockDim.x) {
                            const int c = k / r.ldv, i = k - c * r.ldv;
                            V[k] = (i == c) ? 1.0 : 0.0;
                        }
                    }
                    // A_t (float, ldw x nt, zero rows >= mt) staged in X2.
                    float *As = (float *)X2;
                    zero_fill(As, (size_t)r.ldw * nt);
                    __syncthreads();
                    load_stage(A, g, r.ldw, As);
                    __syncthreads();
                    gemm_nn<float>(W, r.ldw, As, r.ldw, V, r.ldv, r.ldw, r.npb, nt, ldexp(1.0, -e));
                    for (int j = r.npb; j < r.ncp; ++j)
                        for (int i = threadIdx.x; i < r.ldw; i += blockDim.x) W[(size_t)j * r.ldw + i] = 0.0;
                }
                __syncthreads();
                const double tol = MIXED ? (p.tol > 0 ? (double)(float)p.tol : (double)(10.0f * Lim<float>::eps()))
                                         : (p.tol > 0 ? p.tol : 10.0 * Lim<double>::eps());
                bool conv;
                // MIXED: norm updates carried through ax.sig (rb_sweeps UPD 2); the
                // confirming Gram pass that ends the solve measures exact norms.
                ns += rb_dispatch<double, kB64, kMaxR, kMaxRV, MIXED ? 2 : 0>(r, W, V, tol, p.max_sweeps, true, ax.red,
                                                                          conv, 0.0, ax.sig);
                if (!conv) {
                    st = JB_ST_NOT_CONVERGED;
                } else {
                    TI *U = p.U ? (TI *)p.U + d.u_off : nullptr;
                    TI *Vh = p.Vh ? (TI *)p.Vh + d.v_off : nullptr;
                    st = epilogue<double, TI>(W, V, g, e, U, (TI *)p.S + d.s_off, Vh, ax);
                }
            }
        }
        if (threadIdx.x == 0) {
            if (p.status) p.status[mat] = st;
            if (p.sweeps) p.sweeps[mat] = ns;
        }
        __syncthreads();
    }
}


// K2 of the mixed solve for large tiles (after rb32_kernel_t<true, kT32L>):
// the FP64 phase on the Gram of W (jb_gram64.cuh).  Work arrays in the
// per-CTA global area: V64 (ldv x np) | W64 (ldw x ncp) | X, Ad (ldx x ncp
// each, ldx = max(ldw, ldv): they also hold the temporaries), FP64; G, D and
// the round bookkeeping in shared memory.
__host__ __device__ inline size_t gram64_region(const Dims &d) {
    const size_t ldx = d.ldw > d.ldv ? d.ldw : d.ldv;
    return align16((size_t)d.ldv * d.np * 8) + align16((size_t)d.ldw * d.ncp * 8) + 2 * align16(ldx * d.ncp * 8);
}

__global__ void __launch_bounds__(kTG, 1) gram64_kernel(Params p) {
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ int s_idx, s_any;
    Aux ax = carve_aux(smem, p.maxd);
    const int npmax = p.maxd.np;
    size_t gsz, dd;
    gram64_regions(npmax, p.maxd.mt, gsz, dd);
    double *G = (double *)(smem + aux_bytes(p.maxd));
    float *D = (float *)((unsigned char *)G + gsz);
    double *cs = (double *)((unsigned char *)D + dd);
    unsigned char *pq = (unsigned char *)(cs + npmax);
    unsigned char *sched = pq + npmax;
    unsigned char *area = p.gws + (size_t)blockIdx.x * p.gws_stride;
    for (;;) {
        int64_t idx;
        next_ticket(p.counter, s_idx, idx);
        if (idx >= p.count) break;
        const int64_t mat = p.order ? (int64_t)p.order[idx] : idx;
        const jb_matrix_desc d = desc_of(p, mat);
        if (threadIdx.x < 4) ax.flag[threadIdx.x] = 0;
        __syncthreads();
        if (threadIdx.x == 0) { ax.flag[3] = p.status[mat]; ax.flag[2] = p.sweeps[mat]; }
        __syncthreads();
        const int prev = ax.flag[3], s1 = ax.flag[2];
        __syncthreads();
        if (threadIdx.x == 0) ax.flag[2] = 0;
        __syncthreads();
        if (prev != JB_ST_OK) continue;  // K1 already reported this matrix
        int ns = s1, st = JB_ST_OK;
        if (!desc_fits(d, p.maxd) || d.x_off < 0) {
            st = JB_ST_BAD_DESC;
        } else {
            const Geo g = make_geo(d.m, d.n, d.rank, d.flags);
            const float *A = (const float *)p.A + d.a_off;
            const int np = g.np, nt = g.nt, mt = g.mt, ldv = g.ldv, ldw = g.ldw;
            const int ldx = ldw > ldv ? ldw : ldv;
            double *V64 = (double *)area;
            double *W64 = (double *)((unsigned char *)V64 + align16((size_t)ldv * np * 8));
            double *X = (double *)((unsigned char *)W64 + align16((size_t)ldw * g.ncp * 8));
            double *Ad = (double *)((unsigned char *)X + align16((size_t)ldx * g.ncp * 8));
            bool bad;
            const int e = scan_input(A, g.m * g.n, ax, bad);
            if (bad) {
                st = JB_ST_NONFINITE_IN;
            } else {
                // V from the FP32 phase (nt x nt, column-major), identity on the padding
                const float *x = p.x32 + d.x_off;
                for (int k = threadIdx.x; k < ldv * np; k += blockDim.x) {
                    const int c = k / ldv, i = k - c * ldv;
                    V64[k] = (c < nt && i < nt) ? (double)x[(size_t)c * nt + i] : ((i == c && i < np) ? 1.0 : 0.0);
                }
                __syncthreads();
                double *stage = (double *)D;
                // Newton-Schulz: X = V^T V, V <- 1.5 V - 0.5 V X (once; twice if V was far from
                // orthogonal); the product V X is staged in Ad (ldx x ncp), free until A_t goes there
                for (int it = 0; it < 2; ++it) {
                    gemm64<true, double>(V64, ldv, V64, ldv, X, ldx, np, np, np, 1.0, 0.0, stage);
                    double dev = 0.0;
                    for (int k = threadIdx.x; k < np * np; k += blockDim.x) {
                        const int c = k / np, i = k - c * np;
                        dev = fmax(dev, fabs(X[(size_t)c * ldx + i] - (i == c ? 1.0 : 0.0)));
                    }
                    dev = block_max(dev, ax.red);
                    if (it == 1 && dev < 1e-10) break;
                    gemm64<false, double>(V64, ldv, X, ldx, Ad, ldx, np, np, np, -0.5, 0.0, stage);
                    for (int k = threadIdx.x; k < np * np; k += blockDim.x) {
                        const int c = k / np, i = k - c * np;
                        V64[(size_t)c * ldv + i] = fma(1.5, V64[(size_t)c * ldv + i], Ad[(size_t)c * ldx + i]);
                    }
                    __syncthreads();
                    if (dev < 1e-5) break;   // one step took it to ~dev^2
                }
                // A_t, scaled by 2^-e (exact), zero padding column (ld ldx)
                for (int k = threadIdx.x; k < ldx * np; k += blockDim.x) {
                    const int c = k / ldx, i = k - c * ldx;
                    double a = 0.0;
                    if (c < nt && i < mt) a = ldexp((double)(g.wide ? A[(size_t)c * g.n + i] : A[(size_t)i * g.n + c]), -e);
                    Ad[k] = a;
                }
                __syncthreads();
                // W = A_t V (FP64); extra full-basis columns zero
                gemm64<false, double>(Ad, ldx, V64, ldv, W64, ldw, mt, np, np, 1.0, 0.0, stage);
                for (int k = threadIdx.x; k < ldw * (g.ncp - np); k += blockDim.x) W64[(size_t)np * ldw + k] = 0.0;
                // G = W^T W in shared memory
                gemm64<true, double>(W64, ldw, W64, ldw, G, np, np, np, mt, 1.0, 0.0, stage);
                const double tol = p.tol > 0 ? (double)(float)p.tol : (double)(10.0f * Lim<float>::eps());
                const int s2 = gram_sweeps(G, D, np, tol, p.max_sweeps, sched, pq, cs, &s_any);
                if (s2 > p.max_sweeps) {
                    ns += p.max_sweeps;
                    st = JB_ST_NOT_CONVERGED;
                } else {
                    ns += s2;
                    // W <- W + W D, V <- V + V D (staging in G, no longer needed)
                    stage = G;
                    gemm64<false, float>(W64, ldw, D, np, Ad, ldx, mt, np, np, 1.0, 0.0, stage);
                    for (int k = threadIdx.x; k < mt * np; k += blockDim.x) {
                        const int c = k / mt, i = k - c * mt;
                        W64[(size_t)c * ldw + i] += Ad[(size_t)c * ldx + i];
                    }
                    gemm64<false, float>(V64, ldv, D, np, X, ldx, np, np, np, 1.0, 0.0, stage);
                    for (int k = threadIdx.x; k < np * np; k += blockDim.x) {
                        const int c = k / np, i = k - c * np;
                        V64[(size_t)c * ldv + i] += X[(size_t)c * ldx + i];
                    }
                    __syncthreads();
                    float *U = p.U ? (float *)p.U + d.u_off : nullptr;
                    float *Vh = p.Vh ? (float *)p.Vh + d.v_off : nullptr;
                    st = epilogue<double, float>(W64, V64, g, e, U, (float *)p.S + d.s_off, Vh, ax);
                }
            }
        }
        if (threadIdx.x == 0) {
            if (p.status) p.status[mat] = st;
            if (p.sweeps) p.sweeps[mat] = ns;
        }
        __syncthreads();
    }
}


// ---------------------------------------------------------------------------
// Warm start preparation (one CTA per matrix): V0 (the network's guess,
// row-major n x n, columns = start vectors) -> Householder QR, column signs
// kept (householder_orthonormalize) -> Q.  The start is kept when it lowers
// the Gram off-norm ||offdiag(W^T W)||_F / ||W^T W||_F of W = A Q below that
// of A itself; otherwise the start is the identity (the plain solver).
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) warm_prep_kernel(const float *A, const float *V0, float *Vs, int32_t *used,
                                                        float *off0, float *off1, int64_t batch, int m, int n) {
    extern __shared__ __align__(16) unsigned char smem[];
    const int ldm = (m + 3) & ~3;
    float *Arow = (float *)smem;                                   // m x n row-major
    float *Acol = Arow + (size_t)m * n;                            // ldm x n column-major
    double *G = (double *)(smem + align16(((size_t)m * n + (size_t)ldm * n) * 4));  // n x n
    double *Q = G + (size_t)n * n;
    double *T = Q + (size_t)n * n;
    Aux ax;
    ax.red = T + (size_t)n * n;
    ax.tau = ax.red + 64;
    ax.sig = ax.tau + n;
    for (int64_t z = blockIdx.x; z < batch; z += gridDim.x) {
        const float *a = A + z * (int64_t)m * n;
        for (int k = threadIdx.x; k < ldm * n; k += blockDim.x) Acol[k] = 0.f;
        __syncthreads();
        for (int k = threadIdx.x; k < m * n; k += blockDim.x) {
            const int i = k / n, j = k - i * n;
            const float x = a[k];
            Arow[k] = x;
            Acol[(size_t)j * ldm + i] = x;
        }
        __syncthreads();
        // G = A^T A (A^T column-major is A row-major).
        gemm_nn<float, double, float>(G, n, Arow, n, Acol, ldm, n, n, m, 1.0);
        __syncthreads();
        double on = 0.0, dg = 0.0;
        for (int k = threadIdx.x; k < n * n; k += blockDim.x) {
            const int c = k / n, i = k - c * n;
            const double g2 = G[k] * G[k];
            if (i == c) dg += g2; else on += g2;
        }
        const double off_a = sqrt(block_sum(on, ax.red) / fmax(block_sum(on + dg, ax.red), 1e-300));
        const float *v0 = V0 + z * (int64_t)n * n;
        for (int k = threadIdx.x; k < n * n; k += blockDim.x) {
            const int i = k / n, j = k - i * n;
            Q[(size_t)j * n + i] = (double)v0[k];
        }
        __syncthreads();
        householder_orthonormalize(Q, n, n, T, n, ax);
        // G1 = Q^T (G Q): T = G Q, then G1_ij = q_i . T_j.
        gemm_nn<double, double, double>(T, n, G, n, Q, n, n, n, n, 1.0);
        __syncthreads();
        on = 0.0;
        dg = 0.0;
        for (int k = threadIdx.x; k < n * n; k += blockDim.x) {
            const int j = k / n, i = k - j * n;
            double acc = 0.0;
            for (int t = 0; t < n; ++t) acc = fma(Q[(size_t)i * n + t], T[(size_t)j * n + t], acc);
            if (i == j) dg += acc * acc; else on += acc * acc;
        }
        const double off_q = sqrt(block_sum(on, ax.red) / fmax(block_sum(on + dg, ax.red), 1e-300));
        const bool keep = off_q < off_a;
        float *vs = Vs + z * (int64_t)n * n;
        for (int k = threadIdx.x; k < n * n; k += blockDim.x) {
            const int c = k / n, i = k - c * n;
            vs[k] = keep ? (float)Q[(size_t)c * n + i] : (i == c ? 1.f : 0.f);
        }
        if (threadIdx.x == 0) {
            if (used) used[z] = keep;
            if (off0) off0[z] = (float)off_a;
            if (off1) off1[z] = (float)off_q;
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// Host side.
// ---------------------------------------------------------------------------
constexpr size_t kSmemLimit = 227 * 1024;
constexpr size_t kCounterBytes = 256;

struct DevInfo {
    int sms = 0;
    bool init = false;
};
static DevInfo g_dev[64];

static int sm_count() {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return -1;
    if (!g_dev[dev].init) {
        int sms = 0;
        if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return -1;
        g_dev[dev].sms = sms;
        g_dev[dev].init = true;
    }
    return g_dev[dev].sms;
}

// Launch plan for one batch (sized by its largest tall shape).
struct Plan {
    int bw;               // block width of the FP32 register kernel (4 or 8)
    bool reg;             // register-tile path
    bool big;             // large-tile FP32 kernel (+ round-robin FP64 phase when mixed)
    size_t gram_stride;   // big + mixed: per-CTA area of the Gram FP64 kernel (0: round-robin FP64 phase)
    size_t gram_smem;
    // round-robin path
    Dims d;
    size_t aux, region, smem;
    bool global_region;
    int threads;
    // register path: one sizing per kernel
    Dims d32, d64;
    size_t smem32, smem64, reg32, reg64;
    // size-class split (kNarrowN): a second launch per phase for narrow matrices
    bool split;
    Dims d64n, d32n;
    size_t smem64n, reg64n, smem32n, reg32n;
    // FP32 tile exchange areas: offsets in the work area and size
    size_t xoff32, xoff32n, xbytes32;
};

static Plan make_plan(int max_mt, int max_nt, int elem, int precision, int flags) {
    Plan pl;
    memset(&pl, 0, sizeof(pl));
    pl.bw = (flags & JB_BLOCK_WIDTH_8) ? 8 : kB32;
    pl.d = dims_of(max_mt, max_nt, flags);
    pl.aux = aux_bytes(pl.d);
    pl.region = region_bytes(pl.d, elem, precision);
    pl.global_region = pl.aux + pl.region > kSmemLimit;
    pl.smem = pl.global_region ? pl.aux : pl.aux + pl.region;
    int t = (pl.d.np / 2) * 8;
    t = (t + 31) / 32 * 32;
    if (t < 64) t = 64;
    if (t > 1024) t = 1024;
    pl.threads = t;
    const RGeo r32 = rgeo(max_mt, max_nt, pl.bw, flags), r64 = rgeo(max_mt, max_nt, kB64, flags);
    pl.reg = !(flags & JB_ROUND_ROBIN) && r32.R <= kMaxR && r32.RV <= kMaxRV && r64.RV <= kMaxRV;
    if (pl.reg) {
        pl.d32 = raux_dims(r32);
        pl.d64 = raux_dims(r64);
        pl.reg32 = rregion_bytes(r32, 4);
        pl.reg64 = (elem == 4 && precision == JB_PREC_MIXED) ? rregion_mixed64(r64, max_nt) : rregion_bytes(r64, 8);
        // FP32 kernels: work area, then the tile exchange area (tile_x)
        pl.xoff32 = pl.reg32;
        pl.xbytes32 = xchg_bytes(r32.npb, kMaxR, kMaxRV);
        pl.smem32 = aux_bytes(pl.d32) + pl.reg32 + pl.xbytes32;
        pl.smem64 = aux_bytes(pl.d64) + pl.reg64;
        if (pl.smem64 > kSmemLimit || pl.smem32 > kSmemLimit) pl.reg = false;
        pl.split = pl.reg && pl.bw == kB32 && max_nt > kNarrowN && !(flags & JB_ONE_SIZE_CLASS);
        if (pl.split) {
            const RGeo r32n = rgeo(max_mt, kNarrowN, kB32, flags);
            pl.d32n = raux_dims(r32n);
            pl.reg32n = rregion_bytes(r32n, 4);
            pl.xoff32n = pl.reg32n;
            pl.smem32n = aux_bytes(pl.d32n) + pl.reg32n + xchg_bytes(r32n.npb, kMaxR, kMaxRV);
            const RGeo r64n = rgeo(max_mt, kNarrowN, kB64, flags);
            pl.d64n = raux_dims(r64n);
            pl.reg64n = (elem == 4 && precision == JB_PREC_MIXED) ? rregion_mixed64(r64n, kNarrowN)
                                                                   : rregion_bytes(r64n, 8);
            pl.smem64n = aux_bytes(pl.d64n) + pl.reg64n;
        }
    }
    const RGeo r32l = rgeo(max_mt, max_nt, kB32L, flags);
    if (!pl.reg && elem == 4 && !(flags & JB_ROUND_ROBIN) && r32l.R <= kMaxRL && r32l.RV <= kMaxRVL &&
        r32l.nb / 2 <= kT32L / 32) {
        pl.d32 = raux_dims(r32l);
        pl.reg32 = rregion_bytes(r32l, 4);
        pl.smem32 = aux_bytes(pl.d32) + pl.reg32;
        pl.big = pl.smem32 <= kSmemLimit;
        if (pl.big && precision == JB_PREC_MIXED) {
            pl.gram_smem = aux_bytes(pl.d) + gram64_smem(pl.d.np, pl.d.mt);
            if (pl.gram_smem <= kSmemLimit && pl.d.np <= 256) pl.gram_stride = gram64_region(pl.d) + 256;
        }
    }
    return pl;
}

// Bytes before the mixed-precision scratch: ticket counters and, on the
// round-robin path, per-CTA global work areas.
static size_t base_bytes(const Plan &pl, int64_t count) {
    size_t bytes = kCounterBytes;
    if (pl.gram_stride) {
        const int sms = sm_count();
        int64_t grid = sms > 0 ? sms : 148;
        if (grid > count) grid = count;
        bytes += (size_t)grid * pl.gram_stride;
    } else if (!pl.reg && pl.global_region) {
        const int sms = sm_count();
        int64_t grid = sms > 0 ? sms : 148;
        if (grid > count) grid = count;
        bytes += (size_t)grid * (align16(pl.region) + 256);
    }
    return bytes;
}

template <typename K>
static int occupancy_grid(K kern, int threads, size_t smem, int64_t count, int64_t &grid) {
    const int sms = sm_count();
    if (sms <= 0) return JB_ECUDA;
    if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
        return JB_ECUDA;
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, threads, smem) != cudaSuccess)
        return JB_ECUDA;
    if (per_sm < 1) return JB_ETOOBIG;
    grid = (int64_t)sms * per_sm;
    if (grid > count) grid = count;
    if (grid < 1) grid = 1;
    return JB_OK;
}

template <typename T, int PREC>
static int launch_rr(Params &p, const Plan &pl, unsigned char *ws, size_t ws_bytes, cudaStream_t st) {
    auto kern = batched_kernel<T, PREC>;
    int64_t grid;
    int rc = occupancy_grid(kern, pl.threads, pl.smem, p.count, grid);
    if (rc) return rc;
    p.maxd = pl.d;
    p.counter = (int *)ws;
    p.gws = nullptr;
    p.gws_stride = 0;
    if (pl.global_region) {
        const size_t stride = align16(pl.region) + 256;
        if (ws_bytes < kCounterBytes + stride) return JB_EWORKSPACE;
        // With an FP32-phase V hand-off (x32) in the same workspace, the
        // per-CTA areas may use only the span base_bytes reserved before it.
        const size_t span = p.x32 ? base_bytes(pl, p.count) - kCounterBytes : ws_bytes - kCounterBytes;
        const int64_t max_grid = (int64_t)(span / stride);
        if (max_grid < 1) return JB_EWORKSPACE;
        if (grid > max_grid) grid = max_grid;
        p.gws = ws + kCounterBytes;
        p.gws_stride = stride;
    }
    if (cudaMemsetAsync(p.counter, 0, sizeof(int), st) != cudaSuccess) return JB_ECUDA;
    kern<<<(unsigned)grid, pl.threads, pl.smem, st>>>(p);
    return cudaGetLastError() == cudaSuccess ? JB_OK : JB_ECUDA;
}

static int launch_gram(Params &p, const Plan &pl, unsigned char *ws, size_t ws_bytes, cudaStream_t st);

// elem: 4 (f32 input) or 8 (f64 input).
static int launch_reg(Params &p, const Plan &pl, int elem, int precision, unsigned char *ws, size_t ws_bytes,
                      cudaStream_t st) {
    p.counter = (int *)ws;
    p.counter2 = (int *)ws + 1;
    const bool mixed = elem == 4 && precision == JB_PREC_MIXED;
    if (mixed) {
        const size_t base = base_bytes(pl, p.count);
        if (ws_bytes < base) return JB_EWORKSPACE;
        p.x32 = (float *)(ws + base);
        p.x_cap = (int64_t)((ws_bytes - base) / 4);
    }
    // Shapes are known on the host only for a uniform batch, whose matrices
    // share one class: the split applies to descriptor (uneven) batches.
    const bool split = pl.split && p.descs != nullptr;
    if (cudaMemsetAsync(ws, 0, 4 * sizeof(int), st) != cudaSuccess) return JB_ECUDA;
    int64_t grid;
    int rc;
    if (elem == 4) {
        // block width 4: 8 warps of 256 threads for 64 columns; 8: 4 warps of 128
        auto k1 = pl.bw == 8 ? (mixed ? rb32_kernel_t<true, 128, 8, kMaxR, kMaxRV>
                                      : rb32_kernel_t<false, 128, 8, kMaxR, kMaxRV>)
                             : (mixed ? rb32_kernel_t<true, kT32, kB32, kMaxR, kMaxRV>
                                      : rb32_kernel_t<false, kT32, kB32, kMaxR, kMaxRV>);
        const int t1 = pl.bw == 8 ? 128 : kT32;
        if ((rc = occupancy_grid(k1, t1, pl.smem32, p.count, grid))) return rc;
        p.maxd = pl.d32;
        p.region_cap = pl.reg32;
        p.cls = split ? 1 : 0;
        p.xchg = 1;
        p.xchg_off = pl.xoff32;
        k1<<<(unsigned)grid, t1, pl.smem32, st>>>(p);
        if (cudaGetLastError() != cudaSuccess) return JB_ECUDA;
        if (split) {
            // narrow matrices: 4 warps (nt <= 32 is at most 8 blocks of 4 columns)
            auto k1n = mixed ? rb32_kernel_t<true, kT32 / 2, kB32, kMaxR, kMaxRV>
                             : rb32_kernel_t<false, kT32 / 2, kB32, kMaxR, kMaxRV>;
            if ((rc = occupancy_grid(k1n, kT32 / 2, pl.smem32n, p.count, grid))) return rc;
            p.counter = (int *)ws + 2;
            p.cls = 2;
            p.maxd = pl.d32n;
            p.region_cap = pl.reg32n;
            p.xchg_off = pl.xoff32n;
            k1n<<<(unsigned)grid, kT32 / 2, pl.smem32n, st>>>(p);
            if (cudaGetLastError() != cudaSuccess) return JB_ECUDA;
            p.counter = (int *)ws;
        }
        p.xchg = 0;
        if (!mixed) return JB_OK;
        auto k2 = rb64_kernel<float, true>;
        if ((rc = occupancy_grid(k2, kT64, pl.smem64, p.count, grid))) return rc;
        p.maxd = pl.d64;
        p.region_cap = pl.reg64;
        p.cls = split ? 1 : 0;
        k2<<<(unsigned)grid, kT64, pl.smem64, st>>>(p);
        if (cudaGetLastError() != cudaSuccess) return JB_ECUDA;
        if (split) {
            // narrow matrices: 8 warps (nt <= 32 is at most 16 blocks of 2 columns),
            // work area sized for nt <= kNarrowN
            auto k2n = rb64_kernel<float, true, kT64 / 2>;
            if ((rc = occupancy_grid(k2n, kT64 / 2, pl.smem64n, p.count, grid))) return rc;
            p.maxd = pl.d64n;
            p.region_cap = pl.reg64n;
            p.counter2 = (int *)ws + 3;
            p.cls = 2;
            k2n<<<(unsigned)grid, kT64 / 2, pl.smem64n, st>>>(p);
            if (cudaGetLastError() != cudaSuccess) return JB_ECUDA;
        }
        return JB_OK;
    }
    auto k2 = rb64_kernel<double, false>;
    if ((rc = occupancy_grid(k2, kT64, pl.smem64, p.count, grid))) return rc;
    p.maxd = pl.d64;
    p.region_cap = pl.reg64;
    p.cls = 0;
    k2<<<(unsigned)grid, kT64, pl.smem64, st>>>(p);
    return cudaGetLastError() == cudaSuccess ? JB_OK : JB_ECUDA;
}

// Large tiles (FP32 input): the 512-thread register kernel for the FP32
// sweeps; with mixed precision the round-robin kernel then runs the FP64
// phase from the FP32 V it left in x32.
static int launch_big(Params &p, const Plan &pl, int precision, unsigned char *ws, size_t ws_bytes,
                      cudaStream_t st) {
    const bool mixed = precision == JB_PREC_MIXED;
    p.counter = (int *)ws;
    if (mixed) {
        const size_t base = base_bytes(pl, p.count);
        if (ws_bytes < base) return JB_EWORKSPACE;
        p.x32 = (float *)(ws + base);
        p.x_cap = (int64_t)((ws_bytes - base) / 4);
    }
    if (cudaMemsetAsync(ws, 0, sizeof(int), st) != cudaSuccess) return JB_ECUDA;
    auto k1 = mixed ? rb32_kernel_t<true, kT32L, kB32L, kMaxRL, kMaxRVL>
                    : rb32_kernel_t<false, kT32L, kB32L, kMaxRL, kMaxRVL>;
    int64_t grid;
    int rc;
    if ((rc = occupancy_grid(k1, kT32L, pl.smem32, p.count, grid))) return rc;
    p.maxd = pl.d32;
    p.region_cap = pl.reg32;
    k1<<<(unsigned)grid, kT32L, pl.smem32, st>>>(p);
    if (cudaGetLastError() != cudaSuccess) return JB_ECUDA;
    if (!mixed) return JB_OK;
    if (!pl.gram_stride) {
        p.from_x32 = 1;
        return launch_rr<float, JB_PREC_MIXED>(p, pl, ws, ws_bytes, st);
    }
    return launch_gram(p, pl, ws, ws_bytes, st);
}

// FP64 phase on the Gram of W (gram64_kernel), one CTA per SM, per-CTA
// global areas after the ticket counters.
static int launch_gram(Params &p, const Plan &pl, unsigned char *ws, size_t ws_bytes, cudaStream_t st) {
    if (cudaFuncSetAttribute(gram64_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)pl.gram_smem) !=
        cudaSuccess)
        return JB_ECUDA;
    const int sms = sm_count();
    if (sms <= 0) return JB_ECUDA;
    int64_t g2 = sms < p.count ? sms : p.count;
    const int64_t fit = (int64_t)((ws_bytes - kCounterBytes) / pl.gram_stride);
    if (g2 > fit) g2 = fit;
    if (g2 < 1) return JB_EWORKSPACE;
    p.maxd = pl.d;
    p.gws = ws + kCounterBytes;
    p.gws_stride = pl.gram_stride;
    if (cudaMemsetAsync(p.counter, 0, sizeof(int), st) != cudaSuccess) return JB_ECUDA;
    gram64_kernel<<<(unsigned)g2, kTG, pl.gram_smem, st>>>(p);
    return cudaGetLastError() == cudaSuccess ? JB_OK : JB_ECUDA;
}

static int launch_any(Params &p, const Plan &pl, int elem, int precision, void *workspace, size_t ws_bytes,
                      cudaStream_t st) {
    unsigned char *ws = (unsigned char *)workspace;
    if (!ws || ws_bytes < kCounterBytes) return JB_EWORKSPACE;
    if (pl.reg) return launch_reg(p, pl, elem, precision, ws, ws_bytes, st);
    if (pl.big && elem == 4) return launch_big(p, pl, precision, ws, ws_bytes, st);
    if (elem == 8) return launch_rr<double, JB_PREC_NATIVE>(p, pl, ws, ws_bytes, st);
    return precision == JB_PREC_MIXED ? launch_rr<float, JB_PREC_MIXED>(p, pl, ws, ws_bytes, st)
                                      : launch_rr<float, JB_PREC_NATIVE>(p, pl, ws, ws_bytes, st);
}

static int check_common(int64_t count, int32_t m, int32_t n, int32_t rank, int32_t flags, int32_t max_sweeps) {
    if (count < 0 || m < 1 || n < 1 || max_sweeps < 1) return JB_EINVAL;
    const int k = m < n ? m : n;
    if (rank < 1 || rank > k) return JB_EINVAL;
    if ((flags & JB_FULL_MATRICES) && rank != k) return JB_EINVAL;
    if ((m > n ? m : n) > 8192 || k > 4096) return JB_ETOOBIG;
    return JB_OK;
}

static size_t uniform_workspace(int32_t m, int32_t n, int64_t count, int32_t elem, int32_t precision,
                                int32_t flags) {
    const int mt = m > n ? m : n, nt = m > n ? n : m;
    const int prec = elem == 4 ? precision : JB_PREC_NATIVE;
    const Plan pl = make_plan(mt, nt, elem, prec, flags);
    size_t bytes = base_bytes(pl, count);
    if ((pl.reg || pl.big) && prec == JB_PREC_MIXED) bytes += (size_t)count * nt * nt * 4;
    return bytes;
}


// ---------------------------------------------------------------------------
// Allocation-free variant of jb_svd_batched_f32.
//
// Some callers cannot allocate device memory at the moment they need an SVD:
// plug-ins whose host framework owns every device allocation through its own
// pool (a raw cudaMalloc would bypass its accounting and limits), and
// latency-bound paths that must not call cudaMalloc/cudaFree, which can
// synchronise the whole device.  This entry point takes only inputs and outputs; its scratch
// (the kernels' work tickets and, in mixed precision, the FP32-phase V of
// every matrix) is the fixed array below, which every GPU that loads this
// library holds until the process exits.
// ---------------------------------------------------------------------------
static __device__ __align__(256) unsigned char g_noalloc_scratch[JB_NOALLOC_SCRATCH_BYTES];

static std::mutex g_noalloc_mutex;
static void *g_noalloc_ptr[64];

// Device address of g_noalloc_scratch on the current device.  In host code
// the array's name is only a host-side stand-in, so the address is looked up
// once per device (with that device current) and cached.
static int noalloc_scratch(void **out) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return JB_ECUDA;
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (!g_noalloc_ptr[dev]) {
        void *ptr = nullptr;
        if (cudaGetSymbolAddress(&ptr, g_noalloc_scratch) != cudaSuccess || !ptr) return JB_ECUDA;
        g_noalloc_ptr[dev] = ptr;
    }
    *out = g_noalloc_ptr[dev];
    return JB_OK;
}

}  // namespace jb

using namespace jb;

extern "C" {

int jb_version(void) { return 200; }

int jb_device_sm_count(void) { return sm_count(); }

size_t jb_workspace_bytes(int32_t max_m, int32_t max_n, int64_t count, int32_t elem_bytes, int32_t precision,
                          int32_t flags) {
    if (max_m < 1 || max_n < 1 || count < 0 || (elem_bytes != 4 && elem_bytes != 8)) return 0;
    return uniform_workspace(max_m, max_n, count, elem_bytes, precision, flags);
}

static int batched_common(const void *A, void *U, void *S, void *Vh, int64_t batch, int32_t m, int32_t n,
                          int32_t rank, int32_t flags, double tol, int32_t max_sweeps, int32_t precision,
                          int32_t *sweeps, int32_t *status, void *workspace, size_t workspace_bytes, void *stream,
                          int elem) {
    int rc = check_common(batch, m, n, rank, flags, max_sweeps);
    if (rc) return rc;
    if (!A || !S || (!(flags & JB_VALUES_ONLY) && (!U || !Vh))) return JB_EINVAL;
    if (precision != JB_PREC_NATIVE && precision != JB_PREC_MIXED) return JB_EINVAL;
    if (batch == 0) return JB_OK;
    if (workspace_bytes < uniform_workspace(m, n, batch, elem, precision, flags)) return JB_EWORKSPACE;
    Params p;
    memset(&p, 0, sizeof(p));
    p.A = A;
    p.U = (flags & JB_VALUES_ONLY) ? nullptr : U;
    p.S = S;
    p.Vh = (flags & JB_VALUES_ONLY) ? nullptr : Vh;
    p.count = batch; p.um = m; p.un = n; p.urank = rank; p.uflags = flags & ~JB_ROUND_ROBIN;
    p.tol = tol; p.max_sweeps = max_sweeps; p.tol32 = tol; p.max_sweeps32 = max_sweeps;
    p.sweeps = sweeps; p.status = status;
    const int mt = m > n ? m : n, nt = m > n ? n : m;
    const int prec = elem == 4 ? precision : JB_PREC_NATIVE;
    const Plan pl = make_plan(mt, nt, elem, prec, flags);
    return launch_any(p, pl, elem, prec, workspace, workspace_bytes, (cudaStream_t)stream);
}

int jb_svd_batched_f32(const float *A, float *U, float *S, float *Vh, int64_t batch, int32_t m, int32_t n,
                       int32_t rank, int32_t flags, double tol, int32_t max_sweeps, int32_t precision,
                       int32_t *sweeps, int32_t *status, void *workspace, size_t workspace_bytes, void *stream) {
    return batched_common(A, U, S, Vh, batch, m, n, rank, flags, tol, max_sweeps, precision, sweeps, status,
                          workspace, workspace_bytes, stream, 4);
}

int jb_svd_batched_f64(const double *A, double *U, double *S, double *Vh, int64_t batch, int32_t m, int32_t n,
                       int32_t rank, int32_t flags, double tol, int32_t max_sweeps, int32_t *sweeps,
                       int32_t *status, void *workspace, size_t workspace_bytes, void *stream) {
    return batched_common(A, U, S, Vh, batch, m, n, rank, flags, tol, max_sweeps, JB_PREC_NATIVE, sweeps, status,
                          workspace, workspace_bytes, stream, 8);
}

size_t jb_uneven_workspace_bytes(int32_t max_m, int32_t max_n, int64_t count, int32_t precision, int32_t flags,
                                 int64_t scratch_floats) {
    if (max_m < 1 || max_n < 1 || count < 0 || scratch_floats < 0) return 0;
    if (precision != JB_PREC_NATIVE && precision != JB_PREC_MIXED) return 0;
    const int mt = max_m > max_n ? max_m : max_n, nt = max_m > max_n ? max_n : max_m;
    const Plan pl = make_plan(mt, nt, 4, precision, flags & kTuneFlags);
    size_t bytes = base_bytes(pl, count);
    if (precision == JB_PREC_MIXED) bytes += (size_t)scratch_floats * 4;
    return bytes;
}

int jb_svd_uneven_f32(const float *A, float *U, float *S, float *Vh, const jb_matrix_desc *descs,
                      const int32_t *order, int64_t count, int32_t max_m, int32_t max_n, double tol,
                      int32_t max_sweeps, int32_t precision, int32_t *sweeps, int32_t *status, void *workspace,
                      size_t workspace_bytes, void *stream) {
    return jb_svd_uneven_f32_ex(A, U, S, Vh, descs, order, count, max_m, max_n, tol, max_sweeps, precision, 0, 0.0,
                                sweeps, status, workspace, workspace_bytes, stream);
}

int jb_svd_uneven_f32_ex(const float *A, float *U, float *S, float *Vh, const jb_matrix_desc *descs,
                         const int32_t *order, int64_t count, int32_t max_m, int32_t max_n, double tol,
                         int32_t max_sweeps, int32_t precision, int32_t flags, double exit_ratio, int32_t *sweeps,
                         int32_t *status, void *workspace, size_t workspace_bytes, void *stream) {
    if (count < 0 || max_m < 1 || max_n < 1 || max_sweeps < 1 || !A || !S || !descs) return JB_EINVAL;
    if (precision != JB_PREC_NATIVE && precision != JB_PREC_MIXED) return JB_EINVAL;
    if (flags & ~kTuneFlags) return JB_EINVAL;
    const int mt = max_m > max_n ? max_m : max_n, nt = max_m > max_n ? max_n : max_m;
    if (mt > 8192 || nt > 4096) return JB_ETOOBIG;
    if (count == 0) return JB_OK;
    const Plan pl = make_plan(mt, nt, 4, precision, flags);
    if (!workspace || workspace_bytes < base_bytes(pl, count)) return JB_EWORKSPACE;
    Params p;
    memset(&p, 0, sizeof(p));
    p.A = A; p.U = U; p.S = S; p.Vh = Vh;
    p.descs = descs; p.order = order; p.count = count;
    p.tol = tol; p.max_sweeps = max_sweeps; p.tol32 = tol; p.max_sweeps32 = max_sweeps;
    p.sweeps = sweeps; p.status = status;
    p.exit_ratio = (float)exit_ratio;
    return launch_any(p, pl, 4, precision, workspace, workspace_bytes, (cudaStream_t)stream);
}


int jb_warm_prep_f32(const float *A, const float *V0, float *Vstart, int32_t *used, float *off0, float *off1,
                     int64_t batch, int32_t m, int32_t n, void *stream) {
    if (!A || !V0 || !Vstart || batch < 0 || m < n || n < 1 || n % 4) return JB_EINVAL;
    if (batch == 0) return JB_OK;
    const int ldm = (m + 3) & ~3;
    const size_t smem = align16(((size_t)m * n + (size_t)ldm * n) * 4) + ((size_t)3 * n * n + 64 + 2 * n) * 8;
    if (smem > kSmemLimit) return JB_ETOOBIG;
    if (cudaFuncSetAttribute(warm_prep_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
        cudaSuccess)
        return JB_ECUDA;
    const int sms = sm_count();
    if (sms <= 0) return JB_ECUDA;
    int64_t grid = (int64_t)sms * 4;
    if (grid > batch) grid = batch;
    warm_prep_kernel<<<(unsigned)grid, 256, smem, (cudaStream_t)stream>>>(A, V0, Vstart, used, off0, off1, batch,
                                                                          m, n);
    return cudaGetLastError() == cudaSuccess ? JB_OK : JB_ECUDA;
}

int jb_svd_warm_f32(const float *A, const float *Vstart, float *U, float *S, float *Vh, int64_t batch, int32_t m,
                    int32_t n, int32_t rank, int32_t flags, double tol, int32_t max_sweeps, int32_t precision,
                    int32_t *sweeps, int32_t *status, void *workspace, size_t workspace_bytes, void *stream) {
    int rc = check_common(batch, m, n, rank, flags, max_sweeps);
    if (rc) return rc;
    if (!A || !Vstart || !S || m < n || (!(flags & JB_VALUES_ONLY) && (!U || !Vh))) return JB_EINVAL;
    if (precision != JB_PREC_NATIVE && precision != JB_PREC_MIXED) return JB_EINVAL;
    if (batch == 0) return JB_OK;
    Plan pl = make_plan(m, n, 4, precision, flags);
    if (!pl.reg) return JB_ETOOBIG;
    const size_t stage = align16((size_t)32 * ((m + 31) / 32) * n * 4);
    // the staging of A follows W / V; the tile exchange area, used only once
    // the sweeps start, shares its space
    pl.reg32 += stage;
    pl.smem32 = aux_bytes(pl.d32) + (pl.reg32 > pl.xoff32 + pl.xbytes32 ? pl.reg32 : pl.xoff32 + pl.xbytes32);
    if (pl.smem32 > kSmemLimit) return JB_ETOOBIG;
    if (workspace_bytes < uniform_workspace(m, n, batch, 4, precision, flags)) return JB_EWORKSPACE;
    Params p;
    memset(&p, 0, sizeof(p));
    p.A = A;
    p.U = (flags & JB_VALUES_ONLY) ? nullptr : U;
    p.S = S;
    p.Vh = (flags & JB_VALUES_ONLY) ? nullptr : Vh;
    p.count = batch; p.um = m; p.un = n; p.urank = rank; p.uflags = flags & ~JB_ROUND_ROBIN;
    p.tol = tol; p.max_sweeps = max_sweeps; p.tol32 = tol; p.max_sweeps32 = max_sweeps;
    p.sweeps = sweeps; p.status = status;
    p.vstart = Vstart;
    return launch_reg(p, pl, 4, precision, (unsigned char *)workspace, workspace_bytes, (cudaStream_t)stream);
}

int jb_svd_batched_f32_noalloc(const float *A, float *U, float *S, float *Vh, int64_t batch, int32_t m, int32_t n,
                               int32_t rank, int32_t flags, double tol, int32_t max_sweeps, int32_t precision,
                               int32_t *sweeps, int32_t *status, void *stream) {
    int rc = check_common(batch, m, n, rank, flags, max_sweeps);
    if (rc) return rc;
    if (!A || !S || (!(flags & JB_VALUES_ONLY) && (!U || !Vh))) return JB_EINVAL;
    if (precision != JB_PREC_NATIVE && precision != JB_PREC_MIXED) return JB_EINVAL;
    if (batch == 0) return JB_OK;
    if (uniform_workspace(m, n, batch, 4, precision, flags) > (size_t)JB_NOALLOC_SCRATCH_BYTES) return JB_ETOOBIG;
    void *scratch = nullptr;
    if ((rc = noalloc_scratch(&scratch))) return rc;
    return jb_svd_batched_f32(A, U, S, Vh, batch, m, n, rank, flags, tol, max_sweeps, precision, sweeps, status,
                              scratch, (size_t)JB_NOALLOC_SCRATCH_BYTES, stream);
}

}  // extern "C"
