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
#include "jacobi_b200.h"
#include "jb_device.cuh"

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
           align16((size_t)d.np * 8) + align16((size_t)d.np * 4) + align16(32 * 8) + align16(4 * 4);
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
    a.red = (double *)p; p += align16(32 * 8);
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
    unsigned char *gws;           // NULL: work area in shared memory
    size_t gws_stride;
    Dims maxd;                    // sizing of aux / region (largest matrix)
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
    Geo g32 = g;
    g32.ncp = g.np;
    load_tall(A, g32, e, W32);
    set_identity(V32, g.np, g.ldv);
    __syncthreads();
    const float tol32 = p.tol32 > 0 ? (float)p.tol32 : 10.0f * Lim<float>::eps();
    bool conv32;
    const int s1 = sweeps<float>(W32, V32, g32, tol32, p.max_sweeps32, ax, conv32);
    for (int idx = threadIdx.x; idx < g.np * g.np; idx += blockDim.x) {
        int c = idx / g.np, i = idx - c * g.np;
        V64[(size_t)c * g.ldv + i] = (double)V32[(size_t)c * g.ldv + i];
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
        if (!desc_fits(d, p.maxd)) st = JB_ST_BAD_DESC;
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

struct Plan {
    Dims d;
    size_t aux, region, smem;
    bool global_region;
    int threads;
};

static Plan make_plan(int max_mt, int max_nt, int elem, int precision, int flags) {
    Plan pl;
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
    return pl;
}

template <typename T, int PREC>
static int launch(Params &p, const Plan &pl, void *workspace, size_t ws_bytes, bool dynamic, cudaStream_t st) {
    const int sms = sm_count();
    if (sms <= 0) return JB_ECUDA;
    auto kern = batched_kernel<T, PREC>;
    if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)pl.smem) != cudaSuccess)
        return JB_ECUDA;
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, pl.threads, pl.smem) != cudaSuccess)
        return JB_ECUDA;
    if (per_sm < 1) return JB_ETOOBIG;
    int64_t grid = (int64_t)sms * per_sm;
    if (grid > p.count) grid = p.count;
    if (grid < 1) grid = 1;
    unsigned char *ws = (unsigned char *)workspace;
    p.maxd = pl.d;
    p.counter = nullptr;
    p.gws = nullptr;
    p.gws_stride = 0;
    if (dynamic || pl.global_region) {
        if (!ws) return JB_EWORKSPACE;
    }
    if (dynamic) {
        p.counter = (int *)ws;
        if (cudaMemsetAsync(p.counter, 0, sizeof(int), st) != cudaSuccess) return JB_ECUDA;
    }
    if (pl.global_region) {
        const size_t stride = align16(pl.region) + 256;
        const int64_t max_grid = (int64_t)((ws_bytes - kCounterBytes) / stride);
        if (ws_bytes < kCounterBytes + stride) return JB_EWORKSPACE;
        if (grid > max_grid) grid = max_grid;
        p.gws = ws + kCounterBytes;
        p.gws_stride = stride;
    }
    kern<<<(unsigned)grid, pl.threads, pl.smem, st>>>(p);
    return cudaGetLastError() == cudaSuccess ? JB_OK : JB_ECUDA;
}

static size_t workspace_for(const Plan &pl, int64_t count) {
    size_t bytes = kCounterBytes;
    if (pl.global_region) {
        const int sms = sm_count();
        int64_t grid = sms > 0 ? sms : 148;
        if (grid > count) grid = count;
        bytes += (size_t)grid * (align16(pl.region) + 256);
    }
    return bytes;
}

static int check_common(int64_t count, int32_t m, int32_t n, int32_t rank, int32_t flags, int32_t max_sweeps) {
    if (count < 0 || m < 1 || n < 1 || max_sweeps < 1) return JB_EINVAL;
    const int k = m < n ? m : n;
    if (rank < 1 || rank > k) return JB_EINVAL;
    if ((flags & JB_FULL_MATRICES) && rank != k) return JB_EINVAL;
    if ((m > n ? m : n) > 8192 || k > 4096) return JB_ETOOBIG;
    return JB_OK;
}

}  // namespace jb

using namespace jb;

extern "C" {

int jb_version(void) { return 100; }

int jb_device_sm_count(void) { return sm_count(); }

size_t jb_workspace_bytes(int32_t max_m, int32_t max_n, int64_t count, int32_t elem_bytes, int32_t precision,
                          int32_t flags) {
    if (max_m < 1 || max_n < 1 || (elem_bytes != 4 && elem_bytes != 8)) return 0;
    const int mt = max_m > max_n ? max_m : max_n, nt = max_m > max_n ? max_n : max_m;
    const Plan pl = make_plan(mt, nt, elem_bytes, elem_bytes == 4 ? precision : JB_PREC_NATIVE, flags);
    return workspace_for(pl, count);
}

int jb_svd_batched_f32(const float *A, float *U, float *S, float *Vh, int64_t batch, int32_t m, int32_t n,
                       int32_t rank, int32_t flags, double tol, int32_t max_sweeps, int32_t precision,
                       int32_t *sweeps, int32_t *status, void *workspace, size_t workspace_bytes, void *stream) {
    int rc = check_common(batch, m, n, rank, flags, max_sweeps);
    if (rc) return rc;
    if (!A || !S || (!(flags & JB_VALUES_ONLY) && (!U || !Vh))) return JB_EINVAL;
    if (precision != JB_PREC_NATIVE && precision != JB_PREC_MIXED) return JB_EINVAL;
    if (batch == 0) return JB_OK;
    Params p;
    memset(&p, 0, sizeof(p));
    p.A = A; p.U = (flags & JB_VALUES_ONLY) ? nullptr : U; p.S = S; p.Vh = (flags & JB_VALUES_ONLY) ? nullptr : Vh;
    p.count = batch; p.um = m; p.un = n; p.urank = rank; p.uflags = flags;
    p.tol = tol; p.max_sweeps = max_sweeps; p.tol32 = tol; p.max_sweeps32 = max_sweeps;
    p.sweeps = sweeps; p.status = status;
    const int mt = m > n ? m : n, nt = m > n ? n : m;
    const Plan pl = make_plan(mt, nt, 4, precision, flags);
    if (workspace && workspace_bytes < workspace_for(pl, batch)) return JB_EWORKSPACE;
    cudaStream_t st = (cudaStream_t)stream;
    return precision == JB_PREC_MIXED ? launch<float, JB_PREC_MIXED>(p, pl, workspace, workspace_bytes, false, st)
                                      : launch<float, JB_PREC_NATIVE>(p, pl, workspace, workspace_bytes, false, st);
}

int jb_svd_batched_f64(const double *A, double *U, double *S, double *Vh, int64_t batch, int32_t m, int32_t n,
                       int32_t rank, int32_t flags, double tol, int32_t max_sweeps, int32_t *sweeps,
                       int32_t *status, void *workspace, size_t workspace_bytes, void *stream) {
    int rc = check_common(batch, m, n, rank, flags, max_sweeps);
    if (rc) return rc;
    if (!A || !S || (!(flags & JB_VALUES_ONLY) && (!U || !Vh))) return JB_EINVAL;
    if (batch == 0) return JB_OK;
    Params p;
    memset(&p, 0, sizeof(p));
    p.A = A; p.U = (flags & JB_VALUES_ONLY) ? nullptr : U; p.S = S; p.Vh = (flags & JB_VALUES_ONLY) ? nullptr : Vh;
    p.count = batch; p.um = m; p.un = n; p.urank = rank; p.uflags = flags;
    p.tol = tol; p.max_sweeps = max_sweeps;
    p.sweeps = sweeps; p.status = status;
    const int mt = m > n ? m : n, nt = m > n ? n : m;
    const Plan pl = make_plan(mt, nt, 8, JB_PREC_NATIVE, flags);
    if (workspace && workspace_bytes < workspace_for(pl, batch)) return JB_EWORKSPACE;
    return launch<double, JB_PREC_NATIVE>(p, pl, workspace, workspace_bytes, false, (cudaStream_t)stream);
}

int jb_svd_uneven_f32(const float *A, float *U, float *S, float *Vh, const jb_matrix_desc *descs,
                      const int32_t *order, int64_t count, int32_t max_m, int32_t max_n, double tol,
                      int32_t max_sweeps, int32_t precision, int32_t *sweeps, int32_t *status, void *workspace,
                      size_t workspace_bytes, void *stream) {
    if (count < 0 || max_m < 1 || max_n < 1 || max_sweeps < 1 || !A || !S || !descs) return JB_EINVAL;
    if (precision != JB_PREC_NATIVE && precision != JB_PREC_MIXED) return JB_EINVAL;
    const int mt = max_m > max_n ? max_m : max_n, nt = max_m > max_n ? max_n : max_m;
    if (mt > 8192 || nt > 4096) return JB_ETOOBIG;
    if (count == 0) return JB_OK;
    Params p;
    memset(&p, 0, sizeof(p));
    p.A = A; p.U = U; p.S = S; p.Vh = Vh;
    p.descs = descs; p.order = order; p.count = count;
    p.tol = tol; p.max_sweeps = max_sweeps; p.tol32 = tol; p.max_sweeps32 = max_sweeps;
    p.sweeps = sweeps; p.status = status;
    const Plan pl = make_plan(mt, nt, 4, precision, 0);
    if (!workspace || workspace_bytes < workspace_for(pl, count)) return JB_EWORKSPACE;
    cudaStream_t st = (cudaStream_t)stream;
    return precision == JB_PREC_MIXED ? launch<float, JB_PREC_MIXED>(p, pl, workspace, workspace_bytes, true, st)
                                      : launch<float, JB_PREC_NATIVE>(p, pl, workspace, workspace_bytes, true, st);
}

}  // extern "C"
