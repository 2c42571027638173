// jb_tc.cuh - tcgen05 (5th-generation tensor core) BF16 GEMM for sm_100a.
//
//   C[z] (M x N, fp32) = alpha * sum_t A_{a(t)}[z] (M x K) * B_{b(t)}[z] (N x K)^T  (+ C)
//
// A_i and B_i are row-major BF16 (K contiguous = "K-major").  Up to two A and
// two B variants and three terms, so one accumulator holds a compensated
// 3xBF16 product  X Y^T ~ Xhi Yhi^T + Xhi Ylo^T + Xlo Yhi^T  (Xhi = bf16(X),
// Xlo = bf16(X - Xhi)).
//
// One CTA computes one 128 x BN tile of C over a K range (split-K over
// blockIdx.z accumulates with atomics).  Warp 0 (one elected lane) streams
// 128 x 64 / BN x 64 tiles with TMA (128-byte swizzle) into a ring of
// shared-memory stages; warp 1 (one elected lane) issues tcgen05.mma
// (M = 128, N = BN, K = 16 per instruction) into a TMEM accumulator and
// releases each stage with tcgen05.commit; all four warps then read the
// accumulator with tcgen05.ld (warp w owns TMEM lanes / tile rows 32w..32w+31)
// and write C.  Every wait is bounded: on a timeout the kernel sets
// *error_flag, drains what it issued, frees its TMEM and returns.
#pragma once
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace jb {
namespace tc {

constexpr int BM = 128;
constexpr int BK = 64;                    // one 128-byte swizzle row of BF16
constexpr uint32_t A_TILE = BM * BK * 2;  // 16 KiB
constexpr long long kWaitCycles = 4000000000LL;  // ~2 s at 2 GHz

struct TcParams {
    CUtensorMap ta[3], tb[6];   // tb[3..5]: the B parts of a second product (nx1 > 0)
    float *C;
    long long ldc, sC;
    int M, N, K;
    int kchunk;        // K range per split (multiple of BK)
    int splits;        // blockIdx.z = batch * splits + split
    int stages;        // shared-memory ring depth
    int nterm;
    int term_a[6], term_b[6];
    int na, nb;        // operand variants actually loaded
    int b_mn;          // B stored K x N (N contiguous) instead of N x K
    float alpha, beta; // beta: 0 overwrite, 1 accumulate (atomic when splits > 1)
    int *error_flag;
    // Accumulation chains: k-blocks (of BK) per TMEM accumulator and the
    // number of accumulators (BN * nacc <= 512 columns); the epilogue sums
    // them in FP32 registers.
    int acc_kb, nacc;
    int a_as_b;        // B = A (a Gram X X^T): the B operand is read from the A tiles
    // Row-mapped BF16-part output instead of C: row r of batch z goes to row
    // out_map[z * M + r] (or z * M + r) of out_part[0..out_nparts), each row
    // out_ld elements long, as hi / mid / lo splits of alpha * (A B^T).
    __nv_bfloat16 *out_part[3];
    int out_nparts;
    const int *out_map;
    long long out_ld;
    // A second product in the same launch (row-mapped output only): the
    // column tiles blockIdx.x >= nx1 (nx1 > 0) compute alpha * A B2^T (B2's
    // parts in tb[3..5]) with the same A, K and row map into out_part2, N2
    // columns, rows out_ld2 long.
    int nx1, N2;
    __nv_bfloat16 *out_part2[3];
    long long out_ld2;
};

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Bounded wait; returns false (and raises the flag) after ~kWaitCycles.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, int *flag) {
    const long long t0 = clock64();
    while (!mbar_try_wait(bar, parity)) {
        if (clock64() - t0 > kWaitCycles) {
            if (flag) atomicExch(flag, 1);
            return false;
        }
    }
    return true;
}

__device__ __forceinline__ void tma_load_3d(void *dst, const CUtensorMap *map, int x, int y, int z, uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4, %5}], [%2];"
        ::"r"(smem_u32(dst)), "l"((uint64_t)map), "r"(smem_u32(bar)), "r"(x), "r"(y), "r"(z)
        : "memory");
}

// Shared-memory matrix descriptor: K-major tile, 128-byte swizzle, rows of
// 128 bytes, 8-row groups 1024 bytes apart (SBO), version 1 (sm_100).
__device__ __forceinline__ uint64_t smem_desc_sw128(const void *tile) {
    const uint64_t addr = smem_u32(tile);
    uint64_t d = 0;
    d |= (addr >> 4) & 0x3FFFull;            // start address
    d |= (uint64_t)1 << 16;                  // leading byte offset (unused with swizzle)
    d |= (uint64_t)(1024 >> 4) << 32;        // stride byte offset
    d |= (uint64_t)1 << 46;                  // version
    d |= (uint64_t)2 << 61;                  // SWIZZLE_128B
    return d;
}

// MN-major tile (N contiguous), 128-byte swizzle: rows of 64 N-elements per
// k, 8-row K groups 1024 bytes apart (SBO), 64-element N chunks (one TMA box
// of 64 x 64) 8192 bytes apart (LBO).
__device__ __forceinline__ uint64_t smem_desc_mn_sw128(const void *tile) {
    const uint64_t addr = smem_u32(tile);
    uint64_t d = 0;
    d |= (addr >> 4) & 0x3FFFull;
    d |= (uint64_t)(8192 >> 4) << 16;        // leading byte offset: next N chunk
    d |= (uint64_t)(1024 >> 4) << 32;        // stride byte offset: next 8-row K group
    d |= (uint64_t)1 << 46;
    d |= (uint64_t)2 << 61;
    return d;
}

// Instruction descriptor, kind::f16: D fp32, A and B bf16, A K-major, B
// K-major or (b_mn) MN-major.
__host__ __device__ constexpr uint32_t idesc_bf16(int M, int N, int b_mn = 0) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(b_mn ? 1 : 0) << 16) | ((uint32_t)(N >> 3) << 17) |
           ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                         uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}"
        ::"r"(tmem_d), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(0), "r"(0), "r"(0), "r"(0));
}

__device__ __forceinline__ void mma_commit(uint64_t *bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32]) {
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

// Stores 32 consecutive values of one output row as hi / mid / lo BF16
// parts (16-byte stores when the row segment is 16-byte aligned and whole).
__device__ __forceinline__ void store_parts32(__nv_bfloat16 *out0, __nv_bfloat16 *out1, __nv_bfloat16 *out2,
                                              int nparts, int N, float alpha, long long base, int col0,
                                              const float (&v)[32]) {
    const bool vec = col0 + 32 <= N && ((base + col0) & 7) == 0;
    if (vec) {
#pragma unroll
        for (int g = 0; g < 4; ++g) {
            uint32_t wh[4], wm[4], wl[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                wh[i] = wm[i] = wl[i] = 0u;
#pragma unroll
                for (int e = 0; e < 2; ++e) {
                    const float x = alpha * v[g * 8 + i * 2 + e];
                    const __nv_bfloat16 h = __float2bfloat16_rn(x);
                    const float r1 = x - __bfloat162float(h);
                    const __nv_bfloat16 m = __float2bfloat16_rn(r1);
                    const __nv_bfloat16 l = __float2bfloat16_rn(r1 - __bfloat162float(m));
                    wh[i] |= (uint32_t)__bfloat16_as_ushort(h) << (16 * e);
                    wm[i] |= (uint32_t)__bfloat16_as_ushort(m) << (16 * e);
                    wl[i] |= (uint32_t)__bfloat16_as_ushort(l) << (16 * e);
                }
            }
            const long long o = base + col0 + g * 8;
            *(uint4 *)(out0 + o) = make_uint4(wh[0], wh[1], wh[2], wh[3]);
            if (nparts > 1) *(uint4 *)(out1 + o) = make_uint4(wm[0], wm[1], wm[2], wm[3]);
            if (nparts > 2) *(uint4 *)(out2 + o) = make_uint4(wl[0], wl[1], wl[2], wl[3]);
        }
    } else {
#pragma unroll
        for (int i = 0; i < 32; ++i) {
            if (col0 + i >= N) break;
            const float x = alpha * v[i];
            const __nv_bfloat16 h = __float2bfloat16_rn(x);
            const float r1 = x - __bfloat162float(h);
            const __nv_bfloat16 m = __float2bfloat16_rn(r1);
            out0[base + col0 + i] = h;
            if (nparts > 1) out1[base + col0 + i] = m;
            if (nparts > 2) out2[base + col0 + i] = __float2bfloat16_rn(r1 - __bfloat162float(m));
        }
    }
}

template <int BN>
__global__ void __launch_bounds__(128, 1) tc_gemm_kernel(const __grid_constant__ TcParams p) {
    const int STAGES = p.stages;
    constexpr uint32_t B_TILE = BN * BK * 2;
    const uint32_t tmem_cols = (uint32_t)(BN * p.nacc) < 32 ? 32u : (uint32_t)(BN * p.nacc);
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    // 1024-byte alignment for the swizzled tiles.
    unsigned char *smem = (unsigned char *)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    const uint32_t stage_bytes = p.na * A_TILE + (p.a_as_b ? 0u : p.nb * B_TILE);
    uint64_t *full = (uint64_t *)(smem + STAGES * stage_bytes);
    uint64_t *empty = full + STAGES;
    uint64_t *done = empty + STAGES;
    uint32_t *tmem_slot = (uint32_t *)(done + 1);
    __shared__ int s_err;

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    // the launch's second product (nx1 > 0): its column tiles follow the first's
    const bool second = p.nx1 > 0 && (int)blockIdx.x >= p.nx1;
    const int n0 = (second ? (int)blockIdx.x - p.nx1 : (int)blockIdx.x) * BN, m0 = blockIdx.y * BM;
    const int Ncols = second ? p.N2 : p.N;
    const int tb0 = second ? 3 : 0;
    // (scalars selected here: a pointer into the parameter arrays chosen at run
    // time would make the compiler copy them to local memory)
    __nv_bfloat16 *const out0 = second ? p.out_part2[0] : p.out_part[0];
    __nv_bfloat16 *const out1 = second ? p.out_part2[1] : p.out_part[1];
    __nv_bfloat16 *const out2 = second ? p.out_part2[2] : p.out_part[2];
    const long long out_ld = second ? p.out_ld2 : p.out_ld;
    const int batch = blockIdx.z / p.splits, split = blockIdx.z % p.splits;
    const int kbeg = split * p.kchunk;
    const int kend = min(p.K, kbeg + p.kchunk);
    const int nk = kend > kbeg ? (kend - kbeg + BK - 1) / BK : 0;
    // accumulators that receive at least one chain
    const int nacc_used = min(p.nacc, (nk + p.acc_kb - 1) / p.acc_kb);

    if (threadIdx.x == 0) {
        s_err = 0;
        for (int s = 0; s < STAGES; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        mbar_init(done, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(tmem_cols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = *tmem_slot;

    if (warp == 0 && lane == 0) {
        // TMA producer.
        int issued = 0;
        for (int kb = 0; kb < nk; ++kb) {
            const int s = kb % STAGES;
            const uint32_t ph = (kb / STAGES) & 1;
            if (!mbar_wait(&empty[s], ph ^ 1, p.error_flag)) { s_err = 1; break; }
            if (s_err) break;
            mbar_expect_tx(&full[s], stage_bytes);
            unsigned char *st = smem + s * stage_bytes;
            const int kx = kbeg + kb * BK;
            for (int a = 0; a < p.na; ++a) tma_load_3d(st + a * A_TILE, &p.ta[a], kx, m0, batch, &full[s]);
            if (!p.a_as_b) {
                for (int b = 0; b < p.nb; ++b) {
                    unsigned char *bt = st + p.na * A_TILE + b * B_TILE;
                    if (!p.b_mn) {
                        tma_load_3d(bt, &p.tb[b + tb0], kx, n0, batch, &full[s]);
                    } else {
                        for (int g = 0; g < BN / 64; ++g)
                            tma_load_3d(bt + g * 8192, &p.tb[b + tb0], n0 + 64 * g, kx, batch, &full[s]);
                    }
                }
            }
            issued = kb + 1;
        }
        // Drain: the last stages' copies must land before the CTA can exit.
        for (int kb = issued - STAGES < 0 ? 0 : issued - STAGES; kb < issued; ++kb)
            mbar_wait(&full[kb % STAGES], (kb / STAGES) & 1, nullptr);
    } else if (warp == 1 && lane == 0) {
        // MMA issuer.
        const uint32_t idesc = idesc_bf16(BM, BN, p.b_mn);
        const uint32_t bstep = p.b_mn ? (2048 >> 4) : 2;  // +16 K rows (MN-major) or +32 bytes (K-major)
        bool ok = true;
        for (int kb = 0; kb < nk && ok; ++kb) {
            const int s = kb % STAGES;
            const uint32_t ph = (kb / STAGES) & 1;
            if (!mbar_wait(&full[s], ph, p.error_flag)) { s_err = 1; ok = false; break; }
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            unsigned char *st = smem + s * stage_bytes;
            const int chain = kb / p.acc_kb;
            const uint32_t acc = tmem + (uint32_t)((chain % p.nacc) * BN);
            const bool fresh = (kb % p.acc_kb) == 0 && chain < p.nacc;
            for (int t = 0; t < p.nterm; ++t) {
                const uint64_t ad = smem_desc_sw128(st + p.term_a[t] * A_TILE);
                const unsigned char *bt = p.a_as_b ? st + p.term_b[t] * A_TILE
                                                   : st + p.na * A_TILE + p.term_b[t] * B_TILE;
                const uint64_t bd = p.b_mn ? smem_desc_mn_sw128(bt) : smem_desc_sw128(bt);
#pragma unroll
                for (int k = 0; k < BK / 16; ++k)  // +32 bytes per K=16 step inside the swizzled row
                    mma_bf16(acc, ad + 2 * k, bd + bstep * k, idesc, (fresh && t == 0 && k == 0) ? 0u : 1u);
            }
            mma_commit(&empty[s]);
        }
        mma_commit(done);
    }
    __syncwarp();
    // Epilogue: all four warps.
    const bool have = nk > 0 && mbar_wait(done, 0, p.error_flag);
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const int row = m0 + warp * 32 + lane;
    // tcgen05.ld is warp-collective: decide per warp.
    if (__all_sync(0xffffffffu, have && !s_err)) {
        const long long obase = p.out_nparts
            ? (long long)(p.out_map && row < p.M ? p.out_map[(long long)batch * p.M + row]
                                                 : (long long)batch * p.M + row) * out_ld
            : 0;
        float *crow = p.C ? p.C + (long long)batch * p.sC + (long long)row * p.ldc : nullptr;
#pragma unroll 1
        for (int c0 = 0; c0 < BN; c0 += 32) {
            float v[32];
            tmem_ld32(tmem + ((uint32_t)(warp * 32) << 16) + c0, v);
            for (int a = 1; a < nacc_used; ++a) {
                float w[32];
                tmem_ld32(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(a * BN) + c0, w);
#pragma unroll
                for (int i = 0; i < 32; ++i) v[i] += w[i];
            }
            if (row >= p.M || n0 + c0 >= Ncols) continue;
            if (p.out_nparts) {
                store_parts32(out0, out1, out2, p.out_nparts, Ncols, p.alpha, obase, n0 + c0, v);
            } else if (p.splits == 1 && n0 + c0 + 32 <= Ncols && (((uintptr_t)(crow + n0 + c0)) & 15) == 0) {
#pragma unroll
                for (int g = 0; g < 8; ++g) {
                    float4 *dst = (float4 *)(crow + n0 + c0 + 4 * g);
                    float4 x = make_float4(p.alpha * v[4 * g], p.alpha * v[4 * g + 1], p.alpha * v[4 * g + 2],
                                           p.alpha * v[4 * g + 3]);
                    if (p.beta != 0.f) {
                        const float4 o = *dst;
                        x.x += o.x; x.y += o.y; x.z += o.z; x.w += o.w;
                    }
                    *dst = x;
                }
            } else {
#pragma unroll
                for (int i = 0; i < 32; ++i) {
                    const int col = n0 + c0 + i;
                    if (col < Ncols) {
                        const float x = p.alpha * v[i];
                        if (p.splits > 1) atomicAdd(&crow[col], x);
                        else crow[col] = p.beta != 0.f ? crow[col] + x : x;
                    }
                }
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(tmem_cols));
    }
}

}  // namespace tc
}  // namespace jb
