/*
 * jacobi_b200.h - C ABI of the B200 (sm_100a) one-sided Jacobi SVD library.
 *
 * Plain pointers and sizes only: every buffer argument is a DEVICE pointer,
 * every stream is a cudaStream_t passed as void*.  Every entry point returns
 * an int status (JB_OK or a JB_E* code) and never aborts the process; it only
 * enqueues work on the given stream (asynchronous).  Per-matrix outcomes
 * (converged / not converged / non-finite input / failed null completion /
 * non-finite output) land in the caller's `status` array on the device.
 *
 * Reference interfaces replaced (uncle-Slava/Pavel-s_SVD, paths relative to
 * that project):
 *   jb_svd_batched_*     svdbench/standalone/primitives.py:316-367 (jacobi_svd),
 *                        with solvers.py:224-230 (wide -> tall via adjoint),
 *                        solvers.py:289-310 (scaling, truncation, full bases)
 *                        and primitives.py:430-467 (null-space completion)
 *                        fused into one launch.
 *   jb_svd_uneven_f32    the per-matrix loop a harness runs over svd(x,'jacobi')
 *                        for matrices of different shapes (the reference can
 *                        only batch equal shapes: solvers.py:289-290).
 */
#ifndef JACOBI_B200_H
#define JACOBI_B200_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define JB_API __attribute__((visibility("default")))
#else
#define JB_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* ---- return codes of the entry points ---------------------------------- */
#define JB_OK               0
#define JB_EINVAL           1   /* bad argument (null pointer, size, tolerance) */
#define JB_ETOOBIG          2   /* shape exceeds what the entry point supports  */
#define JB_EWORKSPACE       3   /* workspace missing or smaller than required   */
#define JB_ECUDA            4   /* a CUDA runtime call failed                   */

/* ---- per-matrix status words written to `status` ------------------------ */
#define JB_ST_OK            0   /* converged, outputs written                        */
#define JB_ST_NOT_CONVERGED 1   /* off > tol after max_sweeps (primitives.py:354-355) */
#define JB_ST_NONFINITE_IN  2   /* NaN/Inf in the input (solvers.py:291-292)          */
#define JB_ST_NULL_FAILED   3   /* null completion failed (primitives.py:451-452)     */
#define JB_ST_NONFINITE_OUT 4   /* NaN/Inf in an output (solvers.py:305-306)          */
#define JB_ST_BAD_DESC      5   /* descriptor outside the launch's max sizes/flags    */
#define JB_ST_TIMEOUT       6   /* a bounded wait inside a multi-CTA kernel ran out   */

/* ---- flags ---------------------------------------------------------------- */
#define JB_FULL_MATRICES    1   /* U is m x m and Vh is n x n (complete_basis)  */
#define JB_VALUES_ONLY      2   /* write S only; U and Vh may be NULL           */
#define JB_ROUND_ROBIN      4   /* sweep in the reference's round-robin pair
                                   order (primitives.py:309-313) instead of the
                                   register-blocked order; same results within
                                   rounding, slower                             */
#define JB_BLOCK_WIDTH_8    8   /* uneven batches: FP32 register sweeps with
                                   8-column blocks (4 warps per 64 columns)
                                   instead of 4-column blocks                   */
#define JB_ONE_SIZE_CLASS  16   /* uneven batches: no second launch per phase
                                   for the matrices of at most 32 columns (tall
                                   view) in half-size CTAs; every matrix runs
                                   in the full-size CTAs.  Same results; a
                                   choice for the autotuner                     */

/* ---- arithmetic of the solve ------------------------------------------- */
#define JB_PREC_NATIVE      0   /* sweeps in the input precision (f32 or f64)   */
#define JB_PREC_MIXED       1   /* f32 input: FP32 sweeps, then Householder-QR
                                   re-orthonormalised V and FP64 sweeps from
                                   W = A V to the same tolerance; f64 input:
                                   same as NATIVE                               */

/* One matrix of an uneven batch.  A is row-major m x n at A + a_off.
 * Outputs (row-major): U at U + u_off (m x ucols), S at S + s_off (k values),
 * Vh at Vh + v_off (vrows x n), where k = rank, ucols = vrows = rank, or with
 * JB_FULL_MATRICES ucols = m, vrows = n.  Offsets count elements.
 * x_off: offset (in floats) of this matrix's min(m,n)^2 scratch floats inside
 * the workspace scratch area (used by JB_PREC_MIXED only). */
typedef struct jb_matrix_desc {
    int32_t m, n;
    int32_t rank;       /* 1 <= rank <= min(m, n) */
    int32_t flags;      /* JB_FULL_MATRICES | JB_VALUES_ONLY | JB_ROUND_ROBIN */
    int64_t a_off, u_off, s_off, v_off;
    int64_t x_off;
} jb_matrix_desc;

/* Library version (major*10000 + minor*100 + patch). */
JB_API int jb_version(void);

/* Number of streaming multiprocessors of the current device, or -1. */
JB_API int jb_device_sm_count(void);

/* Bytes of device workspace that jb_svd_batched_* need for `count` matrices
 * of max_m x max_n (either orientation), the given precision and flags.
 * jb_svd_uneven_f32 needs this for its largest shape plus, with
 * JB_PREC_MIXED, 4 bytes per scratch float addressed by the descriptors'
 * x_off (see jb_svd_uneven_f32). */
JB_API size_t jb_workspace_bytes(int32_t max_m, int32_t max_n, int64_t count,
                          int32_t elem_bytes, int32_t precision, int32_t flags);

/* Equal-shape batch: `batch` row-major m x n matrices at A (stride m*n).
 * U: batch x m x ucols, S: batch x k, Vh: batch x vrows x n (see
 * jb_matrix_desc).  tol <= 0 selects the reference default 10*eps(dtype)
 * (primitives.py:325).  sweeps/status: `batch` int32 each (device).
 * Replaces svd(a, 'jacobi', tol=, max_sweeps=, rank=, full_matrices=,
 * values_only=) of svdbench/standalone/solvers.py:264-310 for real dtypes. */
JB_API int jb_svd_batched_f32(const float *A, float *U, float *S, float *Vh,
                       int64_t batch, int32_t m, int32_t n, int32_t rank,
                       int32_t flags, double tol, int32_t max_sweeps,
                       int32_t precision, int32_t *sweeps, int32_t *status,
                       void *workspace, size_t workspace_bytes, void *stream);

JB_API int jb_svd_batched_f64(const double *A, double *U, double *S, double *Vh,
                       int64_t batch, int32_t m, int32_t n, int32_t rank,
                       int32_t flags, double tol, int32_t max_sweeps,
                       int32_t *sweeps, int32_t *status,
                       void *workspace, size_t workspace_bytes, void *stream);

/* Uneven batch in ONE persistent launch per precision phase.  descs: `count`
 * device descriptors; order: optional device permutation of [0, count)
 * giving the processing order (largest cost first balances the persistent
 * grid), or NULL.  max_m/max_n bound every descriptor (either orientation).
 * Workspace: jb_uneven_workspace_bytes(max_m, max_n, count, precision,
 * scratch_floats) bytes, where scratch_floats (JB_PREC_MIXED) covers every
 * descriptor's x_off + nt^2 (the FP32 V handed from the FP32 to the FP64
 * phase); a descriptor whose scratch does not fit gets JB_ST_BAD_DESC.
 * Replaces a harness loop of svd(x, 'jacobi') over matrices of different
 * shapes. */
JB_API size_t jb_uneven_workspace_bytes(int32_t max_m, int32_t max_n, int64_t count,
                                        int32_t precision, int32_t flags, int64_t scratch_floats);

JB_API int jb_svd_uneven_f32(const float *A, float *U, float *S, float *Vh,
                      const jb_matrix_desc *descs, const int32_t *order,
                      int64_t count, int32_t max_m, int32_t max_n,
                      double tol, int32_t max_sweeps, int32_t precision,
                      int32_t *sweeps, int32_t *status,
                      void *workspace, size_t workspace_bytes, void *stream);

/* jb_svd_uneven_f32 with the launch choices an autotuner varies: flags
 * JB_ROUND_ROBIN, JB_BLOCK_WIDTH_8 and/or JB_ONE_SIZE_CLASS (the workspace
 * query must get the same flags); exit_ratio, the largest pair ratio after which the FP32 phase
 * of a mixed solve hands over to the FP64 phase (0: the default 1e-2; < 0:
 * the FP32 phase runs to tol).  Results converge to the same tolerance
 * whatever the choices. */
JB_API int jb_svd_uneven_f32_ex(const float *A, float *U, float *S, float *Vh,
                                const jb_matrix_desc *descs, const int32_t *order,
                                int64_t count, int32_t max_m, int32_t max_n,
                                double tol, int32_t max_sweeps, int32_t precision,
                                int32_t flags, double exit_ratio,
                                int32_t *sweeps, int32_t *status,
                                void *workspace, size_t workspace_bytes, void *stream);

/* ---- tensor-core building blocks (tcgen05, sm_100a) --------------------- */
#define JB_GEMM_PLAIN   0   /* C = alpha A0 B0^T (+ C)                              */
#define JB_GEMM_SPLIT3  1   /* C = alpha (A0 B0^T + A0 B1^T + A1 B0^T) (+ C): the
                               compensated 3xBF16 product of X = A0 + A1 and
                               Y = B0 + B1 (hi and lo BF16 parts)               */
#define JB_GEMM_SPLIT6  2   /* three-part split X = A0 + A1 + A2 (hi, mid, lo),
                               six products (every pair of parts two or fewer
                               splits below the leading one): ~FP32 accuracy
                               (jb_gemm_bf16x only)                            */
#define JB_GEMM_B_MN    4   /* flag: B_i is stored K x N row-major (N
                               contiguous, leading dimension ldb >= N)         */
#define JB_GEMM_CHAIN128 8  /* flag: accumulate along K in chains of at most
                               128 per tensor-memory accumulator (several per
                               CTA, summed in FP32 registers); split_k is then
                               a lower bound on the CTAs along K               */
#define JB_GEMM_SYRK    16  /* flag: B is A (C = A A^T, M == N): B and ldb /
                               strideB are ignored and the A tiles are read
                               once as both operands                           */

/* Batched BF16 GEMM on the 5th-generation tensor cores with an FP32
 * accumulator in tensor memory.  A_i: batch x M x K, B_i: batch x N x K, both
 * row-major BF16 (leading dimensions lda, ldb, multiples of 8; 16-byte
 * aligned; batch strides in elements).  C: batch x M x N row-major FP32.
 * beta 0 overwrites C, beta 1 adds to it.  split_k > 1 splits K over CTAs
 * and accumulates atomically (C is zeroed first when beta is 0).
 * error_flag (device int, may be NULL) is set to 1 if a pipeline wait timed
 * out.  No counterpart in the reference, whose products are torch matmuls
 * (svdbench/standalone/solvers.py:49-50, 52). */
JB_API int jb_gemm_bf16(const void *A0, const void *A1, const void *B0, const void *B1,
                        int32_t mode, float *C, int64_t M, int64_t N, int64_t K,
                        int64_t lda, int64_t ldb, int64_t ldc, int64_t batch,
                        int64_t strideA, int64_t strideB, int64_t strideC,
                        float alpha, float beta, int32_t split_k, int32_t *error_flag,
                        void *stream);

/* jb_gemm_bf16 with the split parts as arrays: A[0..s), B[0..s) where s is
 * 1 (PLAIN), 2 (SPLIT3) or 3 (SPLIT6). */
JB_API int jb_gemm_bf16x(const void *const *A, const void *const *B, int32_t mode, float *C,
                         int64_t M, int64_t N, int64_t K, int64_t lda, int64_t ldb, int64_t ldc,
                         int64_t batch, int64_t strideA, int64_t strideB, int64_t strideC,
                         float alpha, float beta, int32_t split_k, int32_t *error_flag,
                         void *stream);

/* jb_gemm_bf16x (split_k 1, no beta) whose result is written as BF16 split
 * parts into mapped rows instead of FP32 C: row r of batch z goes to row
 * row_map[z * M + r] (z * M + r when row_map is NULL) of out[0..nparts),
 * each output row ld_out elements long (a multiple of 8); nparts 1..3 gives
 * hi, hi + mid, hi + mid + lo as jb_split3_bf16 would.  This fuses the
 * rotation update of the blocked Jacobi with the move of each rotated block
 * into its next-round slot. */
JB_API int jb_gemm_bf16x_rows(const void *const *A, const void *const *B, int32_t mode,
                              void *const *out, int32_t nparts, const int32_t *row_map,
                              int64_t ld_out, int64_t M, int64_t N, int64_t K, int64_t lda,
                              int64_t ldb, int64_t batch, int64_t strideA, int64_t strideB,
                              float alpha, int32_t *error_flag, void *stream);

/* Two jb_gemm_bf16x_rows products in one launch that share A, K, the split
 * parts, mode and row map: alpha A B^T into out (N columns, rows ld_out long)
 * and alpha A B2^T into out2 (N2 columns, rows ld_out2 long); B2 has the
 * layout of B with its own ldb2 and strideB2.  The blocked Jacobi's rotation
 * update of W^T and of V^T with the same Q^T (solvers.py:49-50), each rotated
 * row moved to its next-round slot, without a second launch. */
JB_API int jb_gemm_bf16x_rows2(const void *const *A, const void *const *B, const void *const *B2,
                               int32_t mode, void *const *out, void *const *out2, int32_t nparts,
                               const int32_t *row_map, int64_t ld_out, int64_t ld_out2, int64_t M,
                               int64_t N, int64_t N2, int64_t K, int64_t lda, int64_t ldb,
                               int64_t ldb2, int64_t batch, int64_t strideA, int64_t strideB,
                               int64_t strideB2, float alpha, int32_t *error_flag, void *stream);

/* hi = bf16(X), lo = bf16(X - hi) for n floats (lo may be NULL). */
JB_API int jb_split_bf16(const float *X, void *hi, void *lo, int64_t n, void *stream);

/* Three-part split: hi = bf16(X), mid = bf16(X - hi), lo = bf16(X - hi - mid)
 * (lo may be NULL, then as jb_split_bf16). */
JB_API int jb_split3_bf16(const float *X, void *hi, void *mid, void *lo, int64_t n, void *stream);

/* ---- learned warm start --------------------------------------------------
 * No counterpart in the reference: its Jacobi always starts from V = I
 * (svdbench/standalone/primitives.py:324). */

/* Warm-start preparation for `batch` tall float32 matrices (m >= n, n a
 * multiple of 4): V0 (batch x n x n, row-major, columns = start vectors, e.g.
 * a network's prediction) is orthonormalised by Householder QR (the
 * primitives.py:41-89 convention, column signs kept); the result is kept as
 * start when it lowers the Gram off-norm ||offdiag(W^T W)||_F / ||W^T W||_F
 * of W = A Q below that of A, else the start is the identity.  Writes
 * Vstart (batch x n x n, column c contiguous), used[z] (1 = warm start kept)
 * and the two off-norms (may be NULL). */
JB_API int jb_warm_prep_f32(const float *A, const float *V0, float *Vstart, int32_t *used,
                            float *off0, float *off1, int64_t batch, int32_t m, int32_t n,
                            void *stream);

/* jb_svd_batched_f32 starting the sweeps from V = Vstart, W = A Vstart
 * instead of V = I (tall matrices up to 128 x 64). */
JB_API int jb_svd_warm_f32(const float *A, const float *Vstart, float *U, float *S, float *Vh,
                           int64_t batch, int32_t m, int32_t n, int32_t rank, int32_t flags,
                           double tol, int32_t max_sweeps, int32_t precision,
                           int32_t *sweeps, int32_t *status,
                           void *workspace, size_t workspace_bytes, void *stream);

/* ---- element-wise kernels of the warm-start network (jb_mlp.cu) --------- */
/* dst[z] (cols x rows, bf16) = transpose of src[z] (rows x cols, f32 or bf16). */
JB_API int jb_transpose_bf16(const void *src, int32_t src_is_f32, void *dst, int64_t rows,
                             int64_t cols, int64_t batch, void *stream);
/* out = act(Z + bias[col]) (ReLU when relu != 0), stored bf16 or f32. */
JB_API int jb_bias_act(const float *Z, const float *bias, void *out, int64_t rows, int64_t cols,
                       int32_t relu, int32_t out_bf16, void *stream);
/* G = dH where H > 0 else 0 (H bf16), stored bf16 or f32. */
JB_API int jb_relu_backward(const float *dH, const void *H, void *G, int32_t out_bf16, int64_t n,
                            void *stream);
/* out[c] = sum over rows of X[r][c]. */
JB_API int jb_col_sum(const float *X, float *out, int64_t rows, int64_t cols, void *stream);
/* dY = scale (Y - T); *loss += sum (Y - T)^2. */
JB_API int jb_mse_grad(const float *Y, const float *T, float *dY, float *loss, int64_t n,
                       float scale, void *stream);
/* Adam step on a rows x cols parameter; refreshes its bf16 copy and (when
 * wT_bf16 is given) its bf16 transpose. */
JB_API int jb_adam(float *w, const float *g, float *m, float *v, void *w_bf16, void *wT_bf16,
                   int64_t rows, int64_t cols, float lr, float beta1, float beta2, float eps,
                   int32_t step, void *stream);
/* X[z] = upper triangle (i <= j, row-major) of A^T A / ||A||_F^2 as bf16, for
 * batch row-major m x n float32 matrices (the network's input sketch). */
JB_API int jb_gram_sketch(const float *A, void *X, int64_t batch, int32_t m, int32_t n, void *stream);

/* ---- blocked one-sided Jacobi (large matrices) ---------------------------
 * Building blocks of block_jacobi (svdbench/standalone/solvers.py:30-68) on
 * the tensor cores: block-pair Grams and rotations run on jb_gemm_bf16x, the
 * rest on these kernels (jb_block.cu). */

/* FP64 eigen-solve of `pairs` symmetric n x n FP32 Grams G[k] (n even): the
 * one-sided Jacobi rotations of the slot's columns applied to its Gram
 * (G <- J^T G J, relative threshold tol, at most max_sweeps sweeps; slots
 * of n = 64 and 128 use the odd-even pair order with registers-resident G,
 * others the round-robin order).  Writes vv^T (rows = eigenvectors,
 * eigenvalues descending: the inner solve's V of solvers.py:48) as hi/lo
 * BF16 (and a third part when Qt_lo2 is given), the largest pair ratio
 * |g_pq| / sqrt(g_pp g_qq) of the first sweep over live columns (g_pp, g_qq
 * > *live_floor, a device double, 0 when NULL: the reference checks only
 * those, solvers.py:55-57) (off), the slot's largest diagonal entry (dmax)
 * and the sweeps used.  The floor is read on the device so that a captured
 * CUDA graph of a whole sweep can be replayed with a new floor. */
JB_API int jb_block_eig_f64(const float *G, void *Qt_hi, void *Qt_lo, void *Qt_lo2, float *off,
                            float *dmax, int32_t *sweeps, int64_t pairs, int32_t n, int32_t max_sweeps,
                            double tol, const double *live_floor, void *stream);
/* jb_block_eig_f64 with the kernel chosen: variant 0 = automatic (as
 * jb_block_eig_f64), 1 = the shared-memory round-robin kernel (any even
 * width up to 256), 4 / 8 / 16 = one CTA per slot with G and Q in registers
 * (slot widths 64 and 128, odd-even order), that many columns per warp
 * (n / variant warps; the same outputs, a different latency / occupancy
 * balance, chosen by the blocked solver's autotuner).  Adding JB_EIG_FP32 to
 * a register variant (or to 0) rotates G in FP32 instead of FP64: for the
 * sweeps whose Gram is itself only ~16-bit accurate (two-part operands). */
#define JB_EIG_FP32 128

/* jb_block_eig_f64_ex with a workspace, for JB_EIG_DEFER_Q: the register
 * eigen-solve records its rotations instead of accumulating Q, and a second
 * kernel forms Q^T from them, one warp per row of Q over the whole GPU (the
 * eigen-solve itself then issues fewer instructions per round on its one SM
 * per slot).  The same Q^T to FP32 rounding.  Register variants only (slot
 * widths 64 and 128).  Workspace: jb_block_eig_workspace_bytes(pairs, n,
 * max_sweeps) bytes (8 max_sweeps n^2 + 4 n per slot, rounded). */
#define JB_EIG_DEFER_Q 256
JB_API size_t jb_block_eig_workspace_bytes(int64_t pairs, int32_t n, int32_t max_sweeps);
JB_API int jb_block_eig_ws(const float *G, void *Qt_hi, void *Qt_lo, void *Qt_lo2, float *off, float *dmax,
                           int32_t *sweeps, int64_t pairs, int32_t n, int32_t max_sweeps, double tol,
                           const double *live_floor, int32_t variant, void *workspace, size_t workspace_bytes,
                           void *stream);
JB_API int jb_block_eig_f64_ex(const float *G, void *Qt_hi, void *Qt_lo, void *Qt_lo2, float *off, float *dmax,
                               int32_t *sweeps, int64_t pairs, int32_t n, int32_t max_sweeps, double tol,
                               const double *live_floor, int32_t variant, void *stream);

/* Row r of src (rows x L, FP32) -> row map[r] (identity when NULL) of the
 * BF16 parts hi, lo, lo2 (a two- or three-part split; any may be NULL)
 * and/or an FP32 destination. */
JB_API int jb_rows_scatter(const float *src, const int32_t *map, void *hi, void *lo, void *lo2,
                           float *f32, int64_t rows, int64_t L, void *stream);

/* Row r of hi (+ lo (+ lo2)) BF16 -> row map[r] of dst (FP32). */
JB_API int jb_rows_combine(const void *hi, const void *lo, const void *lo2, const int32_t *map,
                           float *dst, int64_t rows, int64_t L, void *stream);

/* C (M x N, f32) = A (M x K) B (N x K)^T, FP32 inputs (row-major, K
 * contiguous) with FP64 accumulation on the CUDA cores: recomputes W = A V
 * from the exact input at the end of the blocked solve. */
JB_API int jb_gemm_f64acc(const float *A, const float *B, float *C, int64_t M, int64_t N, int64_t K,
                          int64_t lda, int64_t ldb, int64_t ldc, void *stream);

/* Final step: sigma_j = ||Wt row j|| (FP64), stable descending order perm,
 * S[r] = sigma * 2^e or 0 below eps32 * cut_width * sigma_1, U (m x rank,
 * row-major) = W[:, perm] / sigma, Vh (rank x n) = Vt[perm, :].  sig (n
 * doubles) and perm (n ints) are device scratch. */
JB_API int jb_block_finish(const float *Wt, const float *Vt, float *U, float *S, float *Vh, double *sig,
                           int32_t *perm, int64_t m, int64_t n, int32_t rank, int32_t e,
                           int32_t cut_width, void *stream);

/* ---- symmetric eigen-solver ----------------------------------------------
 * Batched two-sided cyclic Jacobi for real symmetric n x n matrices (n <=
 * 255): svdbench/standalone/primitives.py:370-427 (jacobi_eigh, the syevj
 * structure) for real dtypes.  H: batch x n x n row-major (symmetrised as
 * (H + H^T) / 2).  W: batch x n eigenvalues ascending; V: batch x n x n
 * row-major, column j the eigenvector of W[j].  tol <= 0 selects 10 eps
 * of the dtype; a pair is active when |g_pq| > tol max|G|.  sweeps/status
 * (device int32, batch each; status JB_ST_OK or JB_ST_NOT_CONVERGED).
 * Computed in FP64 for both dtypes.  Workspace: jb_eigh_workspace_bytes
 * (0 when G and V fit in shared memory, n <= 118; above that V, and beyond
 * n = 166 also G, live in the workspace). */
JB_API size_t jb_eigh_workspace_bytes(int32_t n, int64_t batch);
JB_API int jb_eigh_f32(const float *H, float *W, float *V, int32_t *sweeps, int32_t *status,
                       int64_t batch, int32_t n, double tol, int32_t max_sweeps,
                       void *workspace, size_t workspace_bytes, void *stream);
JB_API int jb_eigh_f64(const double *H, double *W, double *V, int32_t *sweeps, int32_t *status,
                       int64_t batch, int32_t n, double tol, int32_t max_sweeps,
                       void *workspace, size_t workspace_bytes, void *stream);
/* The same for complex Hermitian H (complex64 / complex128, interleaved re,
 * im), computed in complex128: the reference's complex branch of jacobi_eigh
 * (primitives.py:393-421, s = t c g_pq / |g_pq|, G <- J^H G J).  W real
 * (batch, n) ascending, V complex (batch, n, n).  Workspace:
 * jb_eigh_complex_workspace_bytes (0 while G and V fit in shared memory). */
JB_API size_t jb_eigh_complex_workspace_bytes(int32_t n, int64_t batch);
JB_API int jb_eigh_c64(const void *H, float *W, void *V, int32_t *sweeps, int32_t *status,
                       int64_t batch, int32_t n, double tol, int32_t max_sweeps,
                       void *workspace, size_t workspace_bytes, void *stream);
JB_API int jb_eigh_c128(const void *H, double *W, void *V, int32_t *sweeps, int32_t *status,
                        int64_t batch, int32_t n, double tol, int32_t max_sweeps,
                        void *workspace, size_t workspace_bytes, void *stream);

/* Batched Householder QR of tall matrices (m >= n): replaces the reference's
 * primitives.qr, svdbench/standalone/primitives.py:74-89 (reflectors by
 * householder_vec :41-59, the LAPACK xLARFG convention; Q by backward
 * accumulation), the QR of its 'qr', 'tsqr' and projected solvers
 * (solvers.py:71-96, 185-220, 245-248).  A (batch, m, n) row-major in;
 * Q (batch, m, n) and R (batch, n, n, upper triangular, real diagonal)
 * row-major out; computed in the input type; _c64 / _c128 take interleaved
 * complex.  Workspace: jb_qr_workspace_bytes with elem the element size (4,
 * 8 for float64 and complex64, 16 for complex128; 0 when a matrix and its Q
 * fit in shared memory). */
JB_API size_t jb_qr_workspace_bytes(int32_t m, int32_t n, int64_t batch, int32_t elem);
JB_API int jb_qr_f32(const float *A, float *Q, float *R, int64_t batch, int32_t m, int32_t n,
                     void *workspace, size_t workspace_bytes, void *stream);
JB_API int jb_qr_f64(const double *A, double *Q, double *R, int64_t batch, int32_t m, int32_t n,
                     void *workspace, size_t workspace_bytes, void *stream);
JB_API int jb_qr_c64(const void *A, void *Q, void *R, int64_t batch, int32_t m, int32_t n,
                     void *workspace, size_t workspace_bytes, void *stream);
JB_API int jb_qr_c128(const void *A, void *Q, void *R, int64_t batch, int32_t m, int32_t n,
                      void *workspace, size_t workspace_bytes, void *stream);

/* Batched one-sided Jacobi SVD of complex matrices: replaces the reference's
 * jacobi_svd for complex64 / complex128 (svdbench/standalone/primitives.py:
 * 316-367, with the phase-aware rotation s = t c apq / |apq| of :345-351),
 * in its round-robin order and input precision.  A (batch, m, n), m >= n
 * (a wide matrix is solved through its conjugate transpose by the caller),
 * interleaved (re, im), row-major; U (batch, m, n) with zero columns where
 * sigma is cut (the caller completes them), S (batch, n) real, descending,
 * 0 where cut; Vh (batch, n, n).  Workspace: jb_svd_complex_workspace_bytes
 * (elem = 8 for complex64, 16 for complex128; 0 when W and V fit in
 * shared memory). */
JB_API size_t jb_svd_complex_workspace_bytes(int32_t m, int32_t n, int64_t batch, int32_t elem);
JB_API int jb_svd_batched_c64(const void *A, void *U, float *S, void *Vh, int64_t batch, int32_t m, int32_t n,
                              double tol, int32_t max_sweeps, int32_t *sweeps, int32_t *status,
                              void *workspace, size_t workspace_bytes, void *stream);
JB_API int jb_svd_batched_c128(const void *A, void *U, double *S, void *Vh, int64_t batch, int32_t m, int32_t n,
                               double tol, int32_t max_sweeps, int32_t *sweeps, int32_t *status,
                               void *workspace, size_t workspace_bytes, void *stream);

/* Rounds [round_begin, round_end) of one-sided Jacobi sweeps applied in place
 * to ONE matrix: replaces the laboratory's jacobi_rotation over its schedule
 * (algorithm_laboratory/algorithms.py:81-102, 121-126: the round-robin
 * tournament on n + n % 2 players without the pairs past n), so that its
 * jacobi (:105-157) can run on the GPU while its trace sees W and V after
 * every sweep or round.  W (m x n, m >= n) and V (n x n) row-major device
 * arrays of dtype 0 float32, 1 float64, 2 complex64, 3 complex128
 * (interleaved re, im); n <= 8192; 0 <= round_begin <= round_end <= n + n % 2
 * - 1; tol > 0.  *off (a device double) becomes max(*off, the largest ratio
 * of an active pair in these rounds). */
JB_API int jb_jacobi_rounds(void *W, void *V, int32_t dtype, int32_t m, int32_t n, int32_t round_begin,
                            int32_t round_end, double tol, double *off, void *stream);

/* Null-space completion of U, svdbench/standalone/primitives.py:430-455
 * (complete_null_columns; complete_basis :458-467 and _finish_columns,
 * solvers.py:18-21, call it).  U: batch x m x n row-major device array of
 * dtype 0 float32, 1 float64, 2 complex64, 3 complex128 (interleaved);
 * keep: batch x n bytes (nonzero = keep the column).  In place, in
 * ascending column order, every column not kept becomes the coordinate
 * vector of largest leftover leverage 1 - sum_c |u_ic|^2, projected out
 * against the kept and already completed columns, normalised; a projected
 * length below 10 eps of the dtype sets status[z] = JB_ST_NULL_FAILED
 * (primitives.py:451-452).  status[z] is written for every matrix.
 * n <= 8192; workspace of jb_complete_null_workspace_bytes bytes. */
JB_API size_t jb_complete_null_workspace_bytes(int32_t dtype, int64_t batch, int64_t m, int64_t n);
JB_API int jb_complete_null(void *U, const uint8_t *keep, int32_t dtype, int64_t batch, int64_t m, int64_t n,
                            int32_t *status, void *workspace, size_t workspace_bytes, void *stream);

/* Measurement kernel for the rooflines of the FP32/FP64 Jacobi kernels (no
 * counterpart in the reference): `blocks` CTAs of 256 threads, each thread
 * 16 independent fused multiply-add chains of `iters` steps; mode 0 FP32
 * (fma.rn.f32), 1 packed FP32 (fma.rn.f32x2), 2 FP64.  jb_fma_loop_flops
 * gives the launch's flops (2 per multiply-add) for timing it. */
JB_API double jb_fma_loop_flops(int32_t blocks, int32_t iters);
JB_API int jb_fma_loop(int32_t mode, int32_t blocks, int32_t iters, float *sink, void *stream);

/* Size of the fixed device scratch array of jb_svd_batched_f32_noalloc. */
#define JB_NOALLOC_SCRATCH_BYTES (16u << 20)

/* jb_svd_batched_f32 without a workspace argument: allocates nothing.
 * No counterpart in the reference (its Python solver always allocates); this
 * is for callers that cannot allocate device memory when they solve: plug-ins
 * whose host framework owns every device allocation through its own pool,
 * and latency-bound paths that must not call cudaMalloc/cudaFree (which can
 * synchronise the whole device).
 *   - Scratch is one file-scope __device__ array of JB_NOALLOC_SCRATCH_BYTES
 *     (16 MiB) that every GPU loading the library keeps until process exit.
 *   - The limit: a call runs exactly when
 *     jb_workspace_bytes(m, n, batch, 4, precision, flags) <=
 *     JB_NOALLOC_SCRATCH_BYTES, and returns JB_ETOOBIG otherwise; callers can
 *     query that before calling.  For shapes of the register kernels (tall
 *     view up to 128 x 64) that is about 256 bytes plus, with JB_PREC_MIXED,
 *     4*batch*min(m,n)^2 bytes (e.g. at most 1023 matrices of 64 columns);
 *     larger shapes also need per-CTA work areas (about one per SM).
 *   - The first call on a device looks up the array's device address
 *     (cudaGetSymbolAddress) and caches it; make that first call before any
 *     stream capture.
 *   - All calls share the array: calls that overlap on the GPU (other
 *     streams, other host threads) race and corrupt each other's results;
 *     serialise them.  Work tickets are cleared on the stream by each call.
 * Other arguments and results: as jb_svd_batched_f32. */
JB_API int jb_svd_batched_f32_noalloc(const float *A, float *U, float *S, float *Vh,
                                      int64_t batch, int32_t m, int32_t n, int32_t rank,
                                      int32_t flags, double tol, int32_t max_sweeps,
                                      int32_t precision, int32_t *sweeps, int32_t *status,
                                      void *stream);

#ifdef __cplusplus
}
#endif

#endif /* JACOBI_B200_H */
