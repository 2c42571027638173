/* jacobi_oracle.c - CPU oracle: C restatement of the reference one-sided
 * Jacobi SVD path of uncle-Slava/Pavel-s_SVD (svdbench/standalone).
 *
 * TEST INFRASTRUCTURE ONLY.  Loaded (ctypes) by tests/, by
 * __graft_entry__.smoke() as the checker, and by bench.py as the timed CPU
 * baseline ("port") and the --impl reference arm.  The product library
 * (pavel-s_svd_b200) never links or calls it.
 *
 * Same buffer layout and status words as include/jacobi_b200.h, so tests
 * compare the two entry points argument for argument.  Matrices of a batch
 * are independent and run on `threads` POSIX threads (<= 0: one per online
 * CPU) that take matrices from an atomic counter.  Arithmetic follows the
 * reference: division by max|a| in the input precision (solvers.py:294-295),
 * sums accumulated in the input precision.
 */
#include <math.h>
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>
#include "jacobi_b200.h"

#define REAL float
#define SUF _f32
#define EPS 1.1920928955078125e-07f
#define TINY 1.1754943508222875e-38f
#include "jacobi_oracle_impl.h"
#undef REAL
#undef SUF
#undef EPS
#undef TINY

#define REAL double
#define SUF _f64
#define EPS 2.220446049250313e-16
#define TINY 2.2250738585072014e-308
#include "jacobi_oracle_impl.h"
#undef REAL
#undef SUF
#undef EPS
#undef TINY

#define API __attribute__((visibility("default")))

API int jo_version(void) { return 100; }

API int jo_max_threads(void) {
    long n = sysconf(_SC_NPROCESSORS_ONLN);
    return n > 0 ? (int)n : 1;
}

/* One job: `count` matrices described either uniformly or by descriptors. */
typedef struct {
    int dbl;
    const void *A;
    void *U, *S, *Vh;
    const jb_matrix_desc *descs;
    int64_t count;
    int32_t m, n, rank, flags;
    double tol;
    int32_t max_sweeps;
    int32_t *sweeps, *status;
    int64_t next;  /* atomic ticket */
} job_t;

static jb_matrix_desc job_desc(const job_t *j, int64_t b) {
    jb_matrix_desc d;
    if (j->descs) return j->descs[b];
    d.m = j->m; d.n = j->n; d.rank = j->rank; d.flags = j->flags;
    d.a_off = b * (int64_t)j->m * j->n;
    d.u_off = b * (int64_t)j->m * ((j->flags & JB_FULL_MATRICES) ? j->m : j->rank);
    d.s_off = b * (int64_t)j->rank;
    d.v_off = b * (int64_t)j->n * ((j->flags & JB_FULL_MATRICES) ? j->n : j->rank);
    return d;
}

static void *worker(void *arg) {
    job_t *j = (job_t *)arg;
    for (;;) {
        const int64_t b = __atomic_fetch_add(&j->next, 1, __ATOMIC_RELAXED);
        jb_matrix_desc d;
        int sw = 0, st;
        if (b >= j->count) break;
        d = job_desc(j, b);
        if (j->dbl) {
            const double *A = (const double *)j->A;
            double *U = (double *)j->U, *S = (double *)j->S, *Vh = (double *)j->Vh;
            st = solve_one__f64(A + d.a_off, d.m, d.n, d.rank, d.flags, j->tol, j->max_sweeps,
                                U ? U + d.u_off : NULL, S + d.s_off, Vh ? Vh + d.v_off : NULL, &sw);
        } else {
            const float *A = (const float *)j->A;
            float *U = (float *)j->U, *S = (float *)j->S, *Vh = (float *)j->Vh;
            st = solve_one__f32(A + d.a_off, d.m, d.n, d.rank, d.flags, j->tol, j->max_sweeps,
                                U ? U + d.u_off : NULL, S + d.s_off, Vh ? Vh + d.v_off : NULL, &sw);
        }
        j->status[b] = st;
        j->sweeps[b] = sw;
    }
    return NULL;
}

static int run_job(job_t *j, int threads) {
    pthread_t tid[256];
    int t, started = 0;
    if (threads <= 0) threads = jo_max_threads();
    if (threads > 256) threads = 256;
    if (threads > j->count) threads = (int)(j->count > 0 ? j->count : 1);
    j->next = 0;
    for (t = 1; t < threads; ++t)
        if (pthread_create(&tid[started], NULL, worker, j) == 0) ++started;
    worker(j);
    for (t = 0; t < started; ++t) pthread_join(tid[t], NULL);
    return JB_OK;
}

static int check_uniform(int64_t batch, int32_t m, int32_t n, int32_t rank, int32_t flags, int32_t max_sweeps) {
    const int k = m < n ? m : n;
    if (batch < 0 || m < 1 || n < 1 || rank < 1 || rank > k || max_sweeps < 1) return JB_EINVAL;
    if ((flags & JB_FULL_MATRICES) && rank != k) return JB_EINVAL;
    return JB_OK;
}

API int jo_svd_batched_f32(const float *A, float *U, float *S, float *Vh, int64_t batch, int32_t m, int32_t n,
                           int32_t rank, int32_t flags, double tol, int32_t max_sweeps, int32_t *sweeps,
                           int32_t *status, int32_t threads) {
    job_t j;
    int rc = check_uniform(batch, m, n, rank, flags, max_sweeps);
    if (rc) return rc;
    memset(&j, 0, sizeof(j));
    j.A = A; j.U = (flags & JB_VALUES_ONLY) ? NULL : U; j.S = S; j.Vh = (flags & JB_VALUES_ONLY) ? NULL : Vh;
    j.count = batch; j.m = m; j.n = n; j.rank = rank; j.flags = flags;
    j.tol = tol; j.max_sweeps = max_sweeps; j.sweeps = sweeps; j.status = status;
    return run_job(&j, threads);
}

API int jo_svd_batched_f64(const double *A, double *U, double *S, double *Vh, int64_t batch, int32_t m,
                           int32_t n, int32_t rank, int32_t flags, double tol, int32_t max_sweeps,
                           int32_t *sweeps, int32_t *status, int32_t threads) {
    job_t j;
    int rc = check_uniform(batch, m, n, rank, flags, max_sweeps);
    if (rc) return rc;
    memset(&j, 0, sizeof(j));
    j.dbl = 1;
    j.A = A; j.U = (flags & JB_VALUES_ONLY) ? NULL : U; j.S = S; j.Vh = (flags & JB_VALUES_ONLY) ? NULL : Vh;
    j.count = batch; j.m = m; j.n = n; j.rank = rank; j.flags = flags;
    j.tol = tol; j.max_sweeps = max_sweeps; j.sweeps = sweeps; j.status = status;
    return run_job(&j, threads);
}

/* Uneven batch with the descriptors of include/jacobi_b200.h (host memory). */
API int jo_svd_uneven_f32(const float *A, float *U, float *S, float *Vh, const jb_matrix_desc *descs,
                          int64_t count, double tol, int32_t max_sweeps, int32_t *sweeps, int32_t *status,
                          int32_t threads) {
    job_t j;
    if (count < 0 || max_sweeps < 1 || !descs) return JB_EINVAL;
    memset(&j, 0, sizeof(j));
    j.A = A; j.U = U; j.S = S; j.Vh = Vh; j.descs = descs; j.count = count;
    j.tol = tol; j.max_sweeps = max_sweeps; j.sweeps = sweeps; j.status = status;
    return run_job(&j, threads);
}
