/* jacobi_oracle_impl.h - body of the C oracle, instantiated for one real type.
 *
 * TEST INFRASTRUCTURE ONLY (see jacobi_oracle.c).  Included twice by
 * jacobi_oracle.c with REAL/SUF/EPS/TINY defined.  Every step restates
 * uncle-Slava/Pavel-s_SVD svdbench/standalone/primitives.py and solvers.py;
 * the line numbers are given at each step.  One matrix at a time: the
 * reference's lock-step batch gives each member the same arithmetic, because a
 * member whose pairs are all below tol is not rotated again.
 */

#define CAT_(a, b) a##b
#define CAT(a, b) CAT_(a, b)
#define FN(name) CAT(name, SUF)

/* Circle-method pair k of round r on np players (primitives.py:309-313). */
static void FN(rr_pair_)(int r, int k, int np, int *p, int *q) {
    int a, b;
    a = k == 0 ? 0 : 1 + (((k - 1 - r) % (np - 1)) + (np - 1)) % (np - 1);
    {
        int pos = np - 1 - k;
        b = pos == 0 ? 0 : 1 + (((pos - 1 - r) % (np - 1)) + (np - 1)) % (np - 1);
    }
    *p = a < b ? a : b;
    *q = a < b ? b : a;
}

/* One-sided Jacobi sweeps on W (m x np, column-major) and V (np x np):
 * primitives.py:324-355.  Returns 1 when off <= tol was reached. */
static int FN(sweeps_)(REAL *W, REAL *V, int m, int np, REAL tol, int max_sweeps, int *out_sweeps,
                       REAL *app, REAL *aqq, REAL *apq) {
    const int npairs = np / 2;
    const REAL eps = EPS;
    int sweep;
    REAL off = 0;
    for (sweep = 1; sweep <= max_sweeps; ++sweep) {
        int r;
        off = 0;
        for (r = 0; r < np - 1; ++r) {
            int k;
            REAL rmax = 0;
            for (k = 0; k < npairs; ++k) {                       /* :331-333 */
                int p, q, i;
                REAL a = 0, b = 0, c = 0;
                const REAL *wp, *wq;
                FN(rr_pair_)(r, k, np, &p, &q);
                wp = W + (size_t)p * m;
                wq = W + (size_t)q * m;
                for (i = 0; i < m; ++i) {
                    a += wp[i] * wp[i];
                    b += wq[i] * wq[i];
                    c += wp[i] * wq[i];
                }
                app[k] = a; aqq[k] = b; apq[k] = c;
                if ((a > b ? a : b) > rmax) rmax = a > b ? a : b;
            }
            for (k = 0; k < npairs; ++k) {
                int p, q, i;
                REAL den, ratio, floor_, aa, tau, t, cc, ss;
                REAL *wp, *wq, *vp, *vq;
                den = (REAL)sqrt(app[k]) * (REAL)sqrt(aqq[k]);                  /* :334 */
                ratio = (REAL)fabs(apq[k]) / (den > TINY ? den : TINY);         /* :335 */
                floor_ = eps * eps * rmax;                                      /* :337 */
                if (!(ratio > tol && (app[k] < aqq[k] ? app[k] : aqq[k]) > floor_))   /* :338 */
                    continue;                     /* c = 1, s = 0: no change (:346-347) */
                if (ratio > off) off = ratio;                                   /* :339 */
                aa = (REAL)fabs(apq[k]);                                        /* :340 */
                tau = (aqq[k] - app[k]) / (2 * aa);                             /* :341 */
                if (tau == 0) t = 1;                                            /* :343 */
                else t = (tau > 0 ? (REAL)1 : (REAL)-1) / ((REAL)fabs(tau) + (REAL)hypot(tau, 1));   /* :342 */
                cc = 1 / (REAL)sqrt(1 + t * t);                                 /* :344 */
                ss = t * cc * (apq[k] / aa);                                    /* :345 */
                FN(rr_pair_)(r, k, np, &p, &q);
                wp = W + (size_t)p * m; wq = W + (size_t)q * m;
                for (i = 0; i < m; ++i) {                                       /* :349 */
                    REAL x = wp[i], y = wq[i];
                    wp[i] = cc * x - ss * y;
                    wq[i] = ss * x + cc * y;
                }
                vp = V + (size_t)p * np; vq = V + (size_t)q * np;
                for (i = 0; i < np; ++i) {                                      /* :350-351 */
                    REAL x = vp[i], y = vq[i];
                    vp[i] = cc * x - ss * y;
                    vq[i] = ss * x + cc * y;
                }
            }
        }
        if (off <= tol) { *out_sweeps = sweep; return 1; }                      /* :352-353 */
    }
    *out_sweeps = max_sweeps;
    return 0;                                                                   /* :354-355 */
}

/* complete_null_columns (primitives.py:430-455) on u (m x k, column-major). */
static int FN(complete_null_)(REAL *u, int m, int k, const unsigned char *keep, REAL *v, REAL *y) {
    int j, all = 1;
    for (j = 0; j < k; ++j) all &= keep[j];
    if (all) return 0;                                                          /* :432 */
    for (j = 0; j < k; ++j)
        if (!keep[j]) memset(u + (size_t)j * m, 0, sizeof(REAL) * m);           /* :436 */
    for (j = 0; j < k; ++j) {
        int i, c, pass, idx = 0;
        REAL best = -1, len;
        if (keep[j]) continue;
        for (i = 0; i < m; ++i) {                                               /* :444-445 */
            REAL acc = 0, lev;
            for (c = 0; c < k; ++c) acc += u[(size_t)c * m + i] * u[(size_t)c * m + i];
            lev = 1 - acc;
            if (i == 0 || lev > best) { best = lev; idx = i; }
        }
        for (i = 0; i < m; ++i) v[i] = i == idx ? 1 : 0;                        /* :446-447 */
        for (pass = 0; pass < 2; ++pass) {                                      /* :448-449 */
            for (c = 0; c < k; ++c) {
                REAL acc = 0;
                for (i = 0; i < m; ++i) acc += u[(size_t)c * m + i] * v[i];
                y[c] = acc;
            }
            for (i = 0; i < m; ++i) {
                REAL acc = 0;
                for (c = 0; c < k; ++c) acc += u[(size_t)c * m + i] * y[c];
                v[i] -= acc;
            }
        }
        len = 0;
        for (i = 0; i < m; ++i) len += v[i] * v[i];
        len = (REAL)sqrt(len);                                                  /* :450 */
        if (len < 10 * EPS) return 1;                                           /* :451-452 */
        for (i = 0; i < m; ++i) u[(size_t)j * m + i] = v[i] / (len > TINY ? len : TINY);   /* :453-454 */
    }
    return 0;
}

/* svd(a, 'jacobi') of one real matrix (solvers.py:264-310 with _raw
 * :224-230, _jacobi :24-27, jacobi_svd primitives.py:316-367). */
static int FN(solve_one_)(const REAL *A, int m, int n, int rank, int flags, double tol_in, int max_sweeps,
                          REAL *U, REAL *S, REAL *Vh, int *out_sweeps) {
    const int wide = m < n;
    const int mt = wide ? n : m, nt = wide ? m : n;
    const int np = nt + (nt & 1);                                               /* :320-323 */
    const int full = (flags & JB_FULL_MATRICES) != 0;
    const int kcols = full ? mt : nt;
    REAL scale = 0, tol, cut, *W, *V, *app, *aqq, *apq, *sig, *v, *y, *Ut;
    int *perm, i, j, r, conv, st = JB_ST_OK;
    unsigned char *keep;
    *out_sweeps = 0;
    for (i = 0; i < m * n; ++i) {                                               /* solvers.py:291-292 */
        if (!isfinite(A[i])) return JB_ST_NONFINITE_IN;
        if ((REAL)fabs(A[i]) > scale) scale = (REAL)fabs(A[i]);
    }
    if (!(scale > 0)) scale = 1;                                                /* solvers.py:294-295 */
    W = (REAL *)calloc((size_t)mt * np, sizeof(REAL));
    V = (REAL *)calloc((size_t)np * np, sizeof(REAL));
    app = (REAL *)malloc(sizeof(REAL) * (3 * (np / 2) + np + 2 * (mt + np)));
    aqq = app + np / 2; apq = aqq + np / 2; sig = apq + np / 2; v = sig + np; y = v + mt + np;
    perm = (int *)malloc(sizeof(int) * np);
    keep = (unsigned char *)malloc(kcols + 1);
    Ut = (REAL *)calloc((size_t)mt * kcols, sizeof(REAL));
    for (i = 0; i < m; ++i)                                                     /* tall view of a / scale */
        for (j = 0; j < n; ++j) {
            REAL x = A[(size_t)i * n + j] / scale;
            if (wide) W[(size_t)i * mt + j] = x; else W[(size_t)j * mt + i] = x;
        }
    for (i = 0; i < np; ++i) V[(size_t)i * np + i] = 1;                          /* :324 */
    tol = tol_in > 0 ? (REAL)tol_in : 10 * EPS;                                  /* :325 */
    conv = FN(sweeps_)(W, V, mt, np, tol, max_sweeps, out_sweeps, app, aqq, apq);
    if (!conv) { st = JB_ST_NOT_CONVERGED; goto done; }
    for (j = 0; j < nt; ++j) {                                                  /* :356 */
        REAL acc = 0;
        for (i = 0; i < mt; ++i) acc += W[(size_t)j * mt + i] * W[(size_t)j * mt + i];
        sig[j] = (REAL)sqrt(acc);
    }
    for (j = 0; j < nt; ++j) {                                                  /* :359-361, stable */
        int rk = 0;
        for (i = 0; i < nt; ++i) rk += sig[i] > sig[j] || (sig[i] == sig[j] && i < j);
        perm[rk] = j;
    }
    cut = EPS * (REAL)(mt > np ? mt : np) * sig[perm[0]];                       /* :362 */
    for (r = 0; r < nt; ++r) {                                                  /* :363-364 */
        REAL s = sig[perm[r]];
        keep[r] = s > cut;
        for (i = 0; i < mt; ++i) Ut[(size_t)r * mt + i] = W[(size_t)perm[r] * mt + i] / (keep[r] ? s : 1);
    }
    if (FN(complete_null_)(Ut, mt, nt, keep, v, y)) { st = JB_ST_NULL_FAILED; goto done; }   /* :365 */
    if (full && kcols > nt) {                                                   /* complete_basis :458-467 */
        for (r = 0; r < kcols; ++r) keep[r] = r < nt;
        if (FN(complete_null_)(Ut, mt, kcols, keep, v, y)) { st = JB_ST_NULL_FAILED; goto done; }
    }
    for (r = 0; r < rank; ++r) {                                                /* :366, solvers.py:299 */
        REAL s = sig[perm[r]];
        S[r] = (s > cut ? s : 0) * scale;
        if (!isfinite(S[r])) st = JB_ST_NONFINITE_OUT;
    }
    if (!(flags & JB_VALUES_ONLY)) {
        const int ucols = full ? m : rank, vrows = full ? n : rank;
        for (i = 0; i < m; ++i)
            for (r = 0; r < ucols; ++r) {
                REAL x = wide ? V[(size_t)perm[r] * np + i] : Ut[(size_t)r * mt + i];
                U[(size_t)i * ucols + r] = x;
                if (!isfinite(x)) st = JB_ST_NONFINITE_OUT;
            }
        for (r = 0; r < vrows; ++r)                                             /* Vh = v^H (solvers.py:309) */
            for (i = 0; i < n; ++i) {
                REAL x = wide ? Ut[(size_t)r * mt + i] : V[(size_t)perm[r] * np + i];
                Vh[(size_t)r * n + i] = x;
                if (!isfinite(x)) st = JB_ST_NONFINITE_OUT;
            }
    }
done:
    free(W); free(V); free(app); free(perm); free(keep); free(Ut);
    return st;
}

#undef FN
#undef CAT
#undef CAT_
