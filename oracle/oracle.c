/*
 * CPU oracle for the clSPARSE hot path -- TEST INFRASTRUCTURE ONLY.
 *
 * This file restates, in plain C, the reference algorithms the B200 library
 * must reproduce. Only the tests, __graft_entry__.smoke() and bench.py's CPU
 * baseline may load it, and only as the checker or the timed CPU baseline;
 * the product library never calls it. Parity is pinned by
 * tests/golden/rowblocks_*.npz, produced by the reference's own
 * ComputeRowBlocks compiled from its sources (oracle/Makefile -> oracle/_ref/),
 * and, for the SpMV restatements, by tests/golden/spmv_ref.npz: the outputs
 * of the reference's own csrmv_adaptive / csrmv_general OpenCL kernels,
 * compiled from its sources and run on the host through oracle/clc_shim.h.
 * The CG / BiCGStab restatements are pinned by tests/golden/solvers_ref.npz:
 * runs of the reference's host solver code (its OpenCL runtime is not
 * buildable here, so oracle/ref_solvers.py issues the same kernel sequence)
 * over the reference's own SpMV, dot, reduce, blas1, transform and
 * diagonal-extraction kernels, compiled from its sources and run on the
 * host (oracle/_ref/librefblas1.so, librefspmv.so).
 *
 *   oracle_row_blocks  csr-meta.hpp:93-261 (ComputeRowBlocks, incl. the
 *                      trailing-block quirk) and :263-269 (size-only run)
 *   oracle_dcsrmv      src/tests/test-blas2.cpp:231-252 (y = beta*y first, then
 *                      a compensated TwoSum accumulation, :118-130)
 *   oracle_scsrmv      src/tests/test-blas2.cpp:146-163 (float products, double
 *                      accumulation)
 *   oracle_{d,s}cg     src/library/solvers/conjugate-gradients.hpp:47-228 with the
 *                      stop test of solvers/solver-control.hpp:47-64
 *   oracle_{d,s}bicgstab  src/library/solvers/biconjugate-gradients-stabilized.hpp:41-268
 *   oracle_dcsrmv_mt   the same SpMV split over a reused pool of host threads by
 *                      equal-nonzero row ranges (the CPU baseline bench.py times)
 *   oracle_dcg_mt      FP64 Jacobi-PCG in the order of conjugate-gradients.hpp on
 *                      the same thread pool, L2 stop test: reference solutions of
 *                      the large configurations
 */
#include <math.h>
#include <float.h>
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

/* ---------------------------------------------------------------- binning */

static uint64_t threads_for_rows(uint64_t nrows)
{
    /* 256 >> bit_length(nrows - 1), argument truncated to 32 bits
     * (csr-meta.hpp:52-68 with the GCC builtin branch). */
    uint32_t v = (uint32_t)(nrows - 1);
    uint32_t bits = 0;
    while (v) { bits++; v >>= 1; }
    return (uint64_t)(256u >> (bits & 31u));
}

/* Fills words (may be NULL: count only) and returns the reference's
 * rowBlockSize: 2 * words written, or 2 * counted blocks in the size-only run. */
uint32_t oracle_row_blocks(const uint32_t *rp, uint32_t n, uint32_t blk, uint32_t mult,
                           uint32_t rows_for_vector, uint64_t *words)
{
    const int fill = words != NULL;
    uint64_t *w = words;
    uint64_t count = 1;
    uint64_t sum = 0, i, last = 0;
    uint32_t run = 0; /* unsigned run length of rows > 128; 0xFFFFFFFF = just ended */
    if (fill) *w++ = 0;
    for (i = 1; i <= n; i++) {
        uint32_t len = rp[i] - rp[i - 1];
        sum += len;
        if (len > 128) run++;
        else if (run > 0) run = (len < 32) ? 0xFFFFFFFFu : run + 1;

        if (run == 1) {
            if (i - last > 1) {
                if (fill) {
                    *w = (i - 1) << 32;
                    if ((i - 1) - last > rows_for_vector) *(w - 1) |= threads_for_rows((i - 1) - last);
                    w++;
                }
                count++;
                last = i - 1;
                sum = len;
            }
        } else if (run == 0xFFFFFFFFu) {
            if (fill) {
                *w = (i - 1) << 32;
                if ((i - 1) - last > rows_for_vector) *(w - 1) |= threads_for_rows((i - 1) - last);
                w++;
            }
            count++;
            last = i - 1;
            sum = len;
            run = 0;
        }

        if (i - last == 1 && sum > blk) {
            int need = (int)ceil((double)len / (double)(mult * blk));
            if (need > (1 << 24)) need = 1 << 24;
            if (fill) {
                for (int k = 1; k < need; k++) *w++ = ((i - 1) << 32) | (uint64_t)k;
                *w++ = i << 32;
            }
            count += (uint64_t)need;
            last = i;
            sum = 0;
            run = 0;
        } else if (i - last > 1 && sum > blk) {
            i--;
            if (fill) {
                *w = i << 32;
                if (i - last > rows_for_vector) *(w - 1) |= threads_for_rows(i - last);
                w++;
            }
            count++;
            last = i;
            sum = 0;
            run = 0;
        } else if (sum == blk) {
            if (fill) {
                *w = i << 32;
                if (i - last > rows_for_vector) *(w - 1) |= threads_for_rows(i - last);
                w++;
            }
            count++;
            last = i;
            sum = 0;
            run = 0;
        }
    }
    if (fill && ((*(w - 1)) >> 32) != (uint64_t)n) {
        *w = (uint64_t)n << 32;
        if ((uint64_t)n - last > rows_for_vector) *(w - 1) |= threads_for_rows(i - last);
        w++;
    }
    count++;
    if (fill) return (uint32_t)(2 * (uint64_t)(w - words));
    return (uint32_t)(2 * count);
}

/* ------------------------------------------------------------------ SpMV */

static double two_sum(double a, double b, double *err)
{
    double s = a + b;
    double bp = s - a;
    *err += (a - (s - bp)) + (b - bp);
    return s;
}

/* y = alpha*A*x + beta*y, FP64, compensated (test-blas2.cpp:231-252). beta == 0
 * overwrites y (so NaN in y does not propagate), as the library does. */
void oracle_dcsrmv(uint32_t n, const uint32_t *rp, const uint32_t *col, const double *val,
                   double alpha, const double *x, double beta, double *y)
{
    for (uint32_t r = 0; r < n; r++) {
        double t = (beta == 0.0) ? 0.0 : y[r] * beta;
        double err = 0.0;
        for (uint32_t j = rp[r]; j < rp[r + 1]; j++) t = two_sum(t, alpha * val[j] * x[col[j]], &err);
        y[r] = t + err;
    }
}

/* y = alpha*A*x + beta*y, FP32 products accumulated in double (test-blas2.cpp:146-163). */
void oracle_scsrmv(uint32_t n, const uint32_t *rp, const uint32_t *col, const float *val,
                   float alpha, const float *x, float beta, float *y)
{
    for (uint32_t r = 0; r < n; r++) {
        float yb = (beta == 0.0f) ? 0.0f : y[r] * beta;
        double t = yb;
        for (uint32_t j = rp[r]; j < rp[r + 1]; j++) {
            float p = alpha * val[j];
            p = p * x[col[j]];
            t += p;
        }
        y[r] = (float)t;
    }
}

/* Sum of |alpha*a_ij*x_j| + |beta*y_i| per row: the scale the SpMV parity
 * tests measure errors against (robust to cancellation). */
void oracle_dcsrmv_absscale(uint32_t n, const uint32_t *rp, const uint32_t *col, const double *val,
                            double alpha, const double *x, double beta, const double *y, double *out)
{
    for (uint32_t r = 0; r < n; r++) {
        double t = (beta == 0.0) ? 0.0 : fabs(beta * y[r]);
        for (uint32_t j = rp[r]; j < rp[r + 1]; j++) t += fabs(alpha * val[j] * x[col[j]]);
        out[r] = t;
    }
}

/* ------------------------------------------------------ threaded baseline */

/* The CPU baseline's SpMV: rows split into equal-nonzero ranges over a pool of
 * host threads that is created once and reused by every call, so a timed call
 * holds only the SpMV itself (no thread start-up). The calling thread works on
 * the first range. Not thread-safe: one caller at a time. */

typedef struct {
    uint32_t r0, r1;
    const uint32_t *rp, *col;
    const double *val, *x;
    double alpha, beta;
    double *y;
} spmv_task;

static void spmv_rows(const spmv_task *t)
{
    for (uint32_t r = t->r0; r < t->r1; r++) {
        double s = 0.0;
        for (uint32_t j = t->rp[r]; j < t->rp[r + 1]; j++) s += t->alpha * t->val[j] * t->x[t->col[j]];
        t->y[r] = (t->beta == 0.0) ? s : s + t->beta * t->y[r];
    }
}

#define POOL_MAX 256
static int pool_size = 0; /* threads including the caller; 0 = no pool */
static pthread_t pool_tid[POOL_MAX];
static pthread_barrier_t pool_start, pool_done;
static spmv_task pool_task[POOL_MAX];
static volatile int pool_quit = 0;
typedef void (*pool_fn)(int k, void *ctx);
static pool_fn pool_job;
static void *pool_ctx;

static void *pool_worker(void *arg)
{
    const int k = (int)(intptr_t)arg;
    for (;;) {
        pthread_barrier_wait(&pool_start);
        if (pool_quit) break;
        pool_job(k, pool_ctx);
        pthread_barrier_wait(&pool_done);
    }
    return NULL;
}

static void pool_stop(void)
{
    if (pool_size <= 1) {
        pool_size = 0;
        return;
    }
    pool_quit = 1;
    pthread_barrier_wait(&pool_start);
    for (int k = 1; k < pool_size; k++) pthread_join(pool_tid[k], NULL);
    pthread_barrier_destroy(&pool_start);
    pthread_barrier_destroy(&pool_done);
    pool_quit = 0;
    pool_size = 0;
}

static void pool_resize(int threads)
{
    if (threads == pool_size) return;
    pool_stop();
    pool_size = threads;
    if (threads <= 1) return;
    pthread_barrier_init(&pool_start, NULL, (unsigned)threads);
    pthread_barrier_init(&pool_done, NULL, (unsigned)threads);
    for (int k = 1; k < threads; k++) pthread_create(&pool_tid[k], NULL, pool_worker, (void *)(intptr_t)k);
}

/* Runs job(k, ctx) for k in [0, pool_size) and returns when all are done;
 * the calling thread runs k = 0. */
static void pool_run(pool_fn job, void *ctx)
{
    pool_job = job;
    pool_ctx = ctx;
    if (pool_size > 1) pthread_barrier_wait(&pool_start);
    job(0, ctx);
    if (pool_size > 1) pthread_barrier_wait(&pool_done);
}

static void spmv_job(int k, void *ctx)
{
    (void)ctx;
    spmv_rows(&pool_task[k]);
}

/* First row r in [lo, n] with rp[r] >= target. */
static uint32_t first_row_at(const uint32_t *rp, uint32_t lo, uint32_t n, uint64_t target)
{
    uint32_t hi = n;
    while (lo < hi) {
        uint32_t mid = lo + (hi - lo) / 2;
        if ((uint64_t)rp[mid] < target) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

/* Row ranges of `parts` threads with equal nonzeros (bounds[0..parts]). */
static void nnz_ranges(const uint32_t *rp, uint32_t n, int parts, uint32_t *bounds)
{
    const uint64_t nnz = rp[n] - rp[0];
    bounds[0] = 0;
    for (int k = 0; k < parts; k++)
        bounds[k + 1] = (k == parts - 1) ? n
                        : first_row_at(rp, bounds[k], n, rp[0] + (nnz * (uint64_t)(k + 1)) / (uint64_t)parts);
}

/* FP64 SpMV over `threads` host threads (the pool is resized when the count
 * changes), rows split into equal-nonzero ranges by binary search. */
void oracle_dcsrmv_mt(uint32_t n, const uint32_t *rp, const uint32_t *col, const double *val,
                      double alpha, const double *x, double beta, double *y, int threads)
{
    if (threads < 1) threads = 1;
    if (threads > POOL_MAX) threads = POOL_MAX;
    pool_resize(threads);
    uint32_t bounds[POOL_MAX + 1];
    nnz_ranges(rp, n, threads, bounds);
    for (int k = 0; k < threads; k++)
        pool_task[k] = (spmv_task){bounds[k], bounds[k + 1], rp, col, val, x, alpha, beta, y};
    pool_run(spmv_job, NULL);
}

/* Ends the pool's threads (the next threaded call starts a new pool). */
void oracle_pool_shutdown(void)
{
    pool_stop();
}

/* Threaded FP64 Jacobi-PCG used to make reference solutions of the large
 * configurations (the serial oracle_dcg below is the parity oracle for
 * iteration counts). Operation order of conjugate-gradients.hpp:100-226:
 * r = b - A x, z = D^-1 r, p = z, then per iteration q = A p, alpha =
 * <r,z>/<p,q>, x += alpha p, r -= alpha q, z = D^-1 r, beta = <r,z>_new /
 * <r,z>, p = z + beta p; stopped on the L2 relative residual
 * ||r||_2 / ||b||_2 <= rel_tol (the stop test the mixed-precision solvers of
 * this library use). Rows without a diagonal entry keep z_i = r_i. Per-thread
 * partial sums are added in thread order, so a run is reproducible for a
 * given thread count. Returns the iterations. */
typedef struct {
    const uint32_t *rp, *col, *bounds;
    const double *val, *b, *dinv;
    double *x, *r, *z, *p, *q;
    double alpha, beta;
    int phase;
    double part[POOL_MAX][4];
} cg_mt_ctx;

static void cg_mt_job(int k, void *vctx)
{
    cg_mt_ctx *c = (cg_mt_ctx *)vctx;
    const uint32_t r0 = c->bounds[k], r1 = c->bounds[k + 1];
    double s0 = 0.0, s1 = 0.0, s2 = 0.0;
    for (uint32_t i = r0; i < r1; i++) {
        if (c->phase == 0) { /* r = b - A x; z = D^-1 r; p = z; <r,z>, <r,r>, <b,b> */
            double t = 0.0;
            for (uint32_t j = c->rp[i]; j < c->rp[i + 1]; j++) t += c->val[j] * c->x[c->col[j]];
            const double ri = c->b[i] - t;
            c->r[i] = ri;
            c->z[i] = c->dinv[i] * ri;
            c->p[i] = c->z[i];
            s0 += ri * c->z[i];
            s1 += ri * ri;
            s2 += c->b[i] * c->b[i];
        } else if (c->phase == 1) { /* q = A p; <p,q> */
            double t = 0.0;
            for (uint32_t j = c->rp[i]; j < c->rp[i + 1]; j++) t += c->val[j] * c->p[c->col[j]];
            c->q[i] = t;
            s0 += c->p[i] * t;
        } else if (c->phase == 2) { /* x, r, z updates; <r,z>, <r,r> */
            c->x[i] += c->alpha * c->p[i];
            const double ri = c->r[i] - c->alpha * c->q[i];
            c->r[i] = ri;
            c->z[i] = c->dinv[i] * ri;
            s0 += ri * c->z[i];
            s1 += ri * ri;
        } else { /* p = z + beta p */
            c->p[i] = c->z[i] + c->beta * c->p[i];
        }
    }
    c->part[k][0] = s0;
    c->part[k][1] = s1;
    c->part[k][2] = s2;
}

static void cg_mt_sum(const cg_mt_ctx *c, int parts, double *out)
{
    out[0] = out[1] = out[2] = 0.0;
    for (int k = 0; k < parts; k++) {
        out[0] += c->part[k][0];
        out[1] += c->part[k][1];
        out[2] += c->part[k][2];
    }
}

int oracle_dcg_mt(uint32_t n, const uint32_t *rp, const uint32_t *col, const double *val, double *x,
                  const double *b, int max_iters, double rel_tol, int threads, double *final_rel_res)
{
    if (threads < 1) threads = 1;
    if (threads > POOL_MAX) threads = POOL_MAX;
    pool_resize(threads);
    cg_mt_ctx *c = (cg_mt_ctx *)calloc(1, sizeof(cg_mt_ctx));
    uint32_t *bounds = (uint32_t *)malloc(sizeof(uint32_t) * (size_t)(threads + 1));
    double *work = (double *)malloc(sizeof(double) * (size_t)n * 5);
    double *dinv = work + 4 * (size_t)n;
    nnz_ranges(rp, n, threads, bounds);
    for (uint32_t i = 0; i < n; i++) { /* first matching diagonal entry */
        dinv[i] = 1.0;
        for (uint32_t j = rp[i]; j < rp[i + 1]; j++)
            if (col[j] == i) {
                dinv[i] = 1.0 / val[j];
                break;
            }
    }
    c->rp = rp;
    c->col = col;
    c->val = val;
    c->bounds = bounds;
    c->b = b;
    c->dinv = dinv;
    c->x = x;
    c->r = work;
    c->z = work + n;
    c->p = work + 2 * (size_t)n;
    c->q = work + 3 * (size_t)n;
    double s[3];
    c->phase = 0;
    pool_run(cg_mt_job, c);
    cg_mt_sum(c, threads, s);
    double rz = s[0];
    const double bn = sqrt(s[2]);
    double res = bn > 0.0 ? sqrt(s[1]) / bn : 0.0;
    int it = 0;
    while (bn > 0.0 && res > rel_tol && it < max_iters) {
        c->phase = 1;
        pool_run(cg_mt_job, c);
        cg_mt_sum(c, threads, s);
        c->alpha = rz / s[0];
        c->phase = 2;
        pool_run(cg_mt_job, c);
        cg_mt_sum(c, threads, s);
        res = sqrt(s[1]) / bn;
        c->beta = s[0] / rz;
        rz = s[0];
        it++;
        if (res <= rel_tol) break;
        c->phase = 3;
        pool_run(cg_mt_job, c);
    }
    if (final_rel_res) *final_rel_res = res;
    free(work);
    free(bounds);
    free(c);
    return it;
}

/* --------------------------------------------------------------- solvers */

/* Result block shared by the solver oracles. */
typedef struct {
    int nIters;
    int zero_b;
    double initialResidual;
    double currentResidual;
    double relTol, absTol; /* as left in the solver control after the solve */
} oracle_solve_info;

#define DEFINE_SOLVERS(T, SFX, TMIN)                                                              \
static void spmv_##SFX(uint32_t n, const uint32_t *rp, const uint32_t *col, const T *val,         \
                       const T *x, T *y)                                                          \
{                                                                                                 \
    for (uint32_t r = 0; r < n; r++) {                                                            \
        T s = 0;                                                                                  \
        for (uint32_t j = rp[r]; j < rp[r + 1]; j++) s += val[j] * x[col[j]];                     \
        y[r] = s;                                                                                 \
    }                                                                                             \
}                                                                                                 \
static T nrm1_##SFX(uint32_t n, const T *v)                                                       \
{                                                                                                 \
    double s = 0;                                                                                 \
    for (uint32_t i = 0; i < n; i++) s += fabs((double)v[i]);                                     \
    return (T)s;                                                                                  \
}                                                                                                 \
static T dot_##SFX(uint32_t n, const T *a, const T *b)                                            \
{                                                                                                 \
    double s = 0;                                                                                 \
    for (uint32_t i = 0; i < n; i++) s += (double)a[i] * (double)b[i];                            \
    return (T)s;                                                                                  \
}                                                                                                 \
static int finished_##SFX(double res, double rel, double abs_, double init, int nIters, int maxIt) \
{                                                                                                 \
    return res <= rel || res <= abs_ * init || nIters >= maxIt;                                   \
}                                                                                                 \
/* inverse diagonal, first matching entry; 0 where a row has none (matrix_utils.cl:80-96) */     \
static void invdiag_##SFX(uint32_t n, const uint32_t *rp, const uint32_t *col, const T *val, T *d) \
{                                                                                                 \
    for (uint32_t r = 0; r < n; r++) {                                                            \
        d[r] = 0;                                                                                 \
        for (uint32_t j = rp[r]; j < rp[r + 1]; j++)                                              \
            if (col[j] == r) { d[r] = (T)1 / val[j]; break; }                                     \
    }                                                                                             \
}                                                                                                 \
/* CG of conjugate-gradients.hpp:47-228. precond: 0 none, 1 Jacobi. nIters_in is                 \
 * the solver control's count before the solve (the initial stop test sees it). */              \
int oracle_##SFX##cg(uint32_t n, const uint32_t *rp, const uint32_t *col, const T *val, T *x,    \
                     const T *b, int precond, int maxIters, double relTol, double absTol,         \
                     int nIters_in, oracle_solve_info *info)                                      \
{                                                                                                 \
    memset(info, 0, sizeof(*info));                                                               \
    info->relTol = relTol; info->absTol = absTol; info->nIters = nIters_in;                       \
    T norm_b = nrm1_##SFX(n, b);                                                                  \
    if (norm_b == 0) {                                                                            \
        info->nIters = 0; info->zero_b = 1; info->relTol = 0; info->absTol = 0;                   \
        memcpy(x, b, sizeof(T) * n);                                                              \
        return 0;                                                                                 \
    }                                                                                             \
    T *y = calloc(n, sizeof(T)), *z = calloc(n, sizeof(T)), *r = calloc(n, sizeof(T));            \
    T *p = calloc(n, sizeof(T)), *d = calloc(n, sizeof(T));                                       \
    if (precond) invdiag_##SFX(n, rp, col, val, d);                                               \
    spmv_##SFX(n, rp, col, val, x, y);                                                            \
    for (uint32_t i = 0; i < n; i++) r[i] = b[i] - y[i];                                          \
    T norm_r = nrm1_##SFX(n, r);                                                                  \
    T res = norm_r / norm_b;                                                                      \
    info->initialResidual = (double)res;                                                          \
    info->currentResidual = (double)res;                                                          \
    if (finished_##SFX(info->initialResidual, relTol, absTol, info->initialResidual,              \
                       info->nIters, maxIters)) {                                                 \
        info->nIters = 0;                                                                         \
        goto done;                                                                                \
    }                                                                                             \
    for (uint32_t i = 0; i < n; i++) z[i] = precond ? r[i] * d[i] : r[i];                         \
    memcpy(p, z, sizeof(T) * n);                                                                  \
    T rz = dot_##SFX(n, r, z);                                                                    \
    int it = 0;                                                                                   \
    for (;;) {                                                                                    \
        info->nIters = it;                                                                        \
        spmv_##SFX(n, rp, col, val, p, y);                                                        \
        T yp = dot_##SFX(n, y, p);                                                                \
        T alpha = rz / yp;                                                                        \
        for (uint32_t i = 0; i < n; i++) x[i] = x[i] + alpha * p[i];                              \
        for (uint32_t i = 0; i < n; i++) r[i] = r[i] - alpha * y[i];                              \
        for (uint32_t i = 0; i < n; i++) z[i] = precond ? r[i] * d[i] : r[i];                     \
        T rz_old = rz;                                                                            \
        rz = dot_##SFX(n, r, z);                                                                  \
        T beta = rz / rz_old;                                                                     \
        for (uint32_t i = 0; i < n; i++) p[i] = z[i] + beta * p[i];                               \
        norm_r = nrm1_##SFX(n, r);                                                                \
        res = norm_r / norm_b;                                                                    \
        it++;                                                                                     \
        info->currentResidual = (double)res;                                                      \
        if (finished_##SFX((double)res, relTol, absTol, info->initialResidual, info->nIters,      \
                           maxIters))                                                             \
            break;                                                                                \
    }                                                                                             \
done:                                                                                             \
    free(y); free(z); free(r); free(p); free(d);                                                  \
    return 0;                                                                                     \
}                                                                                                 \
/* BiCGStab of biconjugate-gradients-stabilized.hpp:41-268. */                                    \
int oracle_##SFX##bicgstab(uint32_t n, const uint32_t *rp, const uint32_t *col, const T *val,    \
                           T *x, const T *b, int precond, int maxIters, double relTol,            \
                           double absTol, int nIters_in, oracle_solve_info *info)                 \
{                                                                                                 \
    memset(info, 0, sizeof(*info));                                                               \
    info->relTol = relTol; info->absTol = absTol; info->nIters = nIters_in;                       \
    T norm_b = nrm1_##SFX(n, b);                                                                  \
    if (norm_b <= TMIN) {                                                                         \
        info->nIters = 0; info->zero_b = 1; info->relTol = 0; info->absTol = 0;                   \
        memcpy(x, b, sizeof(T) * n);                                                              \
        return 0;                                                                                 \
    }                                                                                             \
    T *y = calloc(n, sizeof(T)), *p = calloc(n, sizeof(T)), *r = calloc(n, sizeof(T));            \
    T *rs = calloc(n, sizeof(T)), *s = calloc(n, sizeof(T)), *Mp = calloc(n, sizeof(T));          \
    T *AMp = calloc(n, sizeof(T)), *Ms = calloc(n, sizeof(T)), *AMs = calloc(n, sizeof(T));       \
    T *d = calloc(n, sizeof(T));                                                                  \
    if (precond) invdiag_##SFX(n, rp, col, val, d);                                               \
    spmv_##SFX(n, rp, col, val, x, y);                                                            \
    for (uint32_t i = 0; i < n; i++) r[i] = b[i] - y[i];                                          \
    T norm_r = nrm1_##SFX(n, r);                                                                  \
    T res = norm_r / norm_b;                                                                      \
    info->initialResidual = (double)res;                                                          \
    info->currentResidual = (double)res;                                                          \
    if (finished_##SFX(info->initialResidual, relTol, absTol, info->initialResidual,              \
                       info->nIters, maxIters)) {                                                 \
        info->nIters = 0;                                                                         \
        goto done;                                                                                \
    }                                                                                             \
    memcpy(p, r, sizeof(T) * n);                                                                  \
    memcpy(rs, r, sizeof(T) * n);                                                                 \
    T rsr_old = dot_##SFX(n, rs, r);                                                              \
    int it = 0;                                                                                   \
    for (;;) {                                                                                    \
        for (uint32_t i = 0; i < n; i++) Mp[i] = precond ? p[i] * d[i] : p[i];                    \
        spmv_##SFX(n, rp, col, val, Mp, AMp);                                                     \
        T rs_amp = dot_##SFX(n, rs, AMp);                                                         \
        T alpha = rsr_old / rs_amp;                                                               \
        for (uint32_t i = 0; i < n; i++) s[i] = r[i] - alpha * AMp[i];                            \
        T norm_s = nrm1_##SFX(n, s);                                                              \
        res = norm_s / norm_b;                                                                    \
        info->currentResidual = (double)res;                                                      \
        if (finished_##SFX((double)res, relTol, absTol, info->initialResidual, info->nIters,      \
                           maxIters)) {                                                           \
            info->nIters = it;                                                                    \
            for (uint32_t i = 0; i < n; i++) x[i] = x[i] + alpha * Mp[i];                         \
            break;                                                                                \
        }                                                                                         \
        for (uint32_t i = 0; i < n; i++) Ms[i] = precond ? s[i] * d[i] : s[i];                    \
        spmv_##SFX(n, rp, col, val, Ms, AMs);                                                     \
        T amss = dot_##SFX(n, AMs, s);                                                            \
        T amsams = dot_##SFX(n, AMs, AMs);                                                        \
        T omega = amss / amsams;                                                                  \
        for (uint32_t i = 0; i < n; i++) x[i] = x[i] + alpha * Mp[i];                             \
        for (uint32_t i = 0; i < n; i++) x[i] = x[i] + omega * Ms[i];                             \
        for (uint32_t i = 0; i < n; i++) r[i] = s[i] - omega * AMs[i];                            \
        norm_r = nrm1_##SFX(n, r);                                                                \
        res = norm_r / norm_b;                                                                    \
        info->currentResidual = (double)res;                                                      \
        if (finished_##SFX((double)res, relTol, absTol, info->initialResidual, info->nIters,      \
                           maxIters)) {                                                           \
            info->nIters = it;                                                                    \
            break;                                                                                \
        }                                                                                         \
        T rsr_new = dot_##SFX(n, rs, r);                                                          \
        T beta = rsr_new / rsr_old;                                                               \
        beta = beta * alpha;                                                                      \
        beta = beta / omega;                                                                      \
        rsr_old = rsr_new;                                                                        \
        for (uint32_t i = 0; i < n; i++) p[i] = r[i] + beta * p[i];                               \
        T bw = beta * omega;                                                                      \
        for (uint32_t i = 0; i < n; i++) p[i] = p[i] - bw * AMp[i];                               \
        it++;                                                                                     \
        info->nIters = it;                                                                        \
    }                                                                                             \
done:                                                                                             \
    free(y); free(p); free(r); free(rs); free(s); free(Mp); free(AMp); free(Ms); free(AMs);       \
    free(d);                                                                                      \
    return 0;                                                                                     \
}

DEFINE_SOLVERS(double, d, DBL_MIN)
DEFINE_SOLVERS(float, s, FLT_MIN)
