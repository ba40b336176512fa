/*
 * C entries around the reference's own BLAS-1 and preconditioner kernels
 * (src/library/kernels/dot.cl, reduce.cl, atomic_reduce.cl, blas1.cl,
 * elementwise_transform.cl, matrix_utils.cl), compiled from the reference
 * sources through oracle/clc_extract.py and oracle/clc_shim.h by
 * oracle/Makefile into oracle/_ref/librefblas1.so. Test infrastructure only:
 * oracle/ref_solvers.py drives them in the order of the reference's CG and
 * BiCGStab host code to make the solver fixtures the oracle and the library
 * are checked against.
 *
 * One object per kernel build configuration, selected by -D flags as the
 * reference's host code sets them: KIND picks the kernel file, VALUE_TYPE /
 * DOUBLE the precision, OP_* the operation, TAG the exported name. Launch
 * geometries are the host code's: 256 work-groups of 256 for the two-stage
 * reductions (cldense-dot.hpp:112-118, reduce.hpp:119-130), one group of 256
 * for their second stage (atomic-reduce.hpp:94-100), ceil(n / 256) groups of
 * 256 for the element-wise kernels (cldense-axpy.hpp:87-91,
 * elementwise-transform.hpp) and the diagonal extraction
 * (preconditioner_utils.hpp:118-124).
 */
#include <math.h>
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#pragma GCC visibility push(hidden)
#include "clc_shim.h"
#include KERNEL_INC
#pragma GCC visibility pop

#define CLC_CAT2(a, b) a##b
#define CLC_CAT(a, b) CLC_CAT2(a, b)

typedef unsigned int idx_t;

#if defined(KIND_DOT)
typedef struct { idx_t size; VALUE_TYPE *sum; const VALUE_TYPE *x, *y; } dot_args;
static void dot_body(void *p) { dot_args *a = (dot_args *)p; inner_product(a->size, a->sum, (VALUE_TYPE *)a->x, (VALUE_TYPE *)a->y); }
/* partial[256] = per-group sums of x .* y */
int CLC_CAT(ref_inner_product_, TAG)(idx_t size, VALUE_TYPE *partial, const VALUE_TYPE *x, const VALUE_TYPE *y)
{
    dot_args a = {size, partial, x, y};
    return clc_launch(REDUCE_BLOCKS_NUMBER, REDUCE_BLOCK_SIZE, dot_body, &a);
}
#elif defined(KIND_REDUCE)
typedef struct { idx_t size; const VALUE_TYPE *x; VALUE_TYPE *sum; } red_args;
static void red_body(void *p) { red_args *a = (red_args *)p; reduce(a->size, a->x, a->sum); }
int CLC_CAT(ref_global_reduce_, TAG)(idx_t size, const VALUE_TYPE *x, VALUE_TYPE *partial)
{
    red_args a = {size, x, partial};
    return clc_launch(REDUCE_BLOCKS_NUMBER, REDUCE_BLOCK_SIZE, red_body, &a);
}
#elif defined(KIND_ATOMIC)
typedef struct { VALUE_TYPE *sum; const VALUE_TYPE *x; } at_args;
static void at_body(void *p) { at_args *a = (at_args *)p; reduce_block(a->sum, a->x); }
/* *sum += x[0..WG_SIZE) (sum zeroed by the caller, as init_scalar does) */
int CLC_CAT(ref_atomic_reduce_, TAG)(VALUE_TYPE *sum, const VALUE_TYPE *x)
{
    at_args a = {sum, x};
    return clc_launch(1, WG_SIZE, at_body, &a);
}
#elif defined(KIND_TRANSFORM)
typedef struct { idx_t size; VALUE_TYPE *r; const VALUE_TYPE *x, *y; } tr_args;
static void tr_body(void *p) { tr_args *a = (tr_args *)p; transform(a->size, a->r, a->x, a->y); }
int CLC_CAT(ref_transform_, TAG)(idx_t size, VALUE_TYPE *r, const VALUE_TYPE *x, const VALUE_TYPE *y)
{
    tr_args a = {size, r, x, y};
    return clc_launch_seq((size + WG_SIZE - 1) / WG_SIZE, WG_SIZE, tr_body, &a);
}
#elif defined(KIND_BLAS1)
typedef struct { idx_t size; VALUE_TYPE *y; const VALUE_TYPE *alpha, *x, *beta, *z; } ax_args;
static void axpy_body(void *p)
{
    ax_args *a = (ax_args *)p;
    axpy(a->size, a->y, 0, a->alpha, 0, a->x, 0, a->z, 0);
}
static void axpby_body(void *p)
{
    ax_args *a = (ax_args *)p;
    axpby(a->size, a->y, 0, a->alpha, 0, a->x, 0, a->beta, 0, a->z, 0);
}
/* y = z OP alpha * x */
int CLC_CAT(ref_axpy_, TAG)(idx_t size, VALUE_TYPE *y, const VALUE_TYPE *alpha, const VALUE_TYPE *x,
                           const VALUE_TYPE *z)
{
    ax_args a = {size, y, alpha, x, 0, z};
    return clc_launch_seq((size + WG_SIZE - 1) / WG_SIZE, WG_SIZE, axpy_body, &a);
}
/* y = alpha * x OP beta * z */
int CLC_CAT(ref_axpby_, TAG)(idx_t size, VALUE_TYPE *y, const VALUE_TYPE *alpha, const VALUE_TYPE *x,
                            const VALUE_TYPE *beta, const VALUE_TYPE *z)
{
    ax_args a = {size, y, alpha, x, beta, z};
    return clc_launch_seq((size + WG_SIZE - 1) / WG_SIZE, WG_SIZE, axpby_body, &a);
}
#elif defined(KIND_DIAG)
typedef struct { idx_t n; VALUE_TYPE *diag; const idx_t *rp, *cols; const VALUE_TYPE *vals; } dg_args;
static void dg_body(void *p)
{
    dg_args *a = (dg_args *)p;
    extract_diagonal(a->n, a->diag, a->rp, a->cols, a->vals);
}
/* diag[row] = 1 / a_row,row (first match) for rows that have a diagonal entry */
int CLC_CAT(ref_extract_diag_inv_, TAG)(idx_t n, VALUE_TYPE *diag, const idx_t *rp, const idx_t *cols,
                                       const VALUE_TYPE *vals)
{
    dg_args a = {n, diag, rp, cols, vals};
    const unsigned long predicted = (unsigned long)SUBWAVE_SIZE * n;
    unsigned long groups = (predicted + WG_SIZE - 1) / WG_SIZE;
    if (groups < 1) groups = 1;
    return clc_launch_seq((unsigned)groups, WG_SIZE, dg_body, &a);
}
#endif
