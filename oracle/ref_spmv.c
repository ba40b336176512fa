/*
 * C entries around the reference's own SpMV kernels, compiled from its
 * sources (src/library/kernels/csrmv_adaptive.cl, csrmv_general.cl) through
 * oracle/clc_extract.py and oracle/clc_shim.h by oracle/Makefile into
 * oracle/_ref/librefspmv.so. Test infrastructure only: the tests use them to
 * pin the oracle's SpMV restatement and the library's kernels to what the
 * reference's kernels compute.
 *
 * One object per kernel build configuration, selected by -D flags as the
 * reference's host code sets them (csrmv-adaptive.hpp:38-87,
 * csrmv-vector.hpp:34-83): VALUE_TYPE, DOUBLE, EXTENDED_PRECISION, and for
 * csrmv_general SUBWAVE_SIZE. TAG names the exported function.
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

#ifdef ADAPTIVE
typedef struct {
    const VALUE_TYPE *vals;
    const unsigned *cols, *rp;
    const VALUE_TYPE *x;
    VALUE_TYPE *y;
    unsigned long *row_blocks;
    const VALUE_TYPE *alpha, *beta;
} adaptive_args;

static void adaptive_body(void *p)
{
    adaptive_args *a = (adaptive_args *)p;
    csrmv_adaptive(a->vals, a->cols, a->rp, a->x, a->y, a->row_blocks, a->alpha, a->beta);
}

/* y = alpha*A*x + beta*y by the reference's csrmv_adaptive. row_blocks holds
 * the reference's meta buffer: the words of ComputeRowBlocks in its first
 * row_block_size / 2 entries and room for row_block_size entries in all (the
 * second half carries the extended-precision long-row errors); the kernel
 * flips flag bits in it as the reference's does. vals and cols must stay
 * readable BLOCKSIZE entries past the last nonzero (the kernel's unguarded
 * stream loads, csrmv_adaptive.cl:413-416). Launch:
 * (row_block_size / 2 - 1) work-groups of WG_SIZE (csrmv-adaptive.hpp:108). */
int CLC_CAT(ref_csrmv_adaptive_, TAG)(const VALUE_TYPE *vals, const unsigned *cols, const unsigned *rp,
                                      const VALUE_TYPE *x, VALUE_TYPE *y, unsigned long *row_blocks,
                                      unsigned row_block_size, const VALUE_TYPE *alpha, const VALUE_TYPE *beta)
{
    adaptive_args a = {vals, cols, rp, x, y, row_blocks, alpha, beta};
    unsigned groups = row_block_size / 2 - 1;
    if (groups < 1) groups = 1;
    return clc_launch(groups, WG_SIZE, adaptive_body, &a);
}
#else
typedef struct {
    unsigned num_rows;
    const VALUE_TYPE *alpha;
    const unsigned *rp, *cols;
    const VALUE_TYPE *vals, *x, *beta;
    VALUE_TYPE *y;
} general_args;

static void general_body(void *p)
{
    general_args *a = (general_args *)p;
    csrmv_general(a->num_rows, a->alpha, 0, a->rp, a->cols, a->vals, a->x, 0, a->beta, 0, a->y, 0);
}

/* y = alpha*A*x + beta*y by the reference's csrmv_general with this build's
 * SUBWAVE_SIZE; the launch covers SUBWAVE_SIZE * num_rows work-items rounded
 * up to whole groups of WG_SIZE (csrmv-vector.hpp:101-110). */
int CLC_CAT(ref_csrmv_general_, TAG)(unsigned num_rows, const unsigned *rp, const unsigned *cols,
                                     const VALUE_TYPE *vals, const VALUE_TYPE *x, VALUE_TYPE *y,
                                     const VALUE_TYPE *alpha, const VALUE_TYPE *beta)
{
    general_args a = {num_rows, alpha, rp, cols, vals, x, beta, y};
    const unsigned long predicted = (unsigned long)SUBWAVE_SIZE * num_rows;
    unsigned long groups = (predicted + WG_SIZE - 1) / WG_SIZE;
    if (groups < 1) groups = 1;
    return clc_launch((unsigned)groups, WG_SIZE, general_body, &a);
}
#endif
