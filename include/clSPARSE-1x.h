/*
 * clSPARSE-1x.h -- the data structs of the clSPARSE C ABI.
 *
 * Same struct names, field names, field order and field types as the
 * reference's src/include/clSPARSE-1x.h:31-143, so that code written against
 * the reference compiles unchanged. The cl_mem fields hold CUDA device
 * pointers owned by the caller; every off_* field is an offset in elements
 * that the library adds to the pointer (the reference's adaptive SpMV ignored
 * them, src/library/blas2/csrmv-adaptive.hpp:93-97; here they are honoured on
 * every path).
 */
#ifndef CLSPARSE_B200_1X_H_
#define CLSPARSE_B200_1X_H_

#include "clSPARSE-xx.h"

/* A single value in device memory (reference clSPARSE-1x.h:31-39). */
typedef struct clsparseScalar_
{
    cl_mem value;
    clsparseIdx_t off_value;
} clsparseScalar;

/* A dense vector in device memory (reference clSPARSE-1x.h:43-53). */
typedef struct cldenseVector_
{
    clsparseIdx_t num_values;
    cl_mem values;
    clsparseIdx_t off_values;
} cldenseVector;

/* A 0-based CSR matrix in device memory (reference clSPARSE-1x.h:60-90).
 * row_pointer has num_rows+1 entries, col_indices and values num_nonzeros.
 * meta is owned by the library (clsparseCsrMetaCreate / clsparseCsrMetaDelete). */
typedef struct clsparseCsrMatrix_
{
    clsparseIdx_t num_rows;
    clsparseIdx_t num_cols;
    clsparseIdx_t num_nonzeros;

    cl_mem values;
    cl_mem col_indices;
    cl_mem row_pointer;

    clsparseIdx_t off_values;
    clsparseIdx_t off_col_indices;
    clsparseIdx_t off_row_pointer;

    void* meta;
} clsparseCsrMatrix;

/* A 0-based COO matrix (reference clSPARSE-1x.h:97-117). Declared for ABI
 * completeness; no COO operation is on the accelerated path. */
typedef struct clsparseCooMatrix_
{
    clsparseIdx_t num_rows;
    clsparseIdx_t num_cols;
    clsparseIdx_t num_nonzeros;

    cl_mem values;
    cl_mem col_indices;
    cl_mem row_indices;

    clsparseIdx_t off_values;
    clsparseIdx_t off_col_indices;
    clsparseIdx_t off_row_indices;
} clsparseCooMatrix;

/* A dense matrix (reference clSPARSE-1x.h:122-141). Declared for ABI
 * completeness. */
typedef struct cldenseMatrix_
{
    clsparseIdx_t num_rows;
    clsparseIdx_t num_cols;
    clsparseIdx_t lead_dim;
    cldenseMajor major;

    cl_mem values;
    clsparseIdx_t off_values;
} cldenseMatrix;

#endif /* CLSPARSE_B200_1X_H_ */
