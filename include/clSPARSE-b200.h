/*
 * clSPARSE-b200.h -- project extensions next to the drop-in ABI of clSPARSE.h.
 *
 * Nothing here changes a reference entry point. These functions expose what
 * the reference kept private (row-block words, solver statistics) and the
 * additions with no reference counterpart (mixed-precision refinement, batched
 * solves, the learned preconditioner). All take the same struct types and
 * return clsparseStatus.
 */
#ifndef CLSPARSE_B200_EXT_H_
#define CLSPARSE_B200_EXT_H_

#include "clSPARSE.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Name used for the row-block binning step by the reference's sample
 * (samples/sample-spmv.cpp:57) and a dead test (src/tests/test_readMMcoo.cpp:93);
 * the exported reference function is clsparseCsrMetaCreate. Same behaviour. */
CLSPARSE_EXPORT clsparseStatus
clsparseCsrMetaCompute(clsparseCsrMatrix* csrMatx, clsparseControl control);

/* Host-only CSR-Adaptive binning of a row-pointer array held in host memory,
 * the same computation clsparseCsrMetaCreate runs (reference
 * src/library/internal/data-types/csr-meta.hpp:93-261). Writes at most
 * `capacity` 64-bit words to rowBlocks (may be NULL to only size) and stores
 * in *rowBlockSize the reference's rowBlockSize (2 x words written, or the
 * dry-run size when rowBlocks is NULL, csr-meta.hpp:263-269). Needs no GPU. */
CLSPARSE_EXPORT clsparseStatus
clsparseB200ComputeRowBlocksHost(const clsparseIdx_t* rowPointer, clsparseIdx_t numRows,
                                 cl_ulong* rowBlocks, size_t capacity,
                                 clsparseIdx_t* rowBlockSize);

/* Copies the row-block words of an existing meta to host memory. *count gets
 * the number of words (rowBlockSize / 2). */
CLSPARSE_EXPORT clsparseStatus
clsparseB200CsrMetaGetRowBlocks(const clsparseCsrMatrix* csrMatx, cl_ulong* rowBlocks,
                                size_t capacity, size_t* count);

/* Statistics of the last solve run with this solver control (the reference
 * kept them private in _solverControl, solvers/solver-control.hpp:109-127 and
 * only printed them). */
CLSPARSE_EXPORT clsparseStatus
clsparseB200SolverGetInfo(clSParseSolverControl solverControl, cl_int* nIters,
                          cl_double* initialResidual, cl_double* currentResidual);

/* Device status bits found during the last solve (0 when clean):
 *   1  a row without a diagonal entry (Jacobi)     2  a zero diagonal entry
 *   4  CG curvature <p,Ap> <= 0 or not finite       8  BiCGStab rho == 0 / omega == 0
 *  16  non-finite residual                        */
CLSPARSE_EXPORT clsparseStatus
clsparseB200SolverGetDeviceStatus(clSParseSolverControl solverControl, cl_uint* statusBits);

/* Solver loop driver: 0 = one CUDA graph per solve with a device-side
 * conditional WHILE node (no host round trip per iteration, the default);
 * 1 = host-enqueued chunks of iterations with a device done flag. Both give
 * the same iterates. */
CLSPARSE_EXPORT clsparseStatus
clsparseB200SetSolverLoopMode(clsparseControl control, cl_int mode);

#ifdef __cplusplus
}
#endif

#endif /* CLSPARSE_B200_EXT_H_ */
