/*
 * clSPARSE.h -- drop-in C ABI of clsparse-b200.
 *
 * Every entry point of the reference's public header src/include/clSPARSE.h is
 * declared here with the same name, argument list and return type; each
 * declaration cites the reference line it replaces. clsparseStatus keeps the
 * reference's numeric values (clSPARSE.h:45-88).
 *
 * Execution model: all work of a call is enqueued on the control's CUDA stream
 * (the cl_command_queue handed to clsparseCreateControl). With async disabled
 * (the default, as in the reference) a call returns after its work finished;
 * with clsparseEnableAsync(control, CL_TRUE) it returns once the work is
 * enqueued and clsparseGetEvent hands back an event recorded after it.
 *
 * Operations outside the accelerated path (COO SpMV, SpMM, SpGEMM, format
 * conversions, Matrix Market I/O) are declared for source compatibility and
 * return clsparseNotImplemented.
 */
#ifndef CLSPARSE_B200_H_
#define CLSPARSE_B200_H_

#include "clSPARSE-1x.h"

#if defined(_WIN32)
#define CLSPARSE_EXPORT __declspec(dllexport)
#else
#define CLSPARSE_EXPORT __attribute__((visibility("default")))
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes (reference clSPARSE.h:45-88). */
typedef enum clsparseStatus_
{
    clsparseSuccess              = CL_SUCCESS,
    clsparseInvalidValue         = CL_INVALID_VALUE,
    clsparseInvalidCommandQueue  = CL_INVALID_COMMAND_QUEUE,
    clsparseInvalidContext       = CL_INVALID_CONTEXT,
    clsparseInvalidMemObject     = CL_INVALID_MEM_OBJECT,
    clsparseInvalidDevice        = CL_INVALID_DEVICE,
    clsparseInvalidEventWaitList = CL_INVALID_EVENT_WAIT_LIST,
    clsparseInvalidEvent         = CL_INVALID_EVENT,
    clsparseOutOfResources       = CL_OUT_OF_RESOURCES,
    clsparseOutOfHostMemory      = CL_OUT_OF_HOST_MEMORY,
    clsparseInvalidOperation     = CL_INVALID_OPERATION,
    clsparseCompilerNotAvailable = CL_COMPILER_NOT_AVAILABLE,
    clsparseBuildProgramFailure  = CL_BUILD_PROGRAM_FAILURE,
    clsparseInvalidKernelArgs    = CL_INVALID_KERNEL_ARGS,
    clsparseNotImplemented       = -1024,
    clsparseNotInitialized,
    clsparseStructInvalid,
    clsparseInvalidSize,
    clsparseInvalidMemObj,
    clsparseInsufficientMemory,
    clsparseInvalidControlObject,
    clsparseInvalidFile,
    clsparseInvalidFileFormat,
    clsparseInvalidKernelExecution,
    clsparseInvalidType,
    clsparseInvalidSolverControlObject = -2048,
    clsparseInvalidSystemSize,
    clsparseIterationsExceeded,
    clsparseToleranceNotReached,
    clsparseSolverError
} clsparseStatus;

/* ---- library state (reference clSPARSE.h:108-135, clsparse-init.cpp:25-61) ---- */
CLSPARSE_EXPORT clsparseStatus clsparseSetup(void);                       /* clSPARSE.h:108-109 */
CLSPARSE_EXPORT clsparseStatus clsparseTeardown(void);                    /* clSPARSE.h:119-120 */
CLSPARSE_EXPORT clsparseStatus clsparseGetVersion(cl_uint* major, cl_uint* minor,
                                                  cl_uint* patch, cl_uint* tweak); /* :134-135 */

/* ---- struct initialisers (reference clSPARSE.h:155-208) ---- */
CLSPARSE_EXPORT clsparseStatus clsparseInitScalar(clsparseScalar* scalar);         /* :155-156 */
CLSPARSE_EXPORT clsparseStatus clsparseInitVector(cldenseVector* vec);             /* :168-169 */
CLSPARSE_EXPORT clsparseStatus clsparseInitCooMatrix(clsparseCooMatrix* cooMatx);  /* :181-182 */
CLSPARSE_EXPORT clsparseStatus clsparseInitCsrMatrix(clsparseCsrMatrix* csrMatx);  /* :194-195 */
CLSPARSE_EXPORT clsparseStatus cldenseInitMatrix(cldenseMatrix* denseMatx);        /* :207-208 */

/* ---- control object (reference clSPARSE.h:211-304) ---- */
typedef struct _clsparseControl* clsparseControl;

typedef struct _clsparseCreateResult
{
    clsparseStatus status;
    clsparseControl control;
} clsparseCreateResult;

/* queue: the CUDA stream every call on this control is ordered on. */
CLSPARSE_EXPORT clsparseCreateResult clsparseCreateControl(cl_command_queue queue); /* :243-244 */
CLSPARSE_EXPORT clsparseStatus clsparseEnableAsync(clsparseControl control, cl_bool async); /* :256-257 */
CLSPARSE_EXPORT clsparseStatus clsparseEnableExtendedPrecision(clsparseControl control,
                                                               cl_bool extPrecision); /* :270-271 */

typedef struct _clsparseEventResult
{
    clsparseStatus status;
    cl_event event;
} clsparseEventResult;

/* Returns an event recorded on the control's stream after the last enqueued
 * call. The event stays owned by the control (valid until the next call on it
 * or clsparseReleaseControl). */
CLSPARSE_EXPORT clsparseEventResult clsparseGetEvent(clsparseControl control);      /* :291-292 */
CLSPARSE_EXPORT clsparseStatus clsparseReleaseControl(clsparseControl control);     /* :303-304 */

/* ---- iterative solvers (reference clSPARSE.h:321-482) ---- */
typedef enum _print_mode
{
    QUIET = 0,
    NORMAL,
    VERBOSE
} PRINT_MODE;

typedef enum _precond
{
    NOPRECOND = 0,
    DIAGONAL
} PRECONDITIONER;

typedef struct _solverControl* clSParseSolverControl;

typedef struct _clsparseCreateSolverResult
{
    clsparseStatus status;
    clSParseSolverControl control;
} clsparseCreateSolverResult;

CLSPARSE_EXPORT clsparseCreateSolverResult
clsparseCreateSolverControl(PRECONDITIONER precond, cl_int maxIters,
                            cl_double relTol, cl_double absTol);                    /* :369-371 */
CLSPARSE_EXPORT clsparseStatus clsparseReleaseSolverControl(clSParseSolverControl solverControl); /* :382-383 */
CLSPARSE_EXPORT clsparseStatus
clsparseSetSolverParams(clSParseSolverControl solverControl, PRECONDITIONER precond,
                        cl_int maxIters, cl_double relTol, cl_double absTol);       /* :398-401 */
CLSPARSE_EXPORT clsparseStatus clsparseSolverPrintMode(clSParseSolverControl solverControl,
                                                       PRINT_MODE mode);            /* :413-414 */

/* Preconditioned conjugate gradients, x is the initial guess on entry and the
 * solution on exit; convergence is ||r||_1/||b||_1 <= relTol or
 * <= absTol * initial residual (reference solvers/solver-control.hpp:47-64). */
CLSPARSE_EXPORT clsparseStatus
clsparseScsrcg(cldenseVector* x, const clsparseCsrMatrix* A, const cldenseVector* b,
               clSParseSolverControl solverControl, clsparseControl control);      /* :429-431 */
CLSPARSE_EXPORT clsparseStatus
clsparseDcsrcg(cldenseVector* x, const clsparseCsrMatrix* A, const cldenseVector* b,
               clSParseSolverControl solverControl, clsparseControl control);      /* :446-448 */

/* Right-preconditioned BiCGStab (reference biconjugate-gradients-stabilized.hpp:41-268). */
CLSPARSE_EXPORT clsparseStatus
clsparseScsrbicgStab(cldenseVector* x, const clsparseCsrMatrix* A, const cldenseVector* b,
                     clSParseSolverControl solverControl, clsparseControl control); /* :463-465 */
CLSPARSE_EXPORT clsparseStatus
clsparseDcsrbicgStab(cldenseVector* x, const clsparseCsrMatrix* A, const cldenseVector* b,
                     clSParseSolverControl solverControl, clsparseControl control); /* :480-482 */

/* ---- Matrix Market input (reference clSPARSE.h:508-611, reader
 * src/library/io/mm-reader.cpp:140-760): coordinate real / integer / pattern
 * files with a ".mtx" path; symmetric files mirrored; explicit zeros dropped
 * unless read_explicit_zeroes; entries sorted by (row, column). The device
 * buffers are allocated by the caller with the sizes clsparseHeaderfromFile
 * reports (nnz is an upper bound for symmetric files); the struct's sizes are
 * set from the file. Pattern entries get seeded pseudo-random values in
 * [0, 5) (the reference used rand()). ---- */
CLSPARSE_EXPORT clsparseStatus
clsparseHeaderfromFile(clsparseIdx_t* nnz, clsparseIdx_t* row, clsparseIdx_t* col,
                       const char* filePath);                                       /* :508-509 */
CLSPARSE_EXPORT clsparseStatus
clsparseSCooMatrixfromFile(clsparseCooMatrix* cooMatx, const char* filePath,
                           clsparseControl control, cl_bool read_explicit_zeroes);  /* :533-534 */
CLSPARSE_EXPORT clsparseStatus
clsparseDCooMatrixfromFile(clsparseCooMatrix* cooMatx, const char* filePath,
                           clsparseControl control, cl_bool read_explicit_zeroes);  /* :559-560 */
CLSPARSE_EXPORT clsparseStatus
clsparseSCsrMatrixfromFile(clsparseCsrMatrix* csrMatx, const char* filePath,
                           clsparseControl control, cl_bool read_explicit_zeroes);  /* :584-585 */
CLSPARSE_EXPORT clsparseStatus
clsparseDCsrMatrixfromFile(clsparseCsrMatrix* csrMatx, const char* filePath,
                           clsparseControl control, cl_bool read_explicit_zeroes);  /* :610-611 */

/* ---- CSR-Adaptive row-block metadata (reference clSPARSE.h:613-659) ---- */
typedef struct _clsparseMetaSizeResult
{
    clsparseStatus status;
    clsparseIdx_t metaSize;
} clsparseMetaSizeResult;

/* Number of 64-bit row-block words the meta of this matrix occupies (twice the
 * number of row-block entries, as in the reference csr-meta.hpp:250-260). */
CLSPARSE_EXPORT clsparseMetaSizeResult
clsparseCsrMetaSize(clsparseCsrMatrix* csrMatx, clsparseControl control);           /* :633-634 */
/* Bins the rows of csrMatx into CSR-Adaptive row blocks and attaches the
 * result to csrMatx->meta, replacing any earlier meta. */
CLSPARSE_EXPORT clsparseStatus
clsparseCsrMetaCreate(clsparseCsrMatrix* csrMatx, clsparseControl control);         /* :648-649 */
CLSPARSE_EXPORT clsparseStatus clsparseCsrMetaDelete(clsparseCsrMatrix* csrMatx);   /* :658-659 */

/* ---- dense BLAS-1 (reference clSPARSE.h:694-1032) ---- */
/* r = alpha * y */
CLSPARSE_EXPORT clsparseStatus cldenseSscale(cldenseVector* r, const clsparseScalar* alpha,
                                             const cldenseVector* y, const clsparseControl control); /* :694-698 */
CLSPARSE_EXPORT clsparseStatus cldenseDscale(cldenseVector* r, const clsparseScalar* alpha,
                                             const cldenseVector* y, const clsparseControl control); /* :710-714 */
/* r = alpha * x + y */
CLSPARSE_EXPORT clsparseStatus cldenseSaxpy(cldenseVector* r, const clsparseScalar* alpha,
                                            const cldenseVector* x, const cldenseVector* y,
                                            const clsparseControl control);             /* :727-731 */
CLSPARSE_EXPORT clsparseStatus cldenseDaxpy(cldenseVector* r, const clsparseScalar* alpha,
                                            const cldenseVector* x, const cldenseVector* y,
                                            const clsparseControl control);             /* :744-748 */
/* r = alpha * x + beta * y */
CLSPARSE_EXPORT clsparseStatus cldenseSaxpby(cldenseVector* r, const clsparseScalar* alpha,
                                             const cldenseVector* x, const clsparseScalar* beta,
                                             const cldenseVector* y, const clsparseControl control); /* :762-767 */
CLSPARSE_EXPORT clsparseStatus cldenseDaxpby(cldenseVector* r, const clsparseScalar* alpha,
                                             const cldenseVector* x, const clsparseScalar* beta,
                                             const cldenseVector* y, const clsparseControl control); /* :781-786 */
/* s = sum(x) */
CLSPARSE_EXPORT clsparseStatus cldenseIreduce(clsparseScalar* s, const cldenseVector* x,
                                              const clsparseControl control);           /* :797-800 */
CLSPARSE_EXPORT clsparseStatus cldenseSreduce(clsparseScalar* s, const cldenseVector* x,
                                              const clsparseControl control);           /* :811-814 */
CLSPARSE_EXPORT clsparseStatus cldenseDreduce(clsparseScalar* s, const cldenseVector* x,
                                              const clsparseControl control);           /* :825-828 */
/* s = sum(|x|) */
CLSPARSE_EXPORT clsparseStatus cldenseSnrm1(clsparseScalar* s, const cldenseVector* x,
                                            const clsparseControl control);             /* :838-841 */
CLSPARSE_EXPORT clsparseStatus cldenseDnrm1(clsparseScalar* s, const cldenseVector* x,
                                            const clsparseControl control);             /* :851-854 */
/* s = sqrt(sum(x^2)) */
CLSPARSE_EXPORT clsparseStatus cldenseSnrm2(clsparseScalar* s, const cldenseVector* x,
                                            const clsparseControl control);             /* :864-867 */
CLSPARSE_EXPORT clsparseStatus cldenseDnrm2(clsparseScalar* s, const cldenseVector* x,
                                            const clsparseControl control);             /* :877-880 */
/* r = <x, y> */
CLSPARSE_EXPORT clsparseStatus cldenseSdot(clsparseScalar* r, const cldenseVector* x,
                                           const cldenseVector* y, const clsparseControl control); /* :891-895 */
CLSPARSE_EXPORT clsparseStatus cldenseDdot(clsparseScalar* r, const cldenseVector* x,
                                           const cldenseVector* y, const clsparseControl control); /* :906-910 */
/* r = x (+ - * /) y, elementwise */
CLSPARSE_EXPORT clsparseStatus cldenseSadd(cldenseVector* r, const cldenseVector* x,
                                           const cldenseVector* y, const clsparseControl control); /* :923-927 */
CLSPARSE_EXPORT clsparseStatus cldenseDadd(cldenseVector* r, const cldenseVector* x,
                                           const cldenseVector* y, const clsparseControl control); /* :938-942 */
CLSPARSE_EXPORT clsparseStatus cldenseSsub(cldenseVector* r, const cldenseVector* x,
                                           const cldenseVector* y, const clsparseControl control); /* :953-957 */
CLSPARSE_EXPORT clsparseStatus cldenseDsub(cldenseVector* r, const cldenseVector* x,
                                           const cldenseVector* y, const clsparseControl control); /* :968-972 */
CLSPARSE_EXPORT clsparseStatus cldenseSmul(cldenseVector* r, const cldenseVector* x,
                                           const cldenseVector* y, const clsparseControl control); /* :983-987 */
CLSPARSE_EXPORT clsparseStatus cldenseDmul(cldenseVector* r, const cldenseVector* x,
                                           const cldenseVector* y, const clsparseControl control); /* :998-1002 */
CLSPARSE_EXPORT clsparseStatus cldenseSdiv(cldenseVector* r, const cldenseVector* x,
                                           const cldenseVector* y, const clsparseControl control); /* :1013-1017 */
CLSPARSE_EXPORT clsparseStatus cldenseDdiv(cldenseVector* r, const cldenseVector* x,
                                           const cldenseVector* y, const clsparseControl control); /* :1028-1032 */

/* ---- sparse BLAS-2 (reference clSPARSE.h:1062-1132) ---- */
/* y = alpha * A * x + beta * y. With A->meta set (clsparseCsrMetaCreate) the
 * CSR-Adaptive kernel runs, otherwise the vector-per-row kernel
 * (reference blas2/clsparse-csrmv.hpp:103-132). beta == 0 overwrites y
 * without reading it. */
CLSPARSE_EXPORT clsparseStatus
clsparseScsrmv(const clsparseScalar* alpha, const clsparseCsrMatrix* matx,
               const cldenseVector* x, const clsparseScalar* beta,
               cldenseVector* y, const clsparseControl control);                    /* :1062-1068 */
CLSPARSE_EXPORT clsparseStatus
clsparseDcsrmv(const clsparseScalar* alpha, const clsparseCsrMatrix* matx,
               const cldenseVector* x, const clsparseScalar* beta,
               cldenseVector* y, const clsparseControl control);                    /* :1085-1091 */
/* Declared but never defined by the reference (clSPARSE.h:1106-1132). Here:
 * y = alpha*A*x + beta*y like csrmv, for a COO matrix sorted by row
 * (duplicates summed); beta == 0 overwrites y without reading it. */
CLSPARSE_EXPORT clsparseStatus
clsparseScoomv(const clsparseScalar* alpha, const clsparseCooMatrix* matx,
               const cldenseVector* x, const clsparseScalar* beta,
               cldenseVector* y, const clsparseControl control);                    /* :1106-1112 */
CLSPARSE_EXPORT clsparseStatus
clsparseDcoomv(const clsparseScalar* alpha, const clsparseCooMatrix* matx,
               const cldenseVector* x, const clsparseScalar* beta,
               cldenseVector* y, const clsparseControl control);                    /* :1126-1132 */

/* ---- sparse BLAS-3 (reference clSPARSE.h:1159-1187): C = alpha*A*B + beta*C,
 * B and C dense (row-major as the reference indexes them; column-major ones
 * are honoured too). SpGEMM and the conversions below are not implemented. ---- */
CLSPARSE_EXPORT clsparseStatus
clsparseScsrmm(const clsparseScalar* alpha, const clsparseCsrMatrix* sparseMatA,
               const cldenseMatrix* denseMatB, const clsparseScalar* beta,
               cldenseMatrix* denseMatC, const clsparseControl control);            /* :1159-1165 */
CLSPARSE_EXPORT clsparseStatus
clsparseDcsrmm(const clsparseScalar* alpha, const clsparseCsrMatrix* sparseMatA,
               const cldenseMatrix* denseMatB, const clsparseScalar* beta,
               cldenseMatrix* denseMatC, const clsparseControl control);            /* :1181-1187 */
CLSPARSE_EXPORT clsparseStatus
clsparseScsrSpGemm(const clsparseCsrMatrix* sparseMatA, const clsparseCsrMatrix* sparseMatB,
                   clsparseCsrMatrix* sparseMatC, const clsparseControl control);   /* :1199-1203 */
CLSPARSE_EXPORT clsparseStatus
clsparseScsr2coo(const clsparseCsrMatrix* csr, clsparseCooMatrix* coo,
                 const clsparseControl control);                                    /* :1225-1228 */
CLSPARSE_EXPORT clsparseStatus
clsparseDcsr2coo(const clsparseCsrMatrix* csr, clsparseCooMatrix* coo,
                 const clsparseControl control);                                    /* :1239-1242 */
CLSPARSE_EXPORT clsparseStatus
clsparseScoo2csr(const clsparseCooMatrix* coo, clsparseCsrMatrix* csr,
                 const clsparseControl control);                                    /* :1253-1256 */
CLSPARSE_EXPORT clsparseStatus
clsparseDcoo2csr(const clsparseCooMatrix* coo, clsparseCsrMatrix* csr,
                 const clsparseControl control);                                    /* :1267-1270 */
CLSPARSE_EXPORT clsparseStatus
clsparseScsr2dense(const clsparseCsrMatrix* csr, cldenseMatrix* A,
                   const clsparseControl control);                                  /* :1281-1284 */
CLSPARSE_EXPORT clsparseStatus
clsparseDcsr2dense(const clsparseCsrMatrix* csr, cldenseMatrix* A,
                   clsparseControl control);                                        /* :1295-1298 */
CLSPARSE_EXPORT clsparseStatus
clsparseSdense2csr(const cldenseMatrix* A, clsparseCsrMatrix* csr,
                   const clsparseControl control);                                  /* :1309-1312 */
CLSPARSE_EXPORT clsparseStatus
clsparseDdense2csr(const cldenseMatrix* A, clsparseCsrMatrix* csr,
                   const clsparseControl control);                                  /* :1323-1325 */

#ifdef __cplusplus
}
#endif

#endif /* CLSPARSE_B200_H_ */
