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

/* clsparseCsrMetaCreate with a chosen row-block shape, the knobs the
 * autotuner sweeps: blkSize (the reference's BLKSIZE, 512, 1024 or 2048),
 * blkMultiplier (long rows are cut into blkMultiplier * blkSize chunks,
 * 1..64), rowsForVector (blocks of at most this many rows are reduced one row
 * at a time by the whole CTA, 1..256) and ctaThreads (threads per CTA of the
 * adaptive kernel: 128, or 256 for blkSize >= 1024). The reference hard-codes
 * these (src/library/include/clSPARSE-private.hpp:46-50) and passes them to
 * ComputeRowBlocks (src/library/internal/data-types/csr-meta.hpp:52-269);
 * clsparseCsrMetaCreate uses them unchanged. Any shape gives the same SpMV
 * results up to summation order; the persistent solver (loop mode 2) needs
 * the default shape and otherwise runs as loop mode 0. */
CLSPARSE_EXPORT clsparseStatus
clsparseB200CsrMetaCreateTuned(clsparseCsrMatrix* csrMatx, cl_uint blkSize, cl_uint blkMultiplier,
                               cl_uint rowsForVector, cl_uint ctaThreads, clsparseControl control);

/* Reads a Matrix Market file into HOST CSR arrays, with the same rules as
 * clsparseDCsrMatrixfromFile (no GPU needed). With rowPointer, colIndices or
 * values NULL only the sizes are returned; otherwise rowPointer needs
 * numRows + 1 entries and colIndices / values `capacity` >= numNonzeros
 * entries (clsparseInsufficientMemory if smaller). Project extension, no
 * reference counterpart. */
CLSPARSE_EXPORT clsparseStatus
clsparseB200ReadMatrixMarketHost(const char* filePath, cl_bool read_explicit_zeroes, clsparseIdx_t* numRows,
                                 clsparseIdx_t* numCols, clsparseIdx_t* numNonzeros, clsparseIdx_t* rowPointer,
                                 clsparseIdx_t* colIndices, cl_double* values, size_t capacity);

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

/* Stop-test norm of clsparse{S,D}csrcg / csrbicgStab on this solver control:
 * 1 = ||r||_1 / ||b||_1 as the reference (the default), 2 = ||r||_2 / ||b||_2. */
CLSPARSE_EXPORT clsparseStatus
clsparseB200SolverSetNormType(clSParseSolverControl solverControl, cl_int normType);

/* Outcome of a mixed-precision refinement solve. */
typedef struct clsparseB200MixedInfo_
{
    cl_int outerIterations;       /* FP64 residual evaluations after the first */
    cl_int innerIterations;       /* CG iterations in the low-precision inner solves */
    cl_double initialTrueResidual;/* ||b - A x0||_2 / ||b||_2, FP64 */
    cl_double trueResidual;       /* ||b - A x||_2 / ||b||_2 on exit, FP64 */
    cl_int converged;             /* trueResidual <= the control's relative tolerance */
} clsparseB200MixedInfo;

/* FP64 iterative refinement around a low-precision Jacobi/none-preconditioned
 * CG: the FP64 residual r = b - A x, the update x += d and the stop test
 * ||r||_2 / ||b||_2 <= relTol run in FP64 on the device; the inner solves of
 * A d = r use the matrix values rounded to FP32 (innerPrecision 0) or BF16
 * (innerPrecision 1) with FP32 vectors and FP32 accumulation, each to a
 * relative L2 reduction of innerTolerance. maxIters of the solver control
 * bounds the total inner iterations. x holds the initial guess on entry.
 * No reference counterpart (a project extension). */
CLSPARSE_EXPORT clsparseStatus
clsparseDcsrcgMixed(cldenseVector* x, const clsparseCsrMatrix* A, const cldenseVector* b,
                    clSParseSolverControl solverControl, cl_int innerPrecision,
                    cl_double innerTolerance, clsparseB200MixedInfo* info,
                    clsparseControl control);

/* The same FP64 refinement around BiCGStab (reference
 * src/library/solvers/biconjugate-gradients-stabilized.hpp:41-268, run on
 * the FP32- or BF16-valued copy with FP32 vectors). No symmetry needed. The
 * inner BiCGStab restarts at every refinement step (the short recurrences of
 * BiCGStab have no residual-replacement continuation here). Project
 * extension, no reference counterpart. */
CLSPARSE_EXPORT clsparseStatus
clsparseDcsrbicgStabMixed(cldenseVector* x, const clsparseCsrMatrix* A, const cldenseVector* b,
                          clSParseSolverControl solverControl, cl_int innerPrecision,
                          cl_double innerTolerance, clsparseB200MixedInfo* info, clsparseControl control);

/* Per-system results of a batched solve. The two arrays are optional (NULL) or
 * hold numSystems entries each. */
typedef struct clsparseB200BatchResult_
{
    cl_int* iterations;        /* CG iterations of each system */
    cl_double* residuals;      /* FP64 ||b - A x||_2 / ||b||_2 of each system on exit */
    cl_int systemsConverged;   /* systems whose FP64 residual met the tolerance */
    cl_int maxIterations;
    cl_double worstResidual;
} clsparseB200BatchResult;

/* Solves numSystems independent SPD systems stacked block-diagonally in A
 * (system s owns rows and columns [systemOffsets[s], systemOffsets[s+1]),
 * systemOffsets a host array of numSystems+1 entries starting at 0 and ending
 * at num_rows) with Jacobi-CG in FP32, in one persistent launch captured into
 * a CUDA graph. Each system stops when its FP64 true residual
 * ||b - A x||_2 / ||b||_2 <= the control's relTol (checked whenever the FP32
 * recursive residual says so; CG restarts from x otherwise) or after maxIters
 * iterations. lanesPerRow (optional, per system: 1..32, a power of two) sets
 * the SpMV width, e.g. from the autotuner. No reference counterpart. */
CLSPARSE_EXPORT clsparseStatus
clsparseScsrcgBatched(cldenseVector* x, const clsparseCsrMatrix* A, const cldenseVector* b,
                      const clsparseIdx_t* systemOffsets, cl_int numSystems,
                      const cl_int* lanesPerRow, clSParseSolverControl solverControl,
                      clsparseB200BatchResult* result, clsparseControl control);

/* ---- learned factorized sparse approximate inverse (no reference counterpart) ----
 * A 4-layer message-passing network (hidden width 64, BF16 weights, FP32
 * accumulation) over the graph of an SPD matrix A emits G on the pattern of
 * tril(A) with a softplus-positive diagonal; M^-1 = G^T G is SPD. Training,
 * inference and the optimiser run on the GPU (clsparse_b200/csrc/gnn.cu). */
typedef struct _clsparseB200Spai* clsparseB200Spai;

/* New network with weights drawn from a generator seeded with `seed`. */
CLSPARSE_EXPORT clsparseStatus clsparseB200SpaiCreate(clsparseB200Spai* spai, cl_ulong seed);
CLSPARSE_EXPORT clsparseStatus clsparseB200SpaiRelease(clsparseB200Spai spai);
/* Prepares the graph of A (FP64 values, sorted columns, positive diagonal,
 * symmetric pattern, row_pointer[0] == 0) for training or building G; the
 * graph is built on the device (no host copy of A beyond the cache key
 * below). clsparseInvalidValue if A does not qualify. Building G takes rows
 * of tril(A) of any length; training (LossGrad / TrainStep) takes at most 32
 * entries per row of tril(A) and returns clsparseInvalidValue beyond. A's
 * arrays must stay valid while the network uses them. The graphs of up to 8
 * earlier matrices of at most 65,536 rows are kept (device memory, freed by
 * clsparseB200SpaiRelease) and reused when a matrix with the same device
 * addresses and bit-identical arrays is set again; larger matrices are
 * rebuilt on every call, into the same buffers when they are large enough.
 * Call clsparseB200SpaiBuild after setting a matrix before using G. */
CLSPARSE_EXPORT clsparseStatus clsparseB200SpaiSetMatrix(clsparseB200Spai spai, const clsparseCsrMatrix* A,
                                                         clsparseControl control);
/* Reads (toDevice = 0) or writes (1) the flat FP32 parameter vector; *count
 * gets its length. */
CLSPARSE_EXPORT clsparseStatus clsparseB200SpaiParams(clsparseB200Spai spai, cl_float* host, size_t capacity,
                                                      size_t* count, cl_int toDevice);
/* Loss and gradient at the current weights for the current matrix: the
 * Kaporin bound log(tr(G A G^T)/n) - (2/n) sum log g_ii of the scaled
 * operator plus lambda * mean_k ||G^T G A r_k - r_k||^2/||r_k||^2 over K probe
 * vectors stored back to back in `probes` (FP32, scaled space). fp32Weights
 * uses the FP32 master weights instead of their BF16 rounding. */
CLSPARSE_EXPORT clsparseStatus clsparseB200SpaiLossGrad(clsparseB200Spai spai, const cldenseVector* probes,
                                                        cl_int K, cl_double lambda, cl_int fp32Weights,
                                                        cl_double* loss, cl_float* grad, size_t capacity,
                                                        clsparseControl control);
/* One Adam step (learning rate lr) on that loss. */
CLSPARSE_EXPORT clsparseStatus clsparseB200SpaiTrainStep(clsparseB200Spai spai, const cldenseVector* probes,
                                                         cl_int K, cl_double lambda, cl_double lr,
                                                         cl_double* loss, clsparseControl control);
/* The network's device gradient buffer (FP32, *count values), which
 * clsparseB200SpaiLossGrad fills: data-parallel training sums it over ranks
 * in place (e.g. one NCCL all-reduce) before clsparseB200SpaiAdamStep. */
CLSPARSE_EXPORT clsparseStatus clsparseB200SpaiGradient(clsparseB200Spai spai, cl_float** deviceGrad, size_t* count);
/* One Adam step (learning rate lr) on gradScale times the gradient buffer
 * (1 / ranks after an all-reduce of summed gradients). */
CLSPARSE_EXPORT clsparseStatus clsparseB200SpaiAdamStep(clsparseB200Spai spai, cl_double lr, cl_double gradScale,
                                                        clsparseControl control);
/* Runs the network on the current matrix and exports G and G^T for the solver. */
CLSPARSE_EXPORT clsparseStatus clsparseB200SpaiBuild(clsparseB200Spai spai, clsparseControl control);
/* Copies the exported G (FP64) and its pattern (row pointers n+1, columns). */
CLSPARSE_EXPORT clsparseStatus clsparseB200SpaiGetFactor(clsparseB200Spai spai, clsparseIdx_t* rowPtr,
                                                         clsparseIdx_t* cols, cl_double* vals,
                                                         size_t capacity, size_t* nnz);
/* Checkpoint of weights and optimiser state: magic "CLSPSPAI", version,
 * sizes, payload and an FNV-1a 64 checksum. */
CLSPARSE_EXPORT clsparseStatus clsparseB200SpaiSave(clsparseB200Spai spai, const char* path);
CLSPARSE_EXPORT clsparseStatus clsparseB200SpaiLoad(clsparseB200Spai spai, const char* path);

/* CG preconditioned with the learned M^-1 = G^T G (after clsparseB200SpaiBuild
 * on A). innerPrecision 0 / 1: FP64 iterative refinement with FP32 / BF16
 * matrix values in the inner PCG (FP32 vectors, BF16 G), as
 * clsparseDcsrcgMixed; when an outer step fails to halve the FP64 residual the
 * remaining inner solves fall back to Jacobi (*fellBack = 1). innerPrecision
 * 2: FP64 PCG with G in FP64, L2 stop test. */
CLSPARSE_EXPORT clsparseStatus
clsparseDcsrcgLearned(cldenseVector* x, const clsparseCsrMatrix* A, const cldenseVector* b,
                      clSParseSolverControl solverControl, clsparseB200Spai spai, cl_int innerPrecision,
                      cl_double innerTolerance, clsparseB200MixedInfo* info, cl_int* fellBack,
                      clsparseControl control);

/* FP64 dot product r = <x, y> that allocates nothing, for callers that may
 * not call cudaMalloc (allocation-free real-time loops, applications that
 * budget every device allocation themselves, code enqueuing into streams it
 * does not own). It needs no clsparseControl (creating one allocates) and
 * takes the CUDA stream directly; its scratch is a fixed device array of
 * about 16 KB inside the library, resident on every GPU that loads it.
 * Limit: at most 33,554,432 elements (clsparseInvalidSize beyond). Returns
 * once the work is enqueued on queue. All calls share the array, so calls
 * that overlap on the GPU race and must be serialised by the caller. The
 * first successful call on a device looks the array up on that device; make
 * it before beginning any stream capture. A failed lookup returns
 * clsparseInvalidDevice and is retried by the next call. Resetting a device
 * (cudaDeviceReset) after the first call on it is not supported. No
 * counterpart in the reference. */
CLSPARSE_EXPORT clsparseStatus
cldenseDdotNoAlloc(clsparseScalar* r, const cldenseVector* x, const cldenseVector* y,
                   cl_command_queue queue);

/* Solver loop driver: 0 = one CUDA graph per solve with a device-side
 * conditional WHILE node (no host round trip per iteration, the default);
 * 1 = host-enqueued chunks of iterations with a device done flag (same
 * iterates as 0); 2 = CG and factorized PCG as ONE persistent cooperative
 * kernel per solve (grid-wide exchanges between phases; needs a
 * CSR-Adaptive meta, otherwise and for BiCGStab the solve runs as in 0;
 * iterates equal up to reduction order); 3 = clsparse{S,D}csrcg and
 * clsparse{S,D}csrbicgStab on a banded matrix with a CSR-Adaptive meta (at
 * most 16 distinct column offsets j - i, columns strictly increasing per row)
 * as ONE cooperative kernel over a private copy of A stored by diagonal,
 * rebuilt at every call (the reference's row order and rounding, stop tests,
 * nIters and solver-control bookkeeping; iterates equal up to the order of
 * the dot-product sums); matrices without a meta or not banded, a zero or
 * missing diagonal under Jacobi, residual history or snapshots, extended
 * precision, and BiCGStab systems larger than L2 run as in 0. */
CLSPARSE_EXPORT clsparseStatus
clsparseB200SetSolverLoopMode(clsparseControl control, cl_int mode);

/* Device-resident residual history of the next CG / BiCGStab solves with this
 * solver control (the reference prints these residuals in VERBOSE mode,
 * src/library/solvers/solver-control.hpp:66-106): history[0] = the initial
 * residuum, history[k] = the residuum the stop test saw after k iterations
 * (BiCGStab: ||r||, or ||s|| at the iteration that stopped on it), FP64,
 * written on the device without host reads, up to capacity entries.
 * NULL (capacity 0) turns it off. */
CLSPARSE_EXPORT clsparseStatus
clsparseB200SolverSetHistory(clSParseSolverControl solverControl, cl_double* deviceHistory, cl_uint capacity);
/* Entries the last solve wrote into the history. */
CLSPARSE_EXPORT clsparseStatus
clsparseB200SolverGetHistoryLength(clSParseSolverControl solverControl, cl_uint* length);
/* Snapshots of the CG residual vector r (the solve's value type, n values
 * each, back to back in deviceVectors) after each of the listed iteration
 * counts (0 = r0 = b - A x0), at most 8; count 0 turns them off. The solves
 * then run on the graph engine (loop modes 0 and 1). */
CLSPARSE_EXPORT clsparseStatus
clsparseB200SolverSetSnapshots(clSParseSolverControl solverControl, const cl_int* iterations, cl_int count,
                               void* deviceVectors);

/* ---- Row-partitioned FP64 CG, one rank's device work (multi-GPU) ----
 * No counterpart in the reference (one queue per control,
 * src/library/internal/clsparse-control.hpp:30-47); it replaces
 * clsparseDcsrcg (include/clSPARSE.h:374-378) for a matrix split by rows
 * over several GPUs. A rank holds its rows (columns renumbered into an
 * "extended" vector of extLength entries whose entries ownOffset ..
 * ownOffset + rows - 1 are the rank's own) and local x, b. Between the
 * stages the caller moves data with its own collectives on the control's
 * stream: the other ranks' entries of the extended vectors (xExt before
 * Residual, zExt before every Product) and a sum over ranks of the four
 * FP64 `sums` before every Update. One solve:
 *   Start; exchange xExt; Residual; exchange zExt; Product; all-reduce sums;
 *   for step = 0, 1, ...: Update(step); exchange zExt; Product; all-reduce
 *   sums; and every few steps State, until it reports done.
 * The iteration is CG in the Chronopoulos-Gear form (one all-reduce per
 * step), with the reference's L1 stop test, residuals and nIters
 * (conjugate-gradients.hpp:65-226, solver-control.hpp:47-64); the decisions
 * are taken on the device and steps after the finish do nothing, so State
 * is the only host synchronisation. */
typedef struct _clsparseB200DistCg* clsparseB200DistCg;

/* Local rows (FP64, num_cols ignored); precond DIAGONAL or NOPRECOND.
 * clsparseInvalidValue if a column is >= extLength or, with DIAGONAL, a
 * row's diagonal (column ownOffset + row) is missing or zero. */
CLSPARSE_EXPORT clsparseStatus
clsparseB200DistCgCreate(clsparseB200DistCg* handle, const clsparseCsrMatrix* localRows, cl_uint extLength,
                         cl_uint ownOffset, cl_int precond, clsparseControl control);
CLSPARSE_EXPORT clsparseStatus clsparseB200DistCgRelease(clsparseB200DistCg handle);
/* Device addresses of the extended vectors and of the four sums. */
CLSPARSE_EXPORT clsparseStatus
clsparseB200DistCgBuffers(clsparseB200DistCg handle, cl_double** xExt, cl_double** zExt, cl_double** sums);
/* Binds x (updated in place) and b; copies x into xExt's own entries. */
CLSPARSE_EXPORT clsparseStatus
clsparseB200DistCgStart(clsparseB200DistCg handle, cldenseVector* x, const cldenseVector* b, clsparseControl control);
CLSPARSE_EXPORT clsparseStatus clsparseB200DistCgResidual(clsparseB200DistCg handle, clsparseControl control);
CLSPARSE_EXPORT clsparseStatus clsparseB200DistCgProduct(clsparseB200DistCg handle, clsparseControl control);
/* Tolerances and iteration limit from solverControl. */
CLSPARSE_EXPORT clsparseStatus
clsparseB200DistCgUpdate(clsparseB200DistCg handle, cl_int step, clSParseSolverControl solverControl,
                         clsparseControl control);
/* Waits for the stream; *done = 1 once finished; fills solverControl's
 * nIters and residuals (clsparseB200SolverGetInfo). */
CLSPARSE_EXPORT clsparseStatus
clsparseB200DistCgState(clsparseB200DistCg handle, cl_int* done, clSParseSolverControl solverControl,
                        clsparseControl control);
/* dst[i] = src[idx[i]] for i < count (packs entries to send). */
CLSPARSE_EXPORT clsparseStatus
clsparseB200DistCgGather(cl_double* dst, const cl_double* src, const cl_uint* idx, cl_uint count,
                         clsparseControl control);

#ifdef __cplusplus
}
#endif

#endif /* CLSPARSE_B200_EXT_H_ */
