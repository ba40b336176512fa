// Library-private runtime state of clsparse-b200: the control object, the
// CSR-Adaptive meta, the solver control and the helpers every entry point
// uses. Host C++17; included by the .cpp and .cu translation units.
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

#include <atomic>
#include <cstddef>
#include <cstdint>
#include <cstdio>
#include <memory>
#include <vector>

#include "clSPARSE.h"
#include "clSPARSE-b200.h"

namespace clsp {

// Library initialisation counter (reference clsparse-init.cpp:25 keeps a plain
// int; an atomic makes concurrent Setup/Teardown well defined).
extern std::atomic<int> g_initialized;

// CSR-Adaptive constants (reference src/library/include/clSPARSE-private.hpp:46-50).
// These five numbers define the row-block format and must equal the reference's
// so that clsparseCsrMetaCreate produces the same words.
constexpr uint32_t kWgBits = 24;
constexpr uint32_t kRowBits = 32;
constexpr uint32_t kBlkSize = 1024;
constexpr uint32_t kBlockMultiplier = 3;
constexpr uint32_t kRowsForVector = 1;

// A grow-only device allocation.
struct DeviceBuffer {
    void* ptr = nullptr;
    size_t bytes = 0;
    cudaError_t ensure(size_t need);
    void release();
    ~DeviceBuffer() { release(); }
};

struct SolverCache;  // cached CUDA graph + work vectors of the last solve

// Device buffers of the banded inner solves (dia.h): offset table, the
// diagonal-storage copies of A, G and G^T, work vectors, exchange area.
struct DiaWork {
    DeviceBuffer table, A, G, GT, vecs, sync;
};

// Work area of the mixed-precision refinement (mixed.cu), owned by the control.
struct MixedWork {
    DeviceBuffer lowvals, y, r32, d, parts;
    std::unique_ptr<DiaWork> dia;
    void* pinned = nullptr;
    ~MixedWork() {
        if (pinned) cudaFreeHost(pinned);
    }
};

// Work area and cached graph of the batched solver (batched.cu).
struct BatchWork {
    DeviceBuffer vecs, meta, out;
    DeviceBuffer dia, dia_meta;  // diagonal-storage copies of banded systems and their offsets
    cudaGraphExec_t exec = nullptr;
    unsigned char args[256] = {};  // kernel arguments the graph was captured with
    uint32_t grid = 0;
    ~BatchWork() {
        if (exec) cudaGraphExecDestroy(exec);
    }
};

}  // namespace clsp

// The control object (reference internal/clsparse-control.hpp:30-80). Owns no
// user memory; keeps a scratch area for reductions and the solver workspace.
struct _clsparseControl {
    cudaStream_t stream = nullptr;  // the caller's queue
    int device = 0;
    int sm_count = 148;
    size_t l2_bytes = 0;
    bool async = false;
    bool extended_precision = false;
    int solver_loop_mode = 0;       // 0 graph while-loop, 1 host chunks, 2 persistent kernel, 3 banded CG
    cudaEvent_t event = nullptr;    // recorded after each call
    cudaStream_t capture_stream = nullptr;  // private stream used for graph capture
    // Reduction scratch: kMaxReduceCtas doubles x 4 partial slots + a ticket.
    clsp::DeviceBuffer reduce_scratch;
    // Pinned host word used to read back reduction results of solver calls.
    void* pinned = nullptr;
    std::unique_ptr<clsp::SolverCache> solver_cache;
    std::unique_ptr<clsp::MixedWork> mixed_work;
    std::unique_ptr<clsp::BatchWork> batch_work;
    std::unique_ptr<clsp::DiaWork> dia_cg;  // banded drop-in CG (solver loop mode 3)
};

// CSR-Adaptive meta attached to clsparseCsrMatrix::meta (reference
// clSPARSE-1x.hpp:45-62). Immutable after creation except for the long-row
// tickets, which every SpMV leaves at zero when it returns.
struct matrix_meta {
    clsparseIdx_t rowBlockSize = 0;     // 2 x number of row-block words (reference semantics)
    size_t num_words = 0;               // row-block words; CTAs of one SpMV = num_words - 1
    cl_ulong* d_rowBlocks = nullptr;    // device copy of the words
    std::vector<cl_ulong> h_rowBlocks;  // host copy (for inspection)
    uint32_t* d_word_nnz = nullptr;     // row_pointer[first row of word w], one per word
    std::vector<uint32_t> h_word_nnz;   // host copy (static CTA partitions of the persistent solvers)
    double* d_lr_partial = nullptr;     // one partial sum per row-block word (long rows)
    uint32_t* d_lr_ticket = nullptr;    // one arrival counter per row-block word (long rows)
    int* d_error = nullptr;             // set by an SpMV whose bounded barrier wait timed out
    clsparseIdx_t num_rows = 0;
    clsparseIdx_t num_nonzeros = 0;
    uint32_t nnz_lo = 0;                // row_pointer[0]
    uint32_t nnz_hi = 0;                // row_pointer[num_rows]
    uint32_t max_row = 0;               // longest row (nonzeros)
    int device = 0;
    int sm_count = 148;                 // SMs of the device the meta was made on
    // Row-block shape the words were made with (the reference's constants by
    // default; clsparseB200CsrMetaCreateTuned sets others) and the CTA width
    // of the adaptive kernel.
    uint32_t blk_size = clsp::kBlkSize;
    uint32_t blk_mult = clsp::kBlockMultiplier;
    uint32_t rows_for_vector = clsp::kRowsForVector;
    int cta_threads = 128;
    ~matrix_meta();
};

// True when a meta has the reference's row-block shape (the only one the
// persistent solver and the TMA variant are built for).
inline bool meta_is_default_shape(const matrix_meta* m) {
    return m->blk_size == clsp::kBlkSize && m->blk_mult == clsp::kBlockMultiplier &&
           m->rows_for_vector == clsp::kRowsForVector;
}

// Solver control (reference solvers/solver-control.hpp:37-128).
struct _solverControl {
    cl_int nIters = 0;
    cl_int maxIters = 0;
    PRECONDITIONER preconditioner = NOPRECOND;
    cl_double relativeTolerance = 0.0;
    cl_double absoluteTolerance = 0.0;
    cl_double initialResidual = 0.0;
    cl_double currentResidual = 0.0;
    PRINT_MODE printMode = QUIET;
    cl_uint deviceStatus = 0;
    cl_int normType = 0;  // 0: reference L1 stop test, 1: L2 (clsparseB200SolverSetNormType)
    cl_int stopOnNonFinite = 0;  // internal: inner solves of the refinement end on a non-finite residual
    // optional device-resident records of the next solves
    cl_double* history = nullptr;   // residuum per iteration (clsparseB200SolverSetHistory)
    cl_uint historyCapacity = 0;
    cl_uint historyLength = 0;      // entries the last solve wrote
    cl_int snapshotCount = 0;       // residual vectors after given iterations (clsparseB200SolverSetSnapshots)
    cl_int snapshotIters[8] = {};
    void* snapshots = nullptr;
    void printSummary(clsparseStatus status) const;
};

namespace clsp {

// Opt-in NVTX ranges around API calls (CLSPARSE_B200_NVTX=1): a profiler's
// timeline then shows each call under its API name. NVTX 3 is header-only and
// costs nothing unless a tool is attached; with the switch off not even the
// push is made.
bool trace_enabled();
class TraceRange {
public:
    explicit TraceRange(const char* name) : on_(trace_enabled()) {
        if (on_) nvtxRangePushA(name);
    }
    ~TraceRange() {
        if (on_) nvtxRangePop();
    }
    TraceRange(const TraceRange&) = delete;
    TraceRange& operator=(const TraceRange&) = delete;
private:
    bool on_;
};

// Sets the control's device current for the scope of an API call.
class DeviceGuard {
public:
    explicit DeviceGuard(int dev);
    ~DeviceGuard();
private:
    int prev_ = -1;
    bool changed_ = false;
};

// Ends an API call: records the control's event and, unless async, waits for
// the stream. Maps launch / execution errors to clsparseInvalidKernelExecution.
clsparseStatus finish_call(clsparseControl control);

// Checks the common preconditions (library initialised, control present).
inline clsparseStatus check_entry(clsparseControl control) {
    if (g_initialized.load() == 0) return clsparseNotInitialized;
    if (control == nullptr) return clsparseInvalidControlObject;
    return clsparseSuccess;
}

template <typename T>
inline T* dev_ptr(cl_mem base, clsparseIdx_t off) {
    return static_cast<T*>(base) + off;
}

constexpr int kMaxReduceCtas = 2048;

// ---- SpMV launch interface (spmv.cu) ----

// Optional fused epilogue of an SpMV: per-row dot products of the result y
// with w0 (and with y itself), reduced deterministically over the grid; the
// last CTA to finish runs a solver-specific finaliser (spmv_epilogue_op).
enum class EpiOp : int { None = 0, CgAlpha = 1, BicgAlpha = 2, BicgOmega = 3, PcgRz = 4, PcgRz0 = 5 };

struct SpmvEpilogue {
    int ndots = 0;            // 0, 1 or 2
    const void* w0 = nullptr; // dot0 = sum y_i * w0_i
    bool dot1_self = false;   // dot1 = sum y_i * y_i
    double* partials = nullptr;   // [ndots][num_ctas + 256] (two-level reduction)
    uint32_t* ticket = nullptr;   // 257 zeroed counters
    EpiOp op = EpiOp::None;
    void* state = nullptr;    // solver state the finaliser updates
    unsigned long long cond = 0;  // graph conditional handle (0 = none)
    const int* done = nullptr;    // when set and *done != 0 the kernel returns at once
};

template <typename T>
struct CsrView {
    const T* vals;
    const uint32_t* cols;
    const uint32_t* rp;
    uint32_t nrows, ncols, nnz;
    const matrix_meta* meta;
};

// Sets *bad (device int, not cleared here) when any of the n column indices
// at cols is >= ncols (spmv.cu); clsparseCsrMetaCreate's structure check.
cudaError_t launch_validate_columns(const uint32_t* cols, size_t n, uint32_t ncols, int* bad, int sm_count,
                                    cudaStream_t s);

// Number of CTAs an SpMV of this matrix launches (sizes epilogue partials).
uint32_t spmv_num_ctas(const matrix_meta* meta, uint32_t nrows, uint32_t nnz);

// y = alpha*A*x + beta*y with matrix values of type V (double, float or
// bf16) and vectors / arithmetic in T.
template <typename V, typename T>
cudaError_t launch_csrmv(const CsrView<V>& A, const T* alpha, const T* beta, const T* x, T* y,
                         bool extended, const SpmvEpilogue& epi, cudaStream_t s);

// Continuation of an inner solve of the mixed-precision refinement: with
// `warm`, the solve starts from x == 0 with r = b (the replaced residual) and
// keeps the previous solve's search direction p, forming
// p = z + (<r,z> / rz) p; on return rz holds the denominator for the next
// continuation. The previous solve must have run on the same operands and
// control.
struct WarmStart {
    bool warm = false;
    double rz = 0.0;
};

// CG with matrix values of type V and vectors in T (solvers.cu); the drop-in
// entry points use V == T, the mixed-precision refinement uses float / bf16.
template <typename V, typename T>
clsparseStatus cg_solve_typed(cldenseVector* x, const clsparseCsrMatrix* A, const cldenseVector* b,
                              clSParseSolverControl sc, clsparseControl c, WarmStart* ws = nullptr);

// BiCGStab with matrix values of type V and vectors in T (solvers.cu).
template <typename V, typename T>
clsparseStatus bicg_solve_typed(cldenseVector* x, const clsparseCsrMatrix* A, const cldenseVector* b,
                                clSParseSolverControl sc, clsparseControl c);

// PCG with the factorized preconditioner M^-1 = G^T G (solvers.cu).
template <typename V, typename T, typename VG>
clsparseStatus pcg_factor_typed(cldenseVector* x, const clsparseCsrMatrix* A, const cldenseVector* b,
                                clSParseSolverControl sc, const CsrView<VG>& G, const CsrView<VG>& Gt,
                                clsparseControl c, WarmStart* ws = nullptr);

// Device views of a learned factor G (L = tril(A) order) and G^T (gnn.cu).
// CSR-Adaptive metas of the factor's patterns, made on first use (gnn.cu).
clsparseStatus spai_ensure_metas(clsparseB200Spai net, clsparseControl c);
bool spai_factor_views(clsparseB200Spai net, CsrView<__nv_bfloat16>& G16, CsrView<__nv_bfloat16>& GT16,
                       CsrView<float>& G32, CsrView<float>& GT32, CsrView<double>& G64,
                       CsrView<double>& GT64);

// Builds the meta of a matrix with the given row-block shape and adaptive
// kernel CTA width (meta.cpp); clsparseCsrMetaCreate uses the reference's
// shape and default_cta_threads().
clsparseStatus create_meta(clsparseCsrMatrix* csrMatx, clsparseControl control, uint32_t blk, uint32_t mult,
                           uint32_t rfv, int nt);
int default_cta_threads();

// Host binning (meta.cpp).
void compute_row_blocks(cl_ulong* rowBlocks, clsparseIdx_t& rowBlockSize, const clsparseIdx_t* rp,
                        clsparseIdx_t nRows, uint32_t blkSize, uint32_t blkMultiplier,
                        uint32_t rowsForVector, bool allocate);

}  // namespace clsp
