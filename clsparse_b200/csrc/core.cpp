// Library state, control object, solver control and the entry points that are
// declared for ABI compatibility but lie outside the accelerated path.
// Reference: src/library/clsparse-init.cpp, internal/clsparse-control.cpp,
// solvers/solver-control.{hpp,cpp}.
#include <cstdlib>
#include <cstring>
#include <iostream>

#include "internal.h"
#include "solver_cache.h"

namespace clsp {

bool trace_enabled() {
    static const bool on = [] {
        const char* e = std::getenv("CLSPARSE_B200_NVTX");
        return e != nullptr && e[0] != '\0' && e[0] != '0';
    }();
    return on;
}

std::atomic<int> g_initialized{0};

cudaError_t DeviceBuffer::ensure(size_t need) {
    if (need <= bytes && ptr != nullptr) return cudaSuccess;
    release();
    cudaError_t e = cudaMalloc(&ptr, need);
    if (e != cudaSuccess) {
        ptr = nullptr;
        bytes = 0;
        return e;
    }
    bytes = need;
    return cudaSuccess;
}

void DeviceBuffer::release() {
    if (ptr) cudaFree(ptr);
    ptr = nullptr;
    bytes = 0;
}

DeviceGuard::DeviceGuard(int dev) {
    if (cudaGetDevice(&prev_) == cudaSuccess && prev_ != dev) {
        changed_ = cudaSetDevice(dev) == cudaSuccess;
    }
}

DeviceGuard::~DeviceGuard() {
    if (changed_) cudaSetDevice(prev_);
}

clsparseStatus finish_call(clsparseControl control) {
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return clsparseInvalidKernelExecution;
    if (control->event) cudaEventRecord(control->event, control->stream);
    if (!control->async) {
        e = cudaStreamSynchronize(control->stream);
        if (e != cudaSuccess) return clsparseInvalidKernelExecution;
    }
    return clsparseSuccess;
}

}  // namespace clsp

void _solverControl::printSummary(clsparseStatus status) const {
    if (printMode != VERBOSE && printMode != NORMAL) return;
    std::cout << "Solver constraints: \n"
              << "\trelative tolerance = " << relativeTolerance
              << "\n\tabsolute tolerance = " << absoluteTolerance
              << "\n\tmax iterations = " << maxIters << "\n\tPreconditioner: "
              << (preconditioner == DIAGONAL ? "Diagonal" : "No preconditioner") << std::endl;
    std::cout << "Solver finished calculations with status " << status << std::endl;
    std::cout << "\tfinal residual = " << currentResidual << "\titerations = " << nIters
              << std::endl;
}

using namespace clsp;

extern "C" {

clsparseStatus clsparseSetup(void) {
    g_initialized.store(1);
    return clsparseSuccess;
}

clsparseStatus clsparseTeardown(void) {
    g_initialized.store(0);
    return clsparseSuccess;
}

// Version of the reference release this library is a drop-in for
// (reference src/CMakeLists.txt:40, project( clSPARSE VERSION 0.10.2.0 )).
clsparseStatus clsparseGetVersion(cl_uint* major, cl_uint* minor, cl_uint* patch, cl_uint* tweak) {
    if (!major || !minor || !patch || !tweak) return clsparseInvalidValue;
    *major = 0;
    *minor = 10;
    *patch = 2;
    *tweak = 0;
    return clsparseSuccess;
}

clsparseStatus clsparseInitScalar(clsparseScalar* scalar) {
    if (!scalar) return clsparseInvalidValue;
    std::memset(scalar, 0, sizeof(*scalar));
    return clsparseSuccess;
}

clsparseStatus clsparseInitVector(cldenseVector* vec) {
    if (!vec) return clsparseInvalidValue;
    std::memset(vec, 0, sizeof(*vec));
    return clsparseSuccess;
}

clsparseStatus clsparseInitCooMatrix(clsparseCooMatrix* m) {
    if (!m) return clsparseInvalidValue;
    std::memset(m, 0, sizeof(*m));
    return clsparseSuccess;
}

clsparseStatus clsparseInitCsrMatrix(clsparseCsrMatrix* m) {
    if (!m) return clsparseInvalidValue;
    std::memset(m, 0, sizeof(*m));
    return clsparseSuccess;
}

clsparseStatus cldenseInitMatrix(cldenseMatrix* m) {
    if (!m) return clsparseInvalidValue;
    std::memset(m, 0, sizeof(*m));
    m->major = rowMajor;
    return clsparseSuccess;
}

// The control binds to the device that is current when it is created and to
// the caller's stream. It queries the device once (the reference JIT-built an
// empty kernel for this, clsparse-control.cpp:29-96) and allocates the small
// reduction scratch area the BLAS-1 reductions use.
clsparseCreateResult clsparseCreateControl(cl_command_queue queue) {
    clsparseCreateResult res{clsparseSuccess, nullptr};
    auto* c = new (std::nothrow) _clsparseControl();
    if (!c) {
        res.status = clsparseOutOfHostMemory;
        return res;
    }
    c->stream = reinterpret_cast<cudaStream_t>(queue);
    if (cudaGetDevice(&c->device) != cudaSuccess) {
        cudaGetLastError();
        delete c;
        res.status = clsparseInvalidDevice;
        return res;
    }
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, c->device) == cudaSuccess) {
        c->sm_count = prop.multiProcessorCount;
        c->l2_bytes = static_cast<size_t>(prop.l2CacheSize);
    }
    if (cudaEventCreateWithFlags(&c->event, cudaEventDisableTiming) != cudaSuccess ||
        cudaStreamCreateWithFlags(&c->capture_stream, cudaStreamNonBlocking) != cudaSuccess ||
        c->reduce_scratch.ensure(sizeof(double) * 4 * kMaxReduceCtas + 256) != cudaSuccess ||
        cudaMallocHost(&c->pinned, 4096) != cudaSuccess) {
        cudaGetLastError();
        delete c;
        res.status = clsparseOutOfResources;
        return res;
    }
    // Tickets live after the partial slots and must start at zero; every
    // reduction leaves them at zero.
    cudaMemsetAsync(c->reduce_scratch.ptr, 0, c->reduce_scratch.bytes, c->stream);
    cudaStreamSynchronize(c->stream);
    if (const char* m = std::getenv("CLSPARSE_B200_SOLVER_LOOP")) c->solver_loop_mode = std::atoi(m);
    res.control = c;
    return res;
}

clsparseStatus clsparseEnableAsync(clsparseControl control, cl_bool async) {
    if (control == nullptr) return clsparseInvalidControlObject;
    control->async = async != 0;
    return clsparseSuccess;
}

clsparseStatus clsparseEnableExtendedPrecision(clsparseControl control, cl_bool ext) {
    if (control == nullptr) return clsparseInvalidControlObject;
    control->extended_precision = ext != 0;
    return clsparseSuccess;
}

clsparseEventResult clsparseGetEvent(clsparseControl control) {
    clsparseEventResult r{clsparseSuccess, nullptr};
    if (control == nullptr) {
        r.status = clsparseInvalidControlObject;
        return r;
    }
    r.event = reinterpret_cast<cl_event>(control->event);
    return r;
}

clsparseStatus clsparseReleaseControl(clsparseControl control) {
    if (control == nullptr) return clsparseInvalidControlObject;
    {
        DeviceGuard g(control->device);
        cudaStreamSynchronize(control->stream);
        control->solver_cache.reset();
        control->mixed_work.reset();
        control->batch_work.reset();
        control->reduce_scratch.release();
        if (control->event) cudaEventDestroy(control->event);
        if (control->capture_stream) cudaStreamDestroy(control->capture_stream);
        if (control->pinned) cudaFreeHost(control->pinned);
    }
    delete control;
    return clsparseSuccess;
}

clsparseStatus clsparseB200SetSolverLoopMode(clsparseControl control, cl_int mode) {
    if (control == nullptr) return clsparseInvalidControlObject;
    if (mode < 0 || mode > 3) return clsparseInvalidValue;
    control->solver_loop_mode = mode;
    return clsparseSuccess;
}

// ---- solver control (reference solvers/solver-control.cpp:20-102) ----

clsparseCreateSolverResult clsparseCreateSolverControl(PRECONDITIONER precond, cl_int maxIters,
                                                       cl_double relTol, cl_double absTol) {
    clsparseCreateSolverResult r{clsparseSuccess, nullptr};
    auto* s = new (std::nothrow) _solverControl();
    if (!s) {
        r.status = clsparseOutOfHostMemory;
        return r;
    }
    s->absoluteTolerance = absTol;
    s->relativeTolerance = relTol;
    s->nIters = 0;
    s->maxIters = maxIters;
    s->initialResidual = 0;
    s->preconditioner = precond;
    r.control = s;
    return r;
}

clsparseStatus clsparseReleaseSolverControl(clSParseSolverControl s) {
    if (s == nullptr) return clsparseInvalidSolverControlObject;
    delete s;
    return clsparseSuccess;
}

clsparseStatus clsparseSetSolverParams(clSParseSolverControl s, PRECONDITIONER precond,
                                       cl_int maxIters, cl_double relTol, cl_double absTol) {
    if (s == nullptr) return clsparseInvalidSolverControlObject;
    s->absoluteTolerance = absTol;
    s->relativeTolerance = relTol;
    s->nIters = 0;
    s->maxIters = maxIters;
    s->initialResidual = 0;
    s->preconditioner = precond;
    return clsparseSuccess;
}

clsparseStatus clsparseSolverPrintMode(clSParseSolverControl s, PRINT_MODE mode) {
    if (s == nullptr) return clsparseInvalidSolverControlObject;
    s->printMode = mode;
    return clsparseSuccess;
}

clsparseStatus clsparseB200SolverGetInfo(clSParseSolverControl s, cl_int* nIters,
                                         cl_double* initialResidual, cl_double* currentResidual) {
    if (s == nullptr) return clsparseInvalidSolverControlObject;
    if (nIters) *nIters = s->nIters;
    if (initialResidual) *initialResidual = s->initialResidual;
    if (currentResidual) *currentResidual = s->currentResidual;
    return clsparseSuccess;
}

clsparseStatus clsparseB200SolverSetHistory(clSParseSolverControl s, cl_double* history, cl_uint capacity) {
    if (s == nullptr) return clsparseInvalidSolverControlObject;
    if (history == nullptr && capacity != 0) return clsparseInvalidValue;
    if (capacity > 0x7fffffffu) return clsparseInvalidSize;
    s->history = history;
    s->historyCapacity = history ? capacity : 0;
    s->historyLength = 0;
    return clsparseSuccess;
}

clsparseStatus clsparseB200SolverGetHistoryLength(clSParseSolverControl s, cl_uint* length) {
    if (s == nullptr) return clsparseInvalidSolverControlObject;
    if (length == nullptr) return clsparseInvalidValue;
    *length = s->historyLength;
    return clsparseSuccess;
}

clsparseStatus clsparseB200SolverSetSnapshots(clSParseSolverControl s, const cl_int* iterations, cl_int count,
                                              void* vectors) {
    if (s == nullptr) return clsparseInvalidSolverControlObject;
    if (count < 0 || count > 8) return clsparseInvalidSize;
    if (count > 0 && (iterations == nullptr || vectors == nullptr)) return clsparseInvalidValue;
    for (int k = 0; k < count; ++k)
        if (iterations[k] < 0) return clsparseInvalidValue;
    s->snapshotCount = count;
    for (int k = 0; k < 8; ++k) s->snapshotIters[k] = k < count ? iterations[k] : -1;
    s->snapshots = count > 0 ? vectors : nullptr;
    return clsparseSuccess;
}

clsparseStatus clsparseB200SolverGetDeviceStatus(clSParseSolverControl s, cl_uint* bits) {
    if (s == nullptr) return clsparseInvalidSolverControlObject;
    if (bits) *bits = s->deviceStatus;
    return clsparseSuccess;
}

// ---- declared, outside the accelerated path ----

clsparseStatus clsparseScsrSpGemm(const clsparseCsrMatrix*, const clsparseCsrMatrix*,
                                  clsparseCsrMatrix*, const clsparseControl) {
    return clsparseNotImplemented;
}

}  // extern "C"
