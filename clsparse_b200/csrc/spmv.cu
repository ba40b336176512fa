// CSR sparse matrix-vector product y = alpha*A*x + beta*y for sm_100a, and the
// clsparseScsrmv / clsparseDcsrmv entry points.
//
// Two kernels, chosen as the reference chooses (src/library/blas2/clsparse-csrmv.hpp:103-132):
//
// * csr_adaptive_kernel -- with a meta (row-block words from
//   clsparseCsrMetaCreate) one CTA of 128 threads (256 with
//   CLSPARSE_B200_SPMV_NT=256) runs per word, in one of the STREAM / VECTOR /
//   LONG modes of spmv_word.cuh. Long rows are merged through per-word
//   tickets: no CTA waits for another (the reference spin-waits on a flag it
//   flips inside the meta, csrmv_adaptive.cl:596-600), the result does not
//   depend on arrival order, and the meta is left as it was found.
// * csr_vector_kernel -- without a meta, G lanes per row (G = 2..32 from the
//   average row length, as csrmv-vector.hpp:34-49 picks its sub-wave).
//
// beta == 0 overwrites y without reading it on every path (the reference reads
// y on its LONG path; csrmv_adaptive.cl:481-483 skips it on the others).
//
// Both kernels can fuse the dot products a Krylov solver takes of the result
// (<y, w> and <y, y>) and finish them with a deterministic grid reduction.
#include <algorithm>
#include <cstdlib>
#include <string>
#include <type_traits>

#include "device_common.cuh"
#include "internal.h"
#include "pipeline.cuh"
#include "solver_state.cuh"
#include "spmv_word.cuh"

namespace clsp {

namespace {

constexpr int kThreads = 256;

// Resident CTAs per SM the register allocator is held to: the gathers of x
// are latency-bound, so more CTAs in flight pay (measured on the irregular,
// 3D and 2D workloads); FP32 accumulators need fewer registers than FP64.
// CLSP_SPMV_MIN_BLOCKS overrides it at build time (1 leaves it free).
// The fused-dot variants the solvers launch (K > 0) keep more registers;
// the compensated (extended-precision) ones are left free.
template <typename T, bool EXT, int K, int NT>
constexpr int spmv_min_blocks() {
#ifdef CLSP_SPMV_MIN_BLOCKS
    return CLSP_SPMV_MIN_BLOCKS * NT <= 2048 ? CLSP_SPMV_MIN_BLOCKS : 1;
#else
    return EXT ? 1 : (K == 0 ? 12 : (sizeof(T) == 8 ? 10 : 12)) * 128 / NT;
#endif
}

template <typename V, typename T, bool EXT, int K, int NT, int BLK>
__global__ void __launch_bounds__(NT, spmv_min_blocks<T, EXT, K, NT>())
    csr_adaptive_kernel(const V* __restrict__ vals, const uint32_t* __restrict__ cols,
                        const uint32_t* __restrict__ rp, const T* __restrict__ x, T* __restrict__ y,
                        const T* __restrict__ alpha_p, const T* __restrict__ beta_p,
                        const uint64_t* __restrict__ words, const uint32_t* __restrict__ word_nnz,
                        uint32_t nblocks, uint32_t lo, uint32_t hi, int vec,
                        double* __restrict__ lr_partial, uint32_t* __restrict__ lr_ticket, WordShape shape,
                        EpiDev<T> epi) {
    __shared__ WordSmem<T, BLK> sm;
    if (epi.done != nullptr && *epi.done) return;
    const T alpha = *alpha_p;
    RowSink<T, K> sink;
    sink.init(y, epi, *beta_p);
    if (blockIdx.x < nblocks)
        adaptive_word<V, T, EXT, NT, BLK>(blockIdx.x, vals, cols, rp, DenseX<T>{x}, alpha, words, word_nnz, lo,
                                          hi, vec, lr_partial, lr_ticket, shape, sm, sink);
    run_epilogue<T, K>(sink, epi);
}

template <typename V, typename T, bool EXT, int G, int K>
__global__ void __launch_bounds__(kThreads)
    csr_vector_kernel(const V* __restrict__ vals, const uint32_t* __restrict__ cols,
                      const uint32_t* __restrict__ rp, const T* __restrict__ x, T* __restrict__ y,
                      const T* __restrict__ alpha_p, const T* __restrict__ beta_p, uint32_t nrows,
                      EpiDev<T> epi) {
    if (epi.done != nullptr && *epi.done) return;
    const T alpha = *alpha_p;
    RowSink<T, K> sink;
    sink.init(y, epi, *beta_p);
    const uint32_t lane = threadIdx.x & (G - 1);
    const uint64_t gtid = static_cast<uint64_t>(blockIdx.x) * kThreads + threadIdx.x;
    const uint32_t grp = static_cast<uint32_t>(gtid / G);
    const uint32_t ngroups = static_cast<uint32_t>(static_cast<uint64_t>(gridDim.x) * kThreads / G);
    for (uint32_t base = 0; base < nrows; base += ngroups) {
        const uint32_t row = base + grp;
        dev::Acc<T, EXT> a;
        if (row < nrows) {
            const uint32_t nb = dev::ld_ro(rp + row);
            const uint32_t ne = dev::ld_ro(rp + row + 1);
            if constexpr (G == 1) {
                // one thread per row: neighbours share lines, keep them in L1
#pragma unroll 4
                for (uint32_t j = nb; j < ne; ++j)
                    a.add_prod(alpha * dev::ld_val_ro<T>(vals + j), dev::ld_ro(x + dev::ld_ro(cols + j)));
            } else {
                for (uint32_t j = nb + lane; j < ne; j += G)
                    a.add_prod(alpha * dev::ld_val<T>(vals + j), dev::ld_ro(x + dev::ld_stream(cols + j)));
            }
        }
        dev::group_reduce<G>(a);
        if (row < nrows && lane == 0) sink.template put<EXT>(row, a);
        if (base > 0xFFFFFFFFu - ngroups) break;
    }
    run_epilogue<T, K>(sink, epi);
}

template <typename T>
EpiDev<T> to_dev(const SpmvEpilogue& e) {
    EpiDev<T> d;
    d.w0 = static_cast<const T*>(e.w0);
    d.dot1_self = e.dot1_self ? 1 : 0;
    d.partials = e.partials;
    d.ticket = e.ticket;
    d.op = static_cast<int>(e.op);
    d.state = e.state;
    d.cond = e.cond;
    d.done = e.done;
    return d;
}

// Sub-warp width of the vector kernel from the average row length
// (reference blas2/csrmv-vector.hpp:34-49 with a 32-wide warp).
uint32_t vector_width(uint32_t nrows, uint32_t nnz) {
    const uint32_t per_row = nrows ? nnz / nrows : 0;
    uint32_t g = 32;
    if (per_row < 32) g = 16;
    if (per_row < 16) g = 8;
    if (per_row < 8) g = 4;
    if (per_row < 4) g = 2;
    return g;
}

uint32_t vector_grid(uint32_t nrows, uint32_t g) {
    const uint64_t threads = static_cast<uint64_t>(nrows) * g;
    uint64_t ctas = (threads + kThreads - 1) / kThreads;
    if (ctas == 0) ctas = 1;
    if (ctas > 0x7fffffffull) ctas = 0x7fffffffull;
    return static_cast<uint32_t>(ctas);
}

template <typename V, typename T, bool EXT, int K>
cudaError_t launch_vector(const CsrView<V>& A, const T* alpha, const T* beta, const T* x, T* y,
                          const EpiDev<T>& e, cudaStream_t s) {
    const uint32_t g = vector_width(A.nrows, A.nnz);
    const uint32_t grid = vector_grid(A.nrows, g);
#define CLSP_VEC(GW)                                                                              \
    csr_vector_kernel<V, T, EXT, GW, K><<<grid, kThreads, 0, s>>>(A.vals, A.cols, A.rp, x, y, alpha, \
                                                               beta, A.nrows, e)
    switch (g) {
        case 2: CLSP_VEC(2); break;
        case 4: CLSP_VEC(4); break;
        case 8: CLSP_VEC(8); break;
        case 16: CLSP_VEC(16); break;
        default: CLSP_VEC(32); break;
    }
#undef CLSP_VEC
    return cudaGetLastError();
}

#include "spmv_tma.cuh"

// Adaptive kernel choice: one CTA per row block (default) or the TMA-staged
// persistent pipeline (CLSPARSE_B200_SPMV_KERNEL=tma, default row-block shape
// only), which measured slower on the irregular workload (its per-block
// barriers leave too little work in flight per SM).
bool use_tma_kernel() {
    static bool on = [] {
        const char* e = std::getenv("CLSPARSE_B200_SPMV_KERNEL");
        return e && std::string(e) == "tma";
    }();
    return on;
}

template <typename V, typename T, bool EXT, int K>
cudaError_t launch_tma(const CsrView<V>& A, const T* alpha, const T* beta, const T* x, T* y,
                       const EpiDev<T>& e, cudaStream_t s, int* err) {
    using L = tma::Layout<V, T>;
    auto kern = tma::csr_adaptive_tma_kernel<V, T, EXT, K>;
    static int blocks_per_sm = -1;
    static int sms = 0;
    if (blocks_per_sm < 0) {
        cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(L::total));
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        int b = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, kern, tma::kThreads, L::total);
        blocks_per_sm = b > 0 ? b : 1;
    }
    const matrix_meta* m = A.meta;
    const uint32_t nblocks = static_cast<uint32_t>(m->num_words - 1);
    uint64_t grid = static_cast<uint64_t>(sms) * blocks_per_sm;
    if (grid > nblocks) grid = nblocks;
    if (grid == 0) grid = 1;
    const int aligned = ((reinterpret_cast<uintptr_t>(A.vals) | reinterpret_cast<uintptr_t>(A.cols) |
                          reinterpret_cast<uintptr_t>(A.rp)) & 15u) == 0;
    kern<<<static_cast<uint32_t>(grid), tma::kThreads, L::total, s>>>(
        A.vals, A.cols, A.rp, x, y, alpha, beta, m->d_rowBlocks, m->d_word_nnz, nblocks, A.nrows,
        m->nnz_hi, aligned, m->d_lr_partial, m->d_lr_ticket, err, e);
    return cudaGetLastError();
}

template <typename V, typename T, bool EXT, int K, int NT, int BLK>
void launch_adaptive(const CsrView<V>& A, const T* alpha, const T* beta, const T* x, T* y, const EpiDev<T>& e,
                     uint32_t grid, uint32_t nblocks, int vec, cudaStream_t s) {
    const matrix_meta* m = A.meta;
    const WordShape shape{m->rows_for_vector, m->blk_size * m->blk_mult};
    csr_adaptive_kernel<V, T, EXT, K, NT, BLK><<<grid, NT, 0, s>>>(
        A.vals, A.cols, A.rp, x, y, alpha, beta, m->d_rowBlocks, m->d_word_nnz, nblocks, m->nnz_lo, m->nnz_hi,
        vec, m->d_lr_partial, m->d_lr_ticket, shape, e);
}

// Matrices whose rows are all short (at most kShortRow nonzeros: stencils,
// the learned factor's tril(A)) run one thread per row. Every row then costs
// one dependent chain of loads, with many rows in flight per SM, where the
// row-block kernel stages blocks through shared memory; measured on the
// 1024^2 five-point matrix (FP32): 14.4 us against 17.6 us.
// CLSPARSE_B200_SHORT_ROWS=0 keeps the row-block kernel.
constexpr uint32_t kShortRow = 16;

bool short_rows_enabled() {
    const char* e = std::getenv("CLSPARSE_B200_SHORT_ROWS");  // read per launch (tests switch it)
    return !(e && e[0] == '0' && e[1] == '\0');
}

bool use_short_rows(const matrix_meta* m) {
    return short_rows_enabled() && m->num_rows > 0 && m->max_row <= kShortRow;
}

// Grid of the short-row path: one thread per row, capped at one wave of
// resident CTAs (8 of 256 threads per SM), so that each thread walks several
// rows and every CTA pays the fused epilogue's reduction tail (block sum,
// ticket) once rather than once per wave. Measured on the 1024^2 GRF matrix
// (4096 CTAs uncapped, 1184 capped): FP64 Jacobi-CG 317.5 -> 265.5 ms, mixed
// 305 -> 240 ms, learned + mixed 335 -> 264 ms; 128^3 CG 57.8 -> 50.9 ms; the
// plain SpMV is unchanged (12.5 us FP32). CLSPARSE_B200_SHORT_WAVES = W sets W
// waves (0: no cap).
uint32_t short_rows_grid(const matrix_meta* m, uint32_t nrows) {
    uint32_t g = vector_grid(nrows, 1);
    const char* e = std::getenv("CLSPARSE_B200_SHORT_WAVES");
    const int w = e ? std::atoi(e) : 1;
    if (w > 0) g = std::min<uint32_t>(g, static_cast<uint32_t>(m->sm_count) * 8u * static_cast<uint32_t>(w));
    return g;
}

template <typename V, typename T, bool EXT, int K>
void launch_row_per_thread(const CsrView<V>& A, const T* alpha, const T* beta, const T* x, T* y,
                           const EpiDev<T>& e, cudaStream_t s) {
    csr_vector_kernel<V, T, EXT, 1, K><<<short_rows_grid(A.meta, A.nrows), kThreads, 0, s>>>(
        A.vals, A.cols, A.rp, x, y, alpha, beta, A.nrows, e);
}

template <typename V, typename T, bool EXT, int K>
cudaError_t launch_kind(const CsrView<V>& A, const T* alpha, const T* beta, const T* x, T* y,
                        const EpiDev<T>& e, cudaStream_t s) {
    if (A.meta == nullptr) return launch_vector<V, T, EXT, K>(A, alpha, beta, x, y, e, s);
    const matrix_meta* m = A.meta;
    if (use_short_rows(m)) {
        // one thread per row: the vector kernel with one lane
        launch_row_per_thread<V, T, EXT, K>(A, alpha, beta, x, y, e, s);
        return cudaGetLastError();
    }
    const uint32_t nblocks = static_cast<uint32_t>(m->num_words - 1);
    uint32_t grid = nblocks;
    if (grid == 0) {
        if (K == 0) return cudaSuccess;
        grid = 1;  // one idle CTA still finishes the fused reduction
    }
    if (use_tma_kernel() && meta_is_default_shape(m))
        return launch_tma<V, T, EXT, K>(A, alpha, beta, x, y, e, s, m->d_error);
    const int vec = ((reinterpret_cast<uintptr_t>(A.vals) | reinterpret_cast<uintptr_t>(A.cols)) & 15u) == 0;
    // Row-block shapes with kernels: BLKSIZE 512 (128 threads), 1024 and 2048
    // (128 or 256 threads); meta creation accepts no other.
    const int nt = m->cta_threads;
    switch (m->blk_size) {
        case 512: launch_adaptive<V, T, EXT, K, 128, 512>(A, alpha, beta, x, y, e, grid, nblocks, vec, s); break;
        case 2048:
            if (nt == 256)
                launch_adaptive<V, T, EXT, K, 256, 2048>(A, alpha, beta, x, y, e, grid, nblocks, vec, s);
            else
                launch_adaptive<V, T, EXT, K, 128, 2048>(A, alpha, beta, x, y, e, grid, nblocks, vec, s);
            break;
        default:
            if (nt == 256)
                launch_adaptive<V, T, EXT, K, 256, 1024>(A, alpha, beta, x, y, e, grid, nblocks, vec, s);
            else
                launch_adaptive<V, T, EXT, K, 128, 1024>(A, alpha, beta, x, y, e, grid, nblocks, vec, s);
    }
    return cudaGetLastError();
}

}  // namespace

uint32_t spmv_num_ctas(const matrix_meta* meta, uint32_t nrows, uint32_t nnz) {
    if (meta && use_short_rows(meta)) return short_rows_grid(meta, nrows);
    if (meta) return std::max<uint32_t>(1u, static_cast<uint32_t>(meta->num_words - 1));
    return vector_grid(nrows, vector_width(nrows, nnz));
}

template <typename V, typename T>
cudaError_t launch_csrmv(const CsrView<V>& A, const T* alpha, const T* beta, const T* x, T* y,
                         bool extended, const SpmvEpilogue& epi, cudaStream_t s) {
    const EpiDev<T> e = to_dev<T>(epi);
    if (extended) {
        if (epi.ndots == 0) return launch_kind<V, T, true, 0>(A, alpha, beta, x, y, e, s);
        if (epi.ndots == 1) return launch_kind<V, T, true, 1>(A, alpha, beta, x, y, e, s);
        return launch_kind<V, T, true, 2>(A, alpha, beta, x, y, e, s);
    }
    if (epi.ndots == 0) return launch_kind<V, T, false, 0>(A, alpha, beta, x, y, e, s);
    if (epi.ndots == 1) return launch_kind<V, T, false, 1>(A, alpha, beta, x, y, e, s);
    return launch_kind<V, T, false, 2>(A, alpha, beta, x, y, e, s);
}

template cudaError_t launch_csrmv<float, float>(const CsrView<float>&, const float*, const float*,
                                                const float*, float*, bool, const SpmvEpilogue&,
                                                cudaStream_t);
template cudaError_t launch_csrmv<double, double>(const CsrView<double>&, const double*,
                                                  const double*, const double*, double*, bool,
                                                  const SpmvEpilogue&, cudaStream_t);
template cudaError_t launch_csrmv<__nv_bfloat16, float>(const CsrView<__nv_bfloat16>&, const float*,
                                                        const float*, const float*, float*, bool,
                                                        const SpmvEpilogue&, cudaStream_t);

namespace {

template <typename T>
clsparseStatus csrmv_entry(const clsparseScalar* alpha, const clsparseCsrMatrix* A,
                           const cldenseVector* x, const clsparseScalar* beta, cldenseVector* y,
                           clsparseControl control) {
    clsparseStatus st = check_entry(control);
    if (st != clsparseSuccess) return st;
    if (!alpha || !A || !x || !beta || !y) return clsparseInvalidValue;
    if (x->num_values < A->num_cols || y->num_values < A->num_rows) return clsparseInvalidSize;
    if (A->num_rows == 0) return clsparseSuccess;
    if (!alpha->value || !beta->value || !x->values || !y->values || !A->row_pointer ||
        (A->num_nonzeros > 0 && (!A->values || !A->col_indices)))
        return clsparseInvalidMemObject;
    const auto* meta = static_cast<const matrix_meta*>(A->meta);
    if (meta && meta->rowBlockSize == 0) return clsparseStructInvalid;
    if (meta && meta->num_rows != A->num_rows) return clsparseStructInvalid;
    DeviceGuard g(control->device);
    CsrView<T> v{dev_ptr<const T>(A->values, A->off_values),
                 dev_ptr<const uint32_t>(A->col_indices, A->off_col_indices),
                 dev_ptr<const uint32_t>(A->row_pointer, A->off_row_pointer),
                 A->num_rows, A->num_cols, A->num_nonzeros, meta};
    SpmvEpilogue none;
    cudaError_t e = launch_csrmv<T, T>(v, dev_ptr<const T>(alpha->value, alpha->off_value),
                                    dev_ptr<const T>(beta->value, beta->off_value),
                                    dev_ptr<const T>(x->values, x->off_values),
                                    dev_ptr<T>(y->values, y->off_values), control->extended_precision,
                                    none, control->stream);
    if (e != cudaSuccess) return clsparseInvalidKernelExecution;
    return finish_call(control);
}

}  // namespace

// Column-range check of a CSR matrix: sets *bad when any of the n column
// indices is >= ncols. One pass over the indices (16-byte loads where the
// buffer is aligned), one flag write per CTA at most.
__global__ void __launch_bounds__(256) validate_columns_kernel(const uint32_t* __restrict__ cols, size_t n,
                                                               uint32_t ncols, int* bad) {
    const size_t stride = static_cast<size_t>(gridDim.x) * blockDim.x;
    const size_t tid = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    bool out = false;
    const size_t head = ((16 - (reinterpret_cast<uintptr_t>(cols) & 15u)) & 15u) / 4;
    const size_t h = head < n ? head : n;
    for (size_t i = tid; i < h; i += stride) out |= cols[i] >= ncols;
    const uint4* q = reinterpret_cast<const uint4*>(cols + h);
    const size_t nq = (n - h) / 4;
    for (size_t i = tid; i < nq; i += stride) {
        const uint4 c = __ldcs(q + i);
        out |= (c.x >= ncols) | (c.y >= ncols) | (c.z >= ncols) | (c.w >= ncols);
    }
    for (size_t i = h + 4 * nq + tid; i < n; i += stride) out |= cols[i] >= ncols;
    if (__syncthreads_or(out) && threadIdx.x == 0) atomicOr(bad, 1);
}

cudaError_t launch_validate_columns(const uint32_t* cols, size_t n, uint32_t ncols, int* bad, int sm_count,
                                    cudaStream_t s) {
    if (n == 0) return cudaSuccess;
    size_t grid = (n / 4 + 255) / 256;
    const size_t cap = static_cast<size_t>(sm_count > 0 ? sm_count : 148) * 8;
    if (grid > cap) grid = cap;
    if (grid == 0) grid = 1;
    validate_columns_kernel<<<static_cast<uint32_t>(grid), 256, 0, s>>>(cols, n, ncols, bad);
    return cudaGetLastError();
}

}  // namespace clsp

extern "C" {

clsparseStatus clsparseScsrmv(const clsparseScalar* alpha, const clsparseCsrMatrix* matx,
                              const cldenseVector* x, const clsparseScalar* beta, cldenseVector* y,
                              const clsparseControl control) {
    clsp::TraceRange trace_("clsparseScsrmv");
    return clsp::csrmv_entry<float>(alpha, matx, x, beta, y, control);
}

clsparseStatus clsparseDcsrmv(const clsparseScalar* alpha, const clsparseCsrMatrix* matx,
                              const cldenseVector* x, const clsparseScalar* beta, cldenseVector* y,
                              const clsparseControl control) {
    clsp::TraceRange trace_("clsparseDcsrmv");
    return clsp::csrmv_entry<double>(alpha, matx, x, beta, y, control);
}

}  // extern "C"
