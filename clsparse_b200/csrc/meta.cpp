// CSR-Adaptive row-block binning and the Meta Size / Create / Delete entry
// points (reference src/library/internal/data-types/csr-meta.{hpp,cpp}).
//
// The binning is a restatement of the reference's ComputeRowBlocks
// (csr-meta.hpp:93-261). The row-block word format is an interface between the
// binning and the SpMV kernel and is kept identical to the reference's so that
// clsparseCsrMetaSize reports the same sizes and the words can be compared bit
// for bit:
//   bits 63..32  first row of the block
//   bit  24      (reference: long-row flag; never set here, the kernel does not
//                 mutate the words)
//   bits 23..0   chunk index inside a long row, or for a block of several short
//                rows the number of threads the reference reduced each row with
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>

#include "internal.h"

namespace clsp {

namespace {

// Threads per row for a block of n short rows in a 256-thread CTA: the largest
// power of two p with p * n <= 256, computed as the reference does
// (csr-meta.hpp:52-68): 256 >> bit_length(n - 1). The argument is truncated to
// 32 bits and the shift count taken modulo 32, matching the x86 build of the
// reference for every row count it can see.
inline uint64_t threads_for_reduction(uint64_t n) {
    const uint32_t v = static_cast<uint32_t>(n - 1);
    const uint32_t bits = v == 0 ? 0u : 32u - static_cast<uint32_t>(__builtin_clz(v));
    return static_cast<uint64_t>(256u >> (bits & 31u));
}

}  // namespace

void compute_row_blocks(cl_ulong* out, clsparseIdx_t& rowBlockSize, const clsparseIdx_t* rp,
                        clsparseIdx_t nRows, uint32_t blkSize, uint32_t blkMultiplier,
                        uint32_t rowsForVector, bool allocate) {
    const uint32_t shift = 64 - kRowBits;
    cl_ulong* base = out;
    size_t words = 1;  // word 0 (row 0) always exists
    if (allocate) {
        *out = 0;
        ++out;
    }
    uint64_t sum = 0;
    uint64_t i = 0, last_i = 0;
    // Length of the current run of long rows; the reference stores it in a
    // 32-bit unsigned and marks "first short row after a long run" with -1.
    uint32_t long_run = 0;
    const uint32_t kRunEnded = 0xFFFFFFFFu;

    auto close_with = [&](uint64_t end_row, uint64_t nrows_in_block, uint64_t nthreads_arg) {
        // Writes the word that ends the current block (= starts the next) and
        // stores the reduction width in the word that started it.
        if (allocate) {
            *out = end_row << shift;
            if (nrows_in_block > rowsForVector) *(out - 1) |= threads_for_reduction(nthreads_arg);
            ++out;
        }
        ++words;
    };

    for (i = 1; i <= nRows; ++i) {
        const uint32_t len = rp[i] - rp[i - 1];
        sum += len;

        // Track transitions between runs of long (>128) and short (<32) rows.
        if (len > 128) {
            ++long_run;
        } else if (long_run > 0) {
            if (len < 32)
                long_run = kRunEnded;
            else
                ++long_run;
        }

        if (long_run == 1) {
            // Entering a long run: end the preceding block of short rows, if any.
            if (i - last_i > 1) {
                close_with(i - 1, (i - 1) - last_i, (i - 1) - last_i);
                last_i = i - 1;
                sum = len;
            }
        } else if (long_run == kRunEnded) {
            // First short row after a long run: end the block there.
            close_with(i - 1, (i - 1) - last_i, (i - 1) - last_i);
            last_i = i - 1;
            sum = len;
            long_run = 0;
        }

        if (i - last_i == 1 && sum > blkSize) {
            // One row longer than a block: vector (one CTA) or long-row chunks.
            const double chunks = std::ceil(static_cast<double>(len) /
                                            static_cast<double>(blkMultiplier * blkSize));
            int need = static_cast<int>(chunks);
            const int cap = 1 << kWgBits;
            need = need < cap ? need : cap;
            if (allocate) {
                for (int w = 1; w < need; ++w) {
                    *out = ((i - 1) << shift) | static_cast<cl_ulong>(w);
                    ++out;
                }
                *out = i << shift;
                ++out;
            }
            words += static_cast<size_t>(need);
            last_i = i;
            sum = 0;
            long_run = 0;
        } else if (i - last_i > 1 && sum > blkSize) {
            // Several rows overflow the block: close before this row and
            // revisit it as the first row of the next block.
            --i;
            close_with(i, i - last_i, i - last_i);
            last_i = i;
            sum = 0;
            long_run = 0;
        } else if (sum == blkSize) {
            close_with(i, i - last_i, i - last_i);
            last_i = i;
            sum = 0;
            long_run = 0;
        }
    }

    // Close the trailing block. The reduction width uses i - last_i with
    // i == nRows + 1, one more than the block's row count (csr-meta.hpp:241-246);
    // kept so the words match.
    if (allocate && ((*(out - 1)) >> shift) != static_cast<cl_ulong>(nRows)) {
        *out = static_cast<cl_ulong>(nRows) << shift;
        if (static_cast<uint64_t>(nRows) - last_i > rowsForVector)
            *(out - 1) |= threads_for_reduction(i - last_i);
        ++out;
    }
    ++words;

    if (allocate)
        rowBlockSize = static_cast<clsparseIdx_t>(2 * static_cast<size_t>(out - base));
    else
        rowBlockSize = static_cast<clsparseIdx_t>(2 * words);
}

namespace {

clsparseStatus read_row_pointer(const clsparseCsrMatrix* A, clsparseControl control,
                                std::vector<clsparseIdx_t>& rp) {
    rp.resize(static_cast<size_t>(A->num_rows) + 1);
    if (A->row_pointer == nullptr) return clsparseInvalidMemObject;
    const clsparseIdx_t* src = dev_ptr<const clsparseIdx_t>(A->row_pointer, A->off_row_pointer);
    cudaError_t e = cudaMemcpyAsync(rp.data(), src, rp.size() * sizeof(clsparseIdx_t),
                                    cudaMemcpyDeviceToHost, control->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(control->stream);
    if (e != cudaSuccess) return clsparseInvalidMemObject;
    for (size_t r = 0; r + 1 < rp.size(); ++r)
        if (rp[r + 1] < rp[r]) return clsparseInvalidValue;
    return clsparseSuccess;
}

}  // namespace

}  // namespace clsp

matrix_meta::~matrix_meta() {
    int prev = -1;
    cudaGetDevice(&prev);
    if (prev != device) cudaSetDevice(device);
    if (d_rowBlocks) cudaFree(d_rowBlocks);
    if (d_word_nnz) cudaFree(d_word_nnz);
    if (d_lr_partial) cudaFree(d_lr_partial);
    if (d_lr_ticket) cudaFree(d_lr_ticket);
    if (d_error) cudaFree(d_error);
    if (prev >= 0 && prev != device) cudaSetDevice(prev);
}

using namespace clsp;

extern "C" {

clsparseMetaSizeResult clsparseCsrMetaSize(clsparseCsrMatrix* csrMatx, clsparseControl control) {
    clsparseMetaSizeResult res{clsparseSuccess, 0};
    if (csrMatx == nullptr) {
        res.status = clsparseInvalidValue;
        return res;
    }
    if (csrMatx->meta) {
        res.metaSize = static_cast<matrix_meta*>(csrMatx->meta)->rowBlockSize;
        return res;
    }
    res.status = check_entry(control);
    if (res.status != clsparseSuccess) return res;
    DeviceGuard g(control->device);
    std::vector<clsparseIdx_t> rp;
    res.status = read_row_pointer(csrMatx, control, rp);
    if (res.status != clsparseSuccess) return res;
    clsparseIdx_t size = 0;
    compute_row_blocks(nullptr, size, rp.data(), csrMatx->num_rows, kBlkSize, kBlockMultiplier,
                       kRowsForVector, false);
    res.metaSize = size;
    return res;
}

clsparseStatus clsparseCsrMetaCreate(clsparseCsrMatrix* csrMatx, clsparseControl control) {
    clsp::TraceRange trace_("clsparseCsrMetaCreate");
    return clsp::create_meta(csrMatx, control, kBlkSize, kBlockMultiplier, kRowsForVector, clsp::default_cta_threads());
}

clsparseStatus clsparseB200CsrMetaCreateTuned(clsparseCsrMatrix* csrMatx, cl_uint blkSize, cl_uint blkMultiplier,
                                              cl_uint rowsForVector, cl_uint ctaThreads, clsparseControl control) {
    if (!((blkSize == 512 && ctaThreads == 128) || ((blkSize == 1024 || blkSize == 2048) && (ctaThreads == 128 || ctaThreads == 256))))
        return clsparseInvalidValue;
    if (blkMultiplier < 1 || blkMultiplier > 64 || rowsForVector < 1 || rowsForVector > 256) return clsparseInvalidValue;
    return clsp::create_meta(csrMatx, control, blkSize, blkMultiplier, rowsForVector, static_cast<int>(ctaThreads));
}

}  // extern "C"

namespace clsp {

int default_cta_threads() {
    static int nt = [] {
        const char* e = std::getenv("CLSPARSE_B200_SPMV_NT");
        return (e && std::atoi(e) == 256) ? 256 : 128;
    }();
    return nt;
}

clsparseStatus create_meta(clsparseCsrMatrix* csrMatx, clsparseControl control, uint32_t blk, uint32_t mult,
                           uint32_t rfv, int nt) {
    clsparseStatus st = check_entry(control);
    if (st != clsparseSuccess) return st;
    if (csrMatx == nullptr) return clsparseInvalidValue;
    DeviceGuard g(control->device);

    std::vector<clsparseIdx_t> rp;
    st = read_row_pointer(csrMatx, control, rp);
    if (st != clsparseSuccess) return st;
    // Structure check before any kernel trusts the matrix: row pointers
    // monotone (read_row_pointer), spanning exactly num_nonzeros entries, and
    // every column index below num_cols (device pass below).
    if (static_cast<size_t>(rp.back() - rp.front()) != static_cast<size_t>(csrMatx->num_nonzeros))
        return clsparseInvalidValue;
    if (csrMatx->num_nonzeros > 0 && csrMatx->col_indices == nullptr) return clsparseInvalidMemObject;

    if (csrMatx->meta) {
        delete static_cast<matrix_meta*>(csrMatx->meta);
        csrMatx->meta = nullptr;
    }

    auto meta = std::make_unique<matrix_meta>();
    meta->device = control->device;
    meta->sm_count = control->sm_count > 0 ? control->sm_count : 148;
    meta->num_rows = csrMatx->num_rows;
    meta->num_nonzeros = csrMatx->num_nonzeros;
    meta->blk_size = blk;
    meta->blk_mult = mult;
    meta->rows_for_vector = rfv;
    meta->cta_threads = nt;
    clsparseIdx_t dry = 0;
    compute_row_blocks(nullptr, dry, rp.data(), csrMatx->num_rows, blk, mult, rfv, false);
    meta->h_rowBlocks.assign(dry / 2 + 1, 0);
    clsparseIdx_t used = dry;
    compute_row_blocks(meta->h_rowBlocks.data(), used, rp.data(), csrMatx->num_rows, blk, mult, rfv, true);
    meta->rowBlockSize = used;
    meta->num_words = used / 2;
    meta->h_rowBlocks.resize(meta->num_words);

    const size_t w = meta->num_words;
    // Nonzero offset of every word's first row, so a CTA finds its range
    // without a dependent row-pointer load.
    std::vector<uint32_t> word_nnz(w);
    for (size_t k = 0; k < w; ++k) word_nnz[k] = rp[static_cast<size_t>(meta->h_rowBlocks[k] >> 32)];
    meta->nnz_lo = rp.front();
    meta->nnz_hi = rp.back();
    for (size_t r = 0; r + 1 < rp.size(); ++r)
        meta->max_row = std::max<uint32_t>(meta->max_row, static_cast<uint32_t>(rp[r + 1] - rp[r]));
    if (cudaMalloc(&meta->d_rowBlocks, w * sizeof(cl_ulong)) != cudaSuccess ||
        cudaMalloc(&meta->d_word_nnz, w * sizeof(uint32_t)) != cudaSuccess ||
        cudaMalloc(&meta->d_lr_partial, w * sizeof(double)) != cudaSuccess ||
        cudaMalloc(&meta->d_lr_ticket, w * sizeof(uint32_t)) != cudaSuccess ||
        cudaMalloc(&meta->d_error, sizeof(int)) != cudaSuccess) {
        cudaGetLastError();
        return clsparseOutOfResources;
    }
    cudaError_t e = cudaMemcpyAsync(meta->d_rowBlocks, meta->h_rowBlocks.data(),
                                    w * sizeof(cl_ulong), cudaMemcpyHostToDevice, control->stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(meta->d_word_nnz, word_nnz.data(), w * sizeof(uint32_t),
                            cudaMemcpyHostToDevice, control->stream);
    if (e == cudaSuccess)
        e = cudaMemsetAsync(meta->d_lr_ticket, 0, w * sizeof(uint32_t), control->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(meta->d_error, 0, sizeof(int), control->stream);
    // column indices of the matrix's entries rp[0] .. rp[n] - 1; the flag
    // borrows the meta's error word, cleared again below
    if (e == cudaSuccess)
        e = launch_validate_columns(dev_ptr<const uint32_t>(csrMatx->col_indices, csrMatx->off_col_indices) + rp.front(),
                                    csrMatx->num_nonzeros, static_cast<uint32_t>(csrMatx->num_cols), meta->d_error,
                                    meta->sm_count, control->stream);
    int bad = 0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&bad, meta->d_error, sizeof(int), cudaMemcpyDeviceToHost, control->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(control->stream);
    if (e != cudaSuccess) return clsparseInvalidKernelExecution;
    if (bad) return clsparseInvalidValue;
    if (cudaMemsetAsync(meta->d_error, 0, sizeof(int), control->stream) != cudaSuccess ||
        cudaStreamSynchronize(control->stream) != cudaSuccess)
        return clsparseInvalidKernelExecution;
    meta->h_word_nnz = std::move(word_nnz);
    csrMatx->meta = meta.release();
    return clsparseSuccess;
}

}  // namespace clsp

extern "C" {

clsparseStatus clsparseCsrMetaCompute(clsparseCsrMatrix* csrMatx, clsparseControl control) {
    return clsparseCsrMetaCreate(csrMatx, control);
}

clsparseStatus clsparseCsrMetaDelete(clsparseCsrMatrix* csrMatx) {
    if (csrMatx == nullptr) return clsparseInvalidValue;
    if (csrMatx->meta == nullptr) return clsparseSuccess;
    delete static_cast<matrix_meta*>(csrMatx->meta);
    csrMatx->meta = nullptr;
    return clsparseSuccess;
}

clsparseStatus clsparseB200ComputeRowBlocksHost(const clsparseIdx_t* rowPointer,
                                                clsparseIdx_t numRows, cl_ulong* rowBlocks,
                                                size_t capacity, clsparseIdx_t* rowBlockSize) {
    if (rowPointer == nullptr || rowBlockSize == nullptr) return clsparseInvalidValue;
    for (clsparseIdx_t r = 0; r < numRows; ++r)
        if (rowPointer[r + 1] < rowPointer[r]) return clsparseInvalidValue;
    clsparseIdx_t dry = 0;
    compute_row_blocks(nullptr, dry, rowPointer, numRows, kBlkSize, kBlockMultiplier,
                       kRowsForVector, false);
    if (rowBlocks == nullptr) {
        *rowBlockSize = dry;
        return clsparseSuccess;
    }
    std::vector<cl_ulong> tmp(dry / 2 + 1, 0);
    clsparseIdx_t used = dry;
    compute_row_blocks(tmp.data(), used, rowPointer, numRows, kBlkSize, kBlockMultiplier,
                       kRowsForVector, true);
    const size_t words = used / 2;
    if (capacity < words) return clsparseInsufficientMemory;
    std::memcpy(rowBlocks, tmp.data(), words * sizeof(cl_ulong));
    *rowBlockSize = used;
    return clsparseSuccess;
}

clsparseStatus clsparseB200CsrMetaGetRowBlocks(const clsparseCsrMatrix* csrMatx,
                                               cl_ulong* rowBlocks, size_t capacity,
                                               size_t* count) {
    if (csrMatx == nullptr || count == nullptr) return clsparseInvalidValue;
    if (csrMatx->meta == nullptr) return clsparseStructInvalid;
    const auto* meta = static_cast<const matrix_meta*>(csrMatx->meta);
    *count = meta->num_words;
    if (rowBlocks == nullptr) return clsparseSuccess;
    if (capacity < meta->num_words) return clsparseInsufficientMemory;
    std::memcpy(rowBlocks, meta->h_rowBlocks.data(), meta->num_words * sizeof(cl_ulong));
    return clsparseSuccess;
}

}  // extern "C"
