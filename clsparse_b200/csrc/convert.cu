// Format conversions (reference src/library/transform/): clsparse{S,D}coo2csr,
// csr2coo, csr2dense and dense2csr; and the COO SpMV clsparse{S,D}coomv, which
// the reference declares (src/include/clSPARSE.h:1106-1132) but never defines.
//
// * coo2csr (clsparse-coo2csr.cpp:20-100): the COO must be sorted by row
//   (the reference's precondition); columns and values are copied and
//   row_pointer[r] is the first position whose row index is >= r, found by a
//   binary search per row (no atomics, no scan; empty rows come out right,
//   which the reference's reduce-by-key of present keys does not guarantee).
// * csr2coo (clsparse-csr2coo.cpp): columns and values copied, each row's
//   positions get its row index (one warp per row).
// * csr2dense (clsparse-csr2dense.cpp): the dense matrix is zeroed, then every
//   entry is written at its (row, column); duplicates: the last one wins.
// * dense2csr (clsparse-dense2csr.cpp): every non-zero of the dense matrix,
//   row by row and column by column; counts per row (warp ballots), an
//   exclusive scan into the row pointer, then an ordered per-row compaction.
//   The CSR buffers must hold the non-zeros (at most rows x columns); the
//   struct's sizes are set.
// Dense matrices: row-major as the reference reads them, column-major
// honoured, lead_dim as given (0 means packed).
#include "device_common.cuh"
#include "scan.cuh"
#include "internal.h"

namespace clsp {
namespace {

constexpr int kThreads = 256;

uint32_t grid_for(uint64_t work, int sms) {
    uint64_t g = (work + kThreads - 1) / kThreads;
    const uint64_t cap = static_cast<uint64_t>(sms) * 32;
    if (g > cap) g = cap;
    return static_cast<uint32_t>(g ? g : 1);
}

struct Dense {
    size_t ld;
    bool cm;
    __device__ __forceinline__ size_t at(size_t r, size_t c) const { return cm ? c * ld + r : r * ld + c; }
};

Dense dense_view(const cldenseMatrix* D) {
    const bool cm = D->major == columnMajor;
    size_t ld = D->lead_dim;
    if (ld == 0) ld = cm ? D->num_rows : D->num_cols;
    return Dense{ld, cm};
}

bool dense_ok(const cldenseMatrix* D) {
    const Dense v = dense_view(D);
    return v.ld >= (v.cm ? D->num_rows : D->num_cols);
}

__global__ void rows_to_offsets_kernel(const uint32_t* __restrict__ ri, uint32_t nnz, uint32_t nrows,
                                       uint32_t* __restrict__ rp) {
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    for (uint64_t r = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; r <= nrows; r += stride) {
        uint32_t lo = 0, hi = nnz;  // first k with ri[k] >= r
        while (lo < hi) {
            const uint32_t mid = lo + (hi - lo) / 2;
            if (ri[mid] < r)
                lo = mid + 1;
            else
                hi = mid;
        }
        rp[r] = r == nrows ? nnz : lo;
    }
}

__global__ void offsets_to_rows_kernel(const uint32_t* __restrict__ rp, uint32_t nrows, uint32_t* __restrict__ ri) {
    const int lane = threadIdx.x & 31;
    const uint64_t warp = (static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    const uint64_t nwarps = (static_cast<uint64_t>(gridDim.x) * blockDim.x) >> 5;
    for (uint64_t r = warp; r < nrows; r += nwarps)
        for (uint32_t k = rp[r] + lane; k < rp[r + 1]; k += 32) ri[k] = static_cast<uint32_t>(r);
}

template <typename T>
__global__ void zero_dense_kernel(T* __restrict__ D, Dense dv, uint32_t rows, uint32_t cols) {
    const uint64_t total = static_cast<uint64_t>(rows) * cols;
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < total; i += stride) {
        const uint64_t major = dv.cm ? i / rows : i / cols, minor = dv.cm ? i % rows : i % cols;
        D[major * dv.ld + minor] = T(0);
    }
}

template <typename T>
__global__ void scatter_dense_kernel(const uint32_t* __restrict__ rp, const uint32_t* __restrict__ cols,
                                     const T* __restrict__ vals, uint32_t nrows, T* __restrict__ D, Dense dv) {
    // one thread per row, entries in order: the last duplicate wins
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    for (uint64_t r = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; r < nrows; r += stride)
        for (uint32_t k = rp[r]; k < rp[r + 1]; ++k) D[dv.at(r, cols[k])] = vals[k];
}

template <typename T>
__global__ void count_rows_kernel(const T* __restrict__ D, Dense dv, uint32_t rows, uint32_t cols,
                                  uint32_t* __restrict__ cnt) {
    const int lane = threadIdx.x & 31;
    const uint64_t warp = (static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    const uint64_t nwarps = (static_cast<uint64_t>(gridDim.x) * blockDim.x) >> 5;
    for (uint64_t r = warp; r < rows; r += nwarps) {
        uint32_t c = 0;
        for (uint32_t j0 = 0; j0 < cols; j0 += 32) {
            const uint32_t j = j0 + lane;
            const bool nz = j < cols && D[dv.at(r, j)] != T(0);
            c += __popc(__ballot_sync(0xffffffffu, nz));
        }
        if (lane == 0) cnt[r] = c;
    }
}

template <typename T>
__global__ void compact_rows_kernel(const T* __restrict__ D, Dense dv, uint32_t rows, uint32_t cols,
                                    const uint32_t* __restrict__ rp, uint32_t* __restrict__ ocols,
                                    T* __restrict__ ovals) {
    const int lane = threadIdx.x & 31;
    const uint64_t warp = (static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    const uint64_t nwarps = (static_cast<uint64_t>(gridDim.x) * blockDim.x) >> 5;
    for (uint64_t r = warp; r < rows; r += nwarps) {
        uint32_t pos = rp[r];
        for (uint32_t j0 = 0; j0 < cols; j0 += 32) {
            const uint32_t j = j0 + lane;
            const T v = j < cols ? D[dv.at(r, j)] : T(0);
            const unsigned ball = __ballot_sync(0xffffffffu, v != T(0));
            if (v != T(0)) {
                const uint32_t k = pos + __popc(ball & ((1u << lane) - 1u));
                ocols[k] = j;
                ovals[k] = v;
            }
            pos += __popc(ball);
        }
    }
}

// y = alpha * A * x + beta * y for a COO matrix sorted by row: G lanes per
// row find the row's entries [lower_bound(r), lower_bound(r + 1)) in the
// sorted row indices and reduce them (duplicates are summed); beta == 0
// overwrites y without reading it.
__device__ __forceinline__ uint32_t lower_bound_u32(const uint32_t* __restrict__ a, uint32_t n, uint32_t key) {
    uint32_t lo = 0, hi = n;
    while (lo < hi) {
        const uint32_t mid = lo + (hi - lo) / 2;
        if (__ldg(a + mid) < key)
            lo = mid + 1;
        else
            hi = mid;
    }
    return lo;
}

template <typename T, int G>
__global__ void __launch_bounds__(kThreads)
    coomv_kernel(const uint32_t* __restrict__ ri, const uint32_t* __restrict__ ci, const T* __restrict__ vals,
                 uint32_t nnz, uint32_t nrows, const T* __restrict__ alpha_p, const T* __restrict__ x,
                 const T* __restrict__ beta_p, T* __restrict__ y) {
    const T alpha = *alpha_p, beta = *beta_p;
    const uint32_t lane = threadIdx.x & (G - 1);
    const uint64_t group = (static_cast<uint64_t>(blockIdx.x) * kThreads + threadIdx.x) / G;
    const uint64_t ngroups = static_cast<uint64_t>(gridDim.x) * kThreads / G;
    // every lane of the warp runs the same trips (the loop bound does not
    // depend on the group), so the full-warp shuffles below are uniform
    for (uint64_t base = 0; base < nrows; base += ngroups) {
        const uint64_t r = base + group;
        T acc = T(0);
        if (r < nrows) {
            const uint32_t lo = lower_bound_u32(ri, nnz, static_cast<uint32_t>(r));
            const uint32_t hi = lower_bound_u32(ri, nnz, static_cast<uint32_t>(r) + 1);
            for (uint32_t k = lo + lane; k < hi; k += G) acc = dev::fma_rn(alpha * vals[k], __ldg(x + ci[k]), acc);
        }
#pragma unroll
        for (int off = G / 2; off > 0; off >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, off, G);
        if (r < nrows && lane == 0) y[r] = beta == T(0) ? acc : acc + beta * y[r];
    }
}

template <typename T>
clsparseStatus coomv(const clsparseScalar* alpha, const clsparseCooMatrix* A, const cldenseVector* x,
                     const clsparseScalar* beta, cldenseVector* y, clsparseControl control) {
    clsparseStatus st = check_entry(control);
    if (st != clsparseSuccess) return st;
    if (!alpha || !A || !x || !beta || !y) return clsparseInvalidValue;
    if (x->num_values < A->num_cols || y->num_values < A->num_rows) return clsparseInvalidSize;
    if (A->num_rows == 0) return clsparseSuccess;
    if (!alpha->value || !beta->value || !x->values || !y->values ||
        (A->num_nonzeros && (!A->values || !A->col_indices || !A->row_indices)))
        return clsparseInvalidMemObject;
    DeviceGuard g(control->device);
    constexpr int G = 8;
    // every lane of a warp runs the same number of rows: whole warps per CTA
    coomv_kernel<T, G><<<grid_for(static_cast<uint64_t>(A->num_rows) * G, control->sm_count), kThreads, 0,
                         control->stream>>>(
        dev_ptr<const uint32_t>(A->row_indices, A->off_row_indices),
        dev_ptr<const uint32_t>(A->col_indices, A->off_col_indices), dev_ptr<const T>(A->values, A->off_values),
        static_cast<uint32_t>(A->num_nonzeros), static_cast<uint32_t>(A->num_rows),
        dev_ptr<const T>(alpha->value, alpha->off_value), dev_ptr<const T>(x->values, x->off_values),
        dev_ptr<const T>(beta->value, beta->off_value), dev_ptr<T>(y->values, y->off_values));
    if (cudaGetLastError() != cudaSuccess) return clsparseInvalidKernelExecution;
    return finish_call(control);
}

bool check_ptrs(const void* a, const void* b, const void* c, size_t n) {
    return n == 0 || (a && b && c);
}

template <typename T>
clsparseStatus coo2csr(const clsparseCooMatrix* coo, clsparseCsrMatrix* csr, clsparseControl control) {
    clsparseStatus st = check_entry(control);
    if (st != clsparseSuccess) return st;
    if (!coo || !csr) return clsparseInvalidValue;
    if (!csr->row_pointer || !check_ptrs(coo->values, coo->col_indices, coo->row_indices, coo->num_nonzeros) ||
        !check_ptrs(csr->values, csr->col_indices, csr->row_pointer, coo->num_nonzeros))
        return clsparseInvalidMemObject;
    DeviceGuard g(control->device);
    csr->num_rows = coo->num_rows;
    csr->num_cols = coo->num_cols;
    csr->num_nonzeros = coo->num_nonzeros;
    cudaStream_t s = control->stream;
    const size_t nnz = coo->num_nonzeros;
    if (nnz) {
        cudaMemcpyAsync(dev_ptr<uint32_t>(csr->col_indices, csr->off_col_indices),
                        dev_ptr<const uint32_t>(coo->col_indices, coo->off_col_indices), nnz * 4,
                        cudaMemcpyDeviceToDevice, s);
        cudaMemcpyAsync(dev_ptr<T>(csr->values, csr->off_values), dev_ptr<const T>(coo->values, coo->off_values),
                        nnz * sizeof(T), cudaMemcpyDeviceToDevice, s);
    }
    rows_to_offsets_kernel<<<grid_for(static_cast<uint64_t>(coo->num_rows) + 1, control->sm_count), kThreads, 0, s>>>(
        dev_ptr<const uint32_t>(coo->row_indices, coo->off_row_indices), static_cast<uint32_t>(nnz),
        static_cast<uint32_t>(coo->num_rows), dev_ptr<uint32_t>(csr->row_pointer, csr->off_row_pointer));
    if (cudaGetLastError() != cudaSuccess) return clsparseInvalidKernelExecution;
    return finish_call(control);
}

template <typename T>
clsparseStatus csr2coo(const clsparseCsrMatrix* csr, clsparseCooMatrix* coo, clsparseControl control) {
    clsparseStatus st = check_entry(control);
    if (st != clsparseSuccess) return st;
    if (!coo || !csr) return clsparseInvalidValue;
    if (!csr->row_pointer || !check_ptrs(coo->values, coo->col_indices, coo->row_indices, csr->num_nonzeros) ||
        !check_ptrs(csr->values, csr->col_indices, csr->row_pointer, csr->num_nonzeros))
        return clsparseInvalidMemObject;
    DeviceGuard g(control->device);
    coo->num_rows = csr->num_rows;
    coo->num_cols = csr->num_cols;
    coo->num_nonzeros = csr->num_nonzeros;
    cudaStream_t s = control->stream;
    const size_t nnz = csr->num_nonzeros;
    if (nnz) {
        cudaMemcpyAsync(dev_ptr<uint32_t>(coo->col_indices, coo->off_col_indices),
                        dev_ptr<const uint32_t>(csr->col_indices, csr->off_col_indices), nnz * 4,
                        cudaMemcpyDeviceToDevice, s);
        cudaMemcpyAsync(dev_ptr<T>(coo->values, coo->off_values), dev_ptr<const T>(csr->values, csr->off_values),
                        nnz * sizeof(T), cudaMemcpyDeviceToDevice, s);
        offsets_to_rows_kernel<<<grid_for(static_cast<uint64_t>(csr->num_rows) * 32, control->sm_count), kThreads,
                                 0, s>>>(dev_ptr<const uint32_t>(csr->row_pointer, csr->off_row_pointer),
                                         static_cast<uint32_t>(csr->num_rows),
                                         dev_ptr<uint32_t>(coo->row_indices, coo->off_row_indices));
    }
    if (cudaGetLastError() != cudaSuccess) return clsparseInvalidKernelExecution;
    return finish_call(control);
}

template <typename T>
clsparseStatus csr2dense(const clsparseCsrMatrix* csr, cldenseMatrix* A, clsparseControl control) {
    clsparseStatus st = check_entry(control);
    if (st != clsparseSuccess) return st;
    if (!csr || !A) return clsparseInvalidValue;
    if (A->num_rows < csr->num_rows || A->num_cols < csr->num_cols || !dense_ok(A)) return clsparseInvalidSize;
    if (!A->values || !csr->row_pointer || (csr->num_nonzeros && (!csr->values || !csr->col_indices)))
        return clsparseInvalidMemObject;
    DeviceGuard g(control->device);
    cudaStream_t s = control->stream;
    const Dense dv = dense_view(A);
    T* D = dev_ptr<T>(A->values, A->off_values);
    const uint32_t rows = A->num_rows, cols = A->num_cols;
    zero_dense_kernel<T><<<grid_for(static_cast<uint64_t>(rows) * cols, control->sm_count), kThreads, 0, s>>>(
        D, dv, rows, cols);
    scatter_dense_kernel<T><<<grid_for(csr->num_rows, control->sm_count), kThreads, 0, s>>>(
        dev_ptr<const uint32_t>(csr->row_pointer, csr->off_row_pointer),
        dev_ptr<const uint32_t>(csr->col_indices, csr->off_col_indices), dev_ptr<const T>(csr->values, csr->off_values),
        static_cast<uint32_t>(csr->num_rows), D, dv);
    if (cudaGetLastError() != cudaSuccess) return clsparseInvalidKernelExecution;
    return finish_call(control);
}

template <typename T>
clsparseStatus dense2csr(const cldenseMatrix* A, clsparseCsrMatrix* csr, clsparseControl control) {
    clsparseStatus st = check_entry(control);
    if (st != clsparseSuccess) return st;
    if (!csr || !A) return clsparseInvalidValue;
    if (!dense_ok(A)) return clsparseInvalidSize;
    if (!A->values || !csr->row_pointer || !csr->values || !csr->col_indices) return clsparseInvalidMemObject;
    const uint32_t rows = A->num_rows, cols = A->num_cols;
    const uint32_t nparts = (rows + 1023) / 1024;
    // the block totals use the partial-sum slots of the control's reduction
    // scratch (its tickets lie after them): at most 16.7 M rows
    if (static_cast<size_t>(nparts) * 4 > static_cast<size_t>(kMaxReduceCtas) * 4 * sizeof(double))
        return clsparseInvalidSize;
    DeviceGuard g(control->device);
    cudaStream_t s = control->stream;
    const Dense dv = dense_view(A);
    const T* D = dev_ptr<const T>(A->values, A->off_values);
    uint32_t* rp = dev_ptr<uint32_t>(csr->row_pointer, csr->off_row_pointer);
    // row counts into rp[1..rows], scanned in place (inclusive), rp[0] = 0
    uint32_t* part = static_cast<uint32_t*>(control->reduce_scratch.ptr);
    cudaMemsetAsync(rp, 0, 4, s);
    count_rows_kernel<T><<<grid_for(static_cast<uint64_t>(rows) * 32, control->sm_count), kThreads, 0, s>>>(
        D, dv, rows, cols, rp + 1);
    if (rows) {
        scan::inclusive_u32(rp + 1, rows, part, s);
    }
    uint32_t* hv = static_cast<uint32_t*>(control->pinned) + 512;
    cudaMemcpyAsync(hv, rp + rows, 4, cudaMemcpyDeviceToHost, s);
    compact_rows_kernel<T><<<grid_for(static_cast<uint64_t>(rows) * 32, control->sm_count), kThreads, 0, s>>>(
        D, dv, rows, cols, rp, dev_ptr<uint32_t>(csr->col_indices, csr->off_col_indices),
        dev_ptr<T>(csr->values, csr->off_values));
    if (cudaGetLastError() != cudaSuccess || cudaStreamSynchronize(s) != cudaSuccess)
        return clsparseInvalidKernelExecution;
    csr->num_rows = rows;
    csr->num_cols = cols;
    csr->num_nonzeros = *hv;
    return finish_call(control);
}

}  // namespace
}  // namespace clsp

using namespace clsp;

extern "C" {

clsparseStatus clsparseScoomv(const clsparseScalar* alpha, const clsparseCooMatrix* matx, const cldenseVector* x,
                              const clsparseScalar* beta, cldenseVector* y, const clsparseControl control) {
    return coomv<float>(alpha, matx, x, beta, y, control);
}
clsparseStatus clsparseDcoomv(const clsparseScalar* alpha, const clsparseCooMatrix* matx, const cldenseVector* x,
                              const clsparseScalar* beta, cldenseVector* y, const clsparseControl control) {
    return coomv<double>(alpha, matx, x, beta, y, control);
}
clsparseStatus clsparseScoo2csr(const clsparseCooMatrix* coo, clsparseCsrMatrix* csr, const clsparseControl control) {
    return coo2csr<float>(coo, csr, control);
}
clsparseStatus clsparseDcoo2csr(const clsparseCooMatrix* coo, clsparseCsrMatrix* csr, const clsparseControl control) {
    return coo2csr<double>(coo, csr, control);
}
clsparseStatus clsparseScsr2coo(const clsparseCsrMatrix* csr, clsparseCooMatrix* coo, const clsparseControl control) {
    return csr2coo<float>(csr, coo, control);
}
clsparseStatus clsparseDcsr2coo(const clsparseCsrMatrix* csr, clsparseCooMatrix* coo, const clsparseControl control) {
    return csr2coo<double>(csr, coo, control);
}
clsparseStatus clsparseScsr2dense(const clsparseCsrMatrix* csr, cldenseMatrix* A, const clsparseControl control) {
    return csr2dense<float>(csr, A, control);
}
clsparseStatus clsparseDcsr2dense(const clsparseCsrMatrix* csr, cldenseMatrix* A, clsparseControl control) {
    return csr2dense<double>(csr, A, control);
}
clsparseStatus clsparseSdense2csr(const cldenseMatrix* A, clsparseCsrMatrix* csr, const clsparseControl control) {
    return dense2csr<float>(A, csr, control);
}
clsparseStatus clsparseDdense2csr(const cldenseMatrix* A, clsparseCsrMatrix* csr, const clsparseControl control) {
    return dense2csr<double>(A, csr, control);
}

}  // extern "C"
