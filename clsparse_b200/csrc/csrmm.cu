// Sparse x dense product C = alpha * A * B + beta * C (clsparseScsrmm /
// clsparseDcsrmm) for sm_100a.
//
// The reference runs it as a batched SpMV: one csrmv pass per column of C
// (src/library/blas3/clsparse-csrmm.hpp:28-118, kernel
// src/library/kernels/csrmm_general.cl:60-167), re-reading A once per
// column. Here A is read once: a group of G lanes owns a row of A and a tile
// of G consecutive columns of C; the lanes load G nonzeros of the row at a
// time (coalesced), broadcast each (column, value) pair with shuffles, and
// every lane multiplies it by its own element of that row of B, so a row of B
// is read as one contiguous segment per group. G (1..32) follows the number
// of columns. alpha multiplies each product and beta == 0 overwrites C
// without reading it, as in the reference (csrmm_general.cl:96-126).
//
// Layouts: the reference indexes B and C row-major through lead_dim whatever
// their `major` field says; here row-major is the same, and column-major
// matrices are indexed as column-major.
#include "device_common.cuh"
#include "internal.h"

namespace clsp {
namespace {

constexpr int kThreads = 256;

struct DenseView {
    size_t ld;
    bool col_major;
    __device__ __forceinline__ size_t at(size_t r, size_t c) const { return col_major ? c * ld + r : r * ld + c; }
};

template <typename T, int G>
__global__ void __launch_bounds__(kThreads)
    csrmm_kernel(const uint32_t* __restrict__ rp, const uint32_t* __restrict__ cols, const T* __restrict__ vals,
                 uint32_t nrows, uint32_t ncols, const T* __restrict__ alpha_p, const T* __restrict__ beta_p,
                 const T* __restrict__ B, DenseView bv, T* __restrict__ C, DenseView cv) {
    const T alpha = *alpha_p, beta = *beta_p;
    const uint32_t lane = threadIdx.x & (G - 1);
    // Groups of one warp may be at different rows and iterations: shuffles
    // name only this group's lanes.
    const unsigned mask = G == 32 ? 0xffffffffu : (((1u << G) - 1u) << ((threadIdx.x & 31u) & ~(G - 1u)));
    const uint64_t group = (static_cast<uint64_t>(blockIdx.x) * kThreads + threadIdx.x) / G;
    const uint64_t ngroups = static_cast<uint64_t>(gridDim.x) * kThreads / G;
    const uint32_t tiles = (ncols + G - 1) / G;
    const uint64_t work = static_cast<uint64_t>(nrows) * tiles;
    for (uint64_t w = group; w < work; w += ngroups) {
        const uint32_t row = static_cast<uint32_t>(w / tiles);
        const uint32_t c = static_cast<uint32_t>(w % tiles) * G + lane;
        const uint32_t rb = dev::ld_ro(rp + row), re = dev::ld_ro(rp + row + 1);
        T acc = T(0);
        for (uint32_t base = rb; base < re; base += G) {
            uint32_t kc = 0;
            T kv = T(0);
            if (base + lane < re) {
                kc = dev::ld_stream(cols + base + lane);
                kv = alpha * dev::ld_stream(vals + base + lane);
            }
            const uint32_t cnt = min(static_cast<uint32_t>(G), re - base);
            for (uint32_t j = 0; j < cnt; ++j) {
                const uint32_t k = G > 1 ? __shfl_sync(mask, kc, j, G) : kc;
                const T v = G > 1 ? __shfl_sync(mask, kv, j, G) : kv;
                if (c < ncols) acc = dev::fma_rn(v, dev::ld_ro(B + bv.at(k, c)), acc);
            }
        }
        if (c < ncols) {
            T* dst = C + cv.at(row, c);
            *dst = beta == T(0) ? acc : (beta == T(1) ? acc + *dst : acc + beta * *dst);
        }
    }
}

template <typename T>
clsparseStatus csrmm_entry(const clsparseScalar* alpha, const clsparseCsrMatrix* A, const cldenseMatrix* B,
                           const clsparseScalar* beta, cldenseMatrix* C, clsparseControl control) {
    clsparseStatus st = check_entry(control);
    if (st != clsparseSuccess) return st;
    if (!alpha || !A || !B || !beta || !C) return clsparseInvalidValue;
    if (B->num_rows < A->num_cols || C->num_rows < A->num_rows || B->num_cols < C->num_cols) return clsparseInvalidSize;
    const bool bcm = B->major == columnMajor, ccm = C->major == columnMajor;
    if (B->lead_dim < (bcm ? B->num_rows : B->num_cols) || C->lead_dim < (ccm ? C->num_rows : C->num_cols))
        return clsparseInvalidSize;
    if (A->num_rows == 0 || C->num_cols == 0) return clsparseSuccess;
    if (!alpha->value || !beta->value || !B->values || !C->values || !A->row_pointer ||
        (A->num_nonzeros > 0 && (!A->values || !A->col_indices)))
        return clsparseInvalidMemObject;
    DeviceGuard g(control->device);
    const uint32_t nrows = A->num_rows, ncols = C->num_cols;
    int G = 32;
    while (G > 1 && static_cast<uint32_t>(G / 2) >= ncols) G /= 2;
    const uint64_t groups = static_cast<uint64_t>(nrows) * ((ncols + G - 1) / G);
    uint64_t ctas = (groups * G + kThreads - 1) / kThreads;
    const uint64_t cap = static_cast<uint64_t>(control->sm_count) * 16;
    if (ctas > cap) ctas = cap;
    if (ctas == 0) ctas = 1;
    const uint32_t* rp = dev_ptr<const uint32_t>(A->row_pointer, A->off_row_pointer);
    const uint32_t* cl = dev_ptr<const uint32_t>(A->col_indices, A->off_col_indices);
    const T* va = dev_ptr<const T>(A->values, A->off_values);
    const T* a = dev_ptr<const T>(alpha->value, alpha->off_value);
    const T* b = dev_ptr<const T>(beta->value, beta->off_value);
    const T* Bp = dev_ptr<const T>(B->values, B->off_values);
    T* Cp = dev_ptr<T>(C->values, C->off_values);
    const DenseView bv{B->lead_dim, bcm}, cv{C->lead_dim, ccm};
    cudaStream_t s = control->stream;
#define CLSP_MM(GW) \
    csrmm_kernel<T, GW><<<static_cast<uint32_t>(ctas), kThreads, 0, s>>>(rp, cl, va, nrows, ncols, a, b, Bp, bv, Cp, cv)
    switch (G) {
        case 1: CLSP_MM(1); break;
        case 2: CLSP_MM(2); break;
        case 4: CLSP_MM(4); break;
        case 8: CLSP_MM(8); break;
        case 16: CLSP_MM(16); break;
        default: CLSP_MM(32); break;
    }
#undef CLSP_MM
    if (cudaGetLastError() != cudaSuccess) return clsparseInvalidKernelExecution;
    return finish_call(control);
}

}  // namespace
}  // namespace clsp

extern "C" {

clsparseStatus clsparseScsrmm(const clsparseScalar* alpha, const clsparseCsrMatrix* sparseMatA,
                              const cldenseMatrix* denseMatB, const clsparseScalar* beta, cldenseMatrix* denseMatC,
                              const clsparseControl control) {
    clsp::TraceRange trace_("clsparseScsrmm");
    return clsp::csrmm_entry<float>(alpha, sparseMatA, denseMatB, beta, denseMatC, control);
}

clsparseStatus clsparseDcsrmm(const clsparseScalar* alpha, const clsparseCsrMatrix* sparseMatA,
                              const cldenseMatrix* denseMatB, const clsparseScalar* beta, cldenseMatrix* denseMatC,
                              const clsparseControl control) {
    clsp::TraceRange trace_("clsparseDcsrmm");
    return clsp::csrmm_entry<double>(alpha, sparseMatA, denseMatB, beta, denseMatC, control);
}

}  // extern "C"
