// Banded (diagonal-storage) solves -- the inner solves of the mixed-precision
// refinement and the drop-in CG / BiCGStab of solver loop mode 3: types shared
// by dia.cu, mixed.cu and solvers.cu. See dia.cu for the storage and the
// engine.
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "fused.h"
#include "internal.h"

namespace clsp {

constexpr int kMaxDiags = 16;  // distinct column offsets a matrix may have to be stored by diagonal

// Column offsets j - i of a matrix's diagonals, increasing.
struct DiaOffsets {
    int nd = 0;
    int32_t off[kMaxDiags] = {};
};

// A matrix stored by diagonal: vals[d * n + i] = A[i][i + off[d]], zero where
// i + off[d] lies outside the matrix.
template <typename V>
struct DiaMat {
    const V* vals = nullptr;
    int nd = 0;
    int32_t off[kMaxDiags] = {};
    // When set, the main diagonal in FP32 (its entries in vals are zero):
    // the row-sum-compensated diagonal of a BF16-valued copy (dia_compensate_diag).
    const float* diag32 = nullptr;
};

// In/out block of one inner solve (device copy written before the launch,
// read back after it).
struct DiaPcgState {
    // in
    double tol = 0.0;    // stop when ||r|| <= tol ||r_0|| (L2, recursive residual)
    int max_iters = 0;
    int warm = 0;        // continue the direction in p[pbuf] with denominator rz_prev
    int pbuf = 0;
    double rz_prev = 0.0;
    // out (pbuf, rz_prev too: the last direction and its denominator)
    int iters = 0;
    double rr0 = 0.0, rr = 0.0;  // squared norms of the first and the last recursive residual
    int xbuf = 0;
    int status = 0;              // kStatusCurvature / kStatusNonFinite / kStatusBarrierTimeout
};

template <typename VA, typename VG>
struct DiaPcgArgs {
    DiaMat<VA> A;
    DiaMat<VG> G, GT;       // learned factor M^-1 = G^T G (learned solves)
    const float* invD;      // Jacobi (or nullptr: no preconditioner) when not learned
    const float* b;         // right-hand side of the inner system
    float* x;               // solution, from 0
    float* r[2];
    float* p[2];
    float* q;
    float* t;               // scratch (unused by the current schedules)
    float* z;
    uint32_t n;
    int gt_diag;            // index of G^T's main diagonal (learned solves)
    uint32_t gt_halo;       // largest column offset of G^T (its offsets are >= 0: G is lower triangular)
    FusedSync sync;
    DiaPcgState* st;
};

// CLSPARSE_B200_DIA=0 keeps every inner solve on CSR.
bool dia_enabled();

// The drop-in clsparse{S,D}csrcg on the banded engine (solver loop mode 3):
// the reference's CG (operation order, scalar type T, L1 or L2 stop test,
// nIters bookkeeping, x as initial guess, x = b for a zero right-hand side)
// as one cooperative launch for a matrix with at most kMaxDiags distinct
// diagonals. clsparseNotImplemented when the matrix does not qualify (not
// banded, or with Jacobi a missing or zero diagonal entry): the caller then
// runs the graph engine, which reports those cases.
template <typename T>
clsparseStatus dia_cg_dropin(cldenseVector* x, const clsparseCsrMatrix* A, const cldenseVector* b,
                             clSParseSolverControl sc, clsparseControl c);

// The drop-in clsparse{S,D}csrbicgStab on the banded engine (solver loop
// mode 3), with the same rules and fallback as dia_cg_dropin.
template <typename T>
clsparseStatus dia_bicg_dropin(cldenseVector* x, const clsparseCsrMatrix* A, const cldenseVector* b,
                               clSParseSolverControl sc, clsparseControl c);

// The distinct column offsets of a CSR matrix when there are at most
// kMaxDiags and they hold at least half of the stored diagonal entries
// (clsparseSuccess), otherwise clsparseInvalidValue (the caller stays on CSR).
clsparseStatus dia_detect(const uint32_t* rp, const uint32_t* cols, uint32_t n, uint32_t nnz, DiaWork& w,
                          cudaStream_t s, DiaOffsets& offs);

// Padded diagonal counts the engine is built for: ca for A (Jacobi / none,
// or the learned pair) and cg for G and G^T; 0 when a count is too large.
void dia_classes(int nda, int ndg, bool learned, int& ca, int& cg);

// Lays a CSR matrix out by diagonal into buf, rounding values to VO, with
// nd_pad >= offs.nd diagonals (the extra ones have offset 0 and zero values).
template <typename VI, typename VO>
clsparseStatus dia_build(const uint32_t* rp, const uint32_t* cols, const VI* vals, uint32_t n,
                         const DiaOffsets& offs, int nd_pad, DeviceBuffer& buf, cudaStream_t s, DiaMat<VO>& out);

// Row-sum-compensated rounding of a DIA copy of A (its values rounded to V):
// diag32[i] = a_ii + sum_{j != i} (a_ij - round_V(a_ij)) in FP32, and A's
// main diagonal in V set to zero with A.diag32 = diag32. The copy keeps A's
// row sums, so the rounding perturbation E has zero row sums and, for an
// M-matrix A, |x^T E x| <= u x^T A x (u the unit roundoff of V): the copy
// stays SPD and spectrally within 1 +- u of A, where plain rounding of every
// entry can make a nearly singular diffusion operator indefinite.
// clsparseInvalidValue if A has no main diagonal.
template <typename V>
clsparseStatus dia_compensate_diag(const uint32_t* rp, const uint32_t* cols, const double* vals, uint32_t n,
                                   DiaMat<V>& A, float* diag32, cudaStream_t s);

// invD = 1 / diag(A) (FP32) from a DIA matrix; status |= kStatusZeroDiag on
// a zero; clsparseInvalidValue without a main diagonal.
template <typename VA>
clsparseStatus dia_jacobi(const DiaMat<VA>& A, uint32_t n, float* invD, int* status, cudaStream_t s);

// One inner solve (one cooperative launch); st in/out as above.
template <typename VA, typename VG>
clsparseStatus dia_pcg_solve(DiaPcgArgs<VA, VG> a, bool learned, DiaWork& w, clsparseControl c,
                             DiaPcgState& st);

}  // namespace clsp
