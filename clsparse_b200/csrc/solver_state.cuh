// Device-resident state of one CG / BiCGStab solve and the scalar steps the
// reference ran as separate 1-element kernels and host reads
// (src/library/solvers/conjugate-gradients.hpp:110-226,
//  biconjugate-gradients-stabilized.hpp:103-266). Scalars are kept in the
// solve's value type T, as the reference's clsparse::scalar<T> were; the
// reductions feeding them are accumulated in double.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace clsp {

// Device status bits reported through clsparseB200SolverGetDeviceStatus.
enum : int {
    kStatusMissingDiag = 1,
    kStatusZeroDiag = 2,
    kStatusCurvature = 4,
    kStatusBicgBreakdown = 8,
    kStatusNonFinite = 16,
    kStatusBarrierTimeout = 32,  // a persistent solver's grid barrier wait ran out
};

constexpr int kMaxSnapshots = 8;

template <typename T>
struct SolverState {
    // parameters (written by the host before each solve)
    double relTol;
    double absTol;
    int maxIters;
    int norm_type;  // 0: ||.||_1 as the reference, 1: ||.||_2
    int stop_nonfinite;  // 1: a non-finite residual ends the solve (inner solves of the refinement)
    // scalars of the iteration, in T like the reference
    T norm_b, rz, rz_old, yp, alpha, beta, omega, norm_r, res;
    T rsr_old, rsr_new, rs_amp, amss, amsams;
    T one, zero;   // device constants for SpMV calls with alpha = 1, beta = 0
    // bookkeeping
    double init_res;
    double cur_res;
    int iteration;
    int nIters;
    int done;      // 1 once the stop test passed; later kernels return at once
    int zero_b;    // ||b||_1 == 0: x = b and stop (conjugate-gradients.hpp:87-95)
    int exit_s;    // BiCGStab stopped on ||s|| (biconjugate-gradients-stabilized.hpp:183-195)
    int status_bits;
    // optional records (clsparseB200SolverSetHistory / SetSnapshots)
    double* hist;      // residuum of the start and of every iteration, FP64
    int hist_cap;
    int hist_len;      // entries written by this solve
    int snap_count;    // residual vectors r kept after snap_iter[k] iterations (CG)
    int snap_iter[kMaxSnapshots];
    T* snap;           // snap_count vectors of n values
};

// Stores the residuum the stop test sees after `iterations` loop iterations
// (0: the start) into the history, when one is attached and has room.
template <typename T>
__device__ __forceinline__ void record_residual(SolverState<T>* st, int iterations, double res) {
    if (st->hist != nullptr && iterations >= 0 && iterations < st->hist_cap) {
        st->hist[iterations] = res;
        st->hist_len = iterations + 1;
    }
}

// Slot of the residual snapshot taken after `iterations` iterations, or -1.
template <typename T>
__device__ __forceinline__ int snapshot_slot(const SolverState<T>* st, int iterations) {
    for (int k = 0; k < st->snap_count; ++k)
        if (st->snap_iter[k] == iterations) return k;
    return -1;
}

// The reference's stop test (solver-control.hpp:47-64): converged if
// res <= relTol or res <= absTol * initial residual, or out of iterations.
// The reference keeps iterating on a non-finite residual until maxIters; the
// inner solves of the mixed-precision refinement stop at once instead
// (stop_nonfinite), so that a broken preconditioner costs one iteration.
template <typename T>
__device__ __forceinline__ bool solver_finished(const SolverState<T>& s, double res) {
    return (res <= s.relTol) || (res <= s.absTol * s.init_res) || (s.nIters >= s.maxIters) ||
           (s.stop_nonfinite && !isfinite(res));
}

__device__ __forceinline__ void set_condition(unsigned long long h, unsigned int v) {
    if (h != 0ull) cudaGraphSetConditional(static_cast<cudaGraphConditionalHandle>(h), v);
}

template <typename T>
__device__ __forceinline__ bool finite_t(T v) {
    return isfinite(v);
}

// Finaliser after q = A p with dot0 = <q, p>: alpha = <r,z> / <q,p>.
template <typename T>
__device__ __forceinline__ void fin_cg_alpha(SolverState<T>* st, double yp) {
    st->yp = static_cast<T>(yp);
    st->alpha = st->rz / st->yp;
    if (!(st->yp > T(0))) st->status_bits |= kStatusCurvature;
}

// Finaliser after z = G^T (G r) with dot0 = <z, r>: new <r,z>, beta.
template <typename T>
__device__ __forceinline__ void fin_pcg_rz(SolverState<T>* st, double rz) {
    st->rz_old = st->rz;
    st->rz = static_cast<T>(rz);
    st->beta = st->rz / st->rz_old;
}

// Finaliser of the first z = G^T (G r0): <r0, z0>.
template <typename T>
__device__ __forceinline__ void fin_pcg_rz0(SolverState<T>* st, double rz) {
    st->rz = static_cast<T>(rz);
}

// Finaliser after AMp = A (M p) with dot0 = <AMp, r*>: alpha = <r*,r> / <r*,AMp>.
template <typename T>
__device__ __forceinline__ void fin_bicg_alpha(SolverState<T>* st, double rs_amp) {
    st->rs_amp = static_cast<T>(rs_amp);
    st->alpha = st->rsr_old / st->rs_amp;
    if (st->rs_amp == T(0)) st->status_bits |= kStatusBicgBreakdown;
}

// Finaliser after AMs = A (M s) with dot0 = <AMs, s>, dot1 = <AMs, AMs>.
template <typename T>
__device__ __forceinline__ void fin_bicg_omega(SolverState<T>* st, double amss, double amsams) {
    st->amss = static_cast<T>(amss);
    st->amsams = static_cast<T>(amsams);
    st->omega = st->amss / st->amsams;
    if (st->omega == T(0)) st->status_bits |= kStatusBicgBreakdown;
}

}  // namespace clsp
