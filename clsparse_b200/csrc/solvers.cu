// Preconditioned CG and BiCGStab (clsparse{S,D}csrcg, clsparse{S,D}csrbicgStab)
// for sm_100a.
//
// The iteration follows the reference operation for operation
// (src/library/solvers/conjugate-gradients.hpp:65-226 and
//  biconjugate-gradients-stabilized.hpp:61-266): same recurrences, same
// roundings of every vector update, the L1 stop test of solver-control.hpp:47-64
// and the same iteration bookkeeping. What changes is where it runs:
//
// * every scalar (alpha, beta, omega, the residual) lives in device memory and
//   is computed by the last CTA of the kernel that finishes its reduction, so
//   an iteration needs no host round trip (the reference blocks on a host read
//   of the residual every iteration, conjugate-gradients.hpp:223);
// * the BLAS-1 steps of an iteration are fused: CG runs three kernels per
//   iteration (SpMV with <Ap,p> fused; x/r/z update with <r,z> and ||r||_1
//   fused; p update), BiCGStab five;
// * the whole solve -- Jacobi extraction, initial residual, the loop and the
//   exit -- is one CUDA graph whose loop is a conditional WHILE node driven by
//   the device-side stop test, with four iteration bodies per trip. The graph
//   is cached per control and re-launched when the same operands are solved
//   again.
//
// The host reads the solver state once, after the graph, to fill the solver
// control (iteration count, residuals) exactly as the reference leaves it.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <limits>
#include <type_traits>

#include "device_common.cuh"
#include "dia.h"
#include "internal.h"
#include "fused.h"
#include "solver_cache.h"
#include "solver_state.cuh"

namespace clsp {
namespace {

constexpr int kThreads = 256;
constexpr size_t kTicketBytes = 2048;  // reduction counters at the head of the solver's partials buffer

// Jacobi extraction runs a warp per row: enough CTAs that each warp walks
// only a few rows (the walk is a chain of dependent loads).
uint32_t diag_grid(size_t n, int sms) {
    size_t ctas = (n + (kThreads / 32) - 1) / (kThreads / 32);
    const size_t cap = static_cast<size_t>(sms) * 64;
    if (ctas > cap) ctas = cap;
    return static_cast<uint32_t>(ctas ? ctas : 1);
}

uint32_t vec_grid(size_t n, int sms) {
    size_t ctas = (n + kThreads * 4 - 1) / (kThreads * 4);
    size_t cap = static_cast<size_t>(sms) * 8;
    if (cap > static_cast<size_t>(kMaxReduceCtas)) cap = kMaxReduceCtas;
    if (ctas > cap) ctas = cap;
    if (ctas == 0) ctas = 1;
    return static_cast<uint32_t>(ctas);
}

template <typename T>
__device__ __forceinline__ T apply_m(const T* __restrict__ invD, size_t i, T r) {
    return invD ? r * invD[i] : r;
}

template <typename T>
__device__ __forceinline__ double dabs(T v) {
    return fabs(static_cast<double>(v));
}

// Contribution of one residual entry to the stop-test norm: |v| for the
// reference's L1 test, v^2 for the L2 option.
template <typename T>
__device__ __forceinline__ double norm_term(T v, int l2) {
    const double d = static_cast<double>(v);
    return l2 ? d * d : fabs(d);
}

__device__ __forceinline__ double norm_finish(double acc, int l2) {
    return l2 ? sqrt(acc) : acc;
}

// invD[row] = 1 / A[row,row], first matching entry of the row as in the
// reference's extract_diagonal (src/library/kernels/matrix_utils.cl:65-98).
// A row without a diagonal entry gets 0 and raises a status bit; a zero
// diagonal gives inf like the reference and raises another.
template <typename V, typename T>
__global__ void __launch_bounds__(kThreads)
    extract_inv_diag_kernel(const uint32_t* __restrict__ rp, const uint32_t* __restrict__ cols,
                            const V* __restrict__ vals, uint32_t n, T* __restrict__ invD,
                            SolverState<T>* st) {
    const int lane = threadIdx.x & 31;
    const uint64_t warp = (static_cast<uint64_t>(blockIdx.x) * kThreads + threadIdx.x) >> 5;
    const uint64_t nwarps = (static_cast<uint64_t>(gridDim.x) * kThreads) >> 5;
    for (uint64_t row = warp; row < n; row += nwarps) {
        const uint32_t nb = rp[row], ne = rp[row + 1];
        bool found = false;
        for (uint32_t base = nb; base < ne && !found; base += 32) {
            const uint32_t j = base + lane;
            const bool m = (j < ne) && (cols[j] == row);
            const unsigned ball = __ballot_sync(0xffffffffu, m);
            if (ball) {
                const int first = __ffs(ball) - 1;
                if (lane == first) {
                    const T v = dev::to_t<T>(vals[j]);
                    invD[row] = T(1) / v;
                    if (v == T(0)) atomicOr(&st->status_bits, kStatusZeroDiag);
                }
                found = true;
            }
        }
        if (!found && lane == 0) {
            invD[row] = T(0);
            atomicOr(&st->status_bits, kStatusMissingDiag);
        }
    }
}

// ---------------------------------------------------------------- CG ----

template <typename T>
struct CgArgs {
    T* x;
    const T* b;
    T* y;
    T* r;
    T* p;
    const T* invD;  // nullptr: no preconditioner
    SolverState<T>* st;
    double* parts;
    uint32_t* ticket;
    size_t n;
    unsigned long long cond;
    int warm;  // x == 0 and p holds the previous solve's direction
};

// r = b - A x (y holds A x), z = M r, p = z; ||b||_1, ||r||_1, <r,z>; initial
// stop test (conjugate-gradients.hpp:73-148).
// Warm start (x == 0, r = b): p is kept; beta = <r,z> / rz_old with rz_old
// preset from the previous solve, and cg_p_kernel then forms p = z + beta p,
// so the solve continues the previous search direction with the residual
// replaced (reliable updates of the mixed-precision refinement).
template <typename T>
__global__ void __launch_bounds__(kThreads) cg_init_kernel(CgArgs<T> a) {
    double acc[3] = {0.0, 0.0, 0.0};
    const int l2 = a.st->norm_type;
    const int slot = a.st->snap != nullptr ? snapshot_slot(a.st, 0) : -1;
    const size_t stride = static_cast<size_t>(gridDim.x) * kThreads;
    for (size_t i = static_cast<size_t>(blockIdx.x) * kThreads + threadIdx.x; i < a.n; i += stride) {
        const T bi = a.b[i];
        const T ri = a.warm ? bi : bi - a.y[i];
        const T zi = apply_m(a.invD, i, ri);
        a.r[i] = ri;
        if (slot >= 0) a.st->snap[static_cast<size_t>(slot) * a.n + i] = ri;
        if (!a.warm) a.p[i] = zi;
        acc[0] += norm_term(bi, l2);
        acc[1] += norm_term(ri, l2);
        acc[2] += static_cast<double>(ri) * static_cast<double>(zi);
    }
    double tot[3];
    if (dev::grid_reduce_last<3>(acc, a.parts, a.ticket, tot) && threadIdx.x == 0) {
        SolverState<T>* st = a.st;
        st->norm_b = static_cast<T>(norm_finish(tot[0], l2));
        if (st->norm_b == T(0)) {
            st->zero_b = 1;
            st->done = 1;
            st->nIters = 0;
            set_condition(a.cond, 0u);
            return;
        }
        st->norm_r = static_cast<T>(norm_finish(tot[1], l2));
        st->res = st->norm_r / st->norm_b;
        st->init_res = static_cast<double>(st->res);
        st->cur_res = st->init_res;
        st->rz = static_cast<T>(tot[2]);
        if (a.warm) st->beta = st->rz / st->rz_old;
        st->iteration = 0;
        record_residual(st, 0, st->init_res);
        // The stop test sees the iteration count the solver control held
        // before this solve, as the reference's does.
        if (solver_finished(*st, st->init_res)) {
            st->nIters = 0;
            st->done = 1;
            set_condition(a.cond, 0u);
        } else {
            set_condition(a.cond, 1u);
        }
    }
}

// x += alpha p; r -= alpha y; z = M r; <r,z>, ||r||_1; beta, residual, stop test
// (conjugate-gradients.hpp:186-224).
template <typename T>
__global__ void __launch_bounds__(kThreads) cg_update_kernel(CgArgs<T> a) {
    if (a.st->done) return;
    const T alpha = a.st->alpha;
    const int l2 = a.st->norm_type;
    // iterations done after this update (read before the last CTA counts it)
    const int slot = a.st->snap != nullptr ? snapshot_slot(a.st, a.st->iteration + 1) : -1;
    double acc[2] = {0.0, 0.0};
    const size_t stride = static_cast<size_t>(gridDim.x) * kThreads;
    for (size_t i = static_cast<size_t>(blockIdx.x) * kThreads + threadIdx.x; i < a.n; i += stride) {
        const T xi = a.x[i] + alpha * a.p[i];
        const T ri = a.r[i] - alpha * a.y[i];
        const T zi = apply_m(a.invD, i, ri);
        a.x[i] = xi;
        a.r[i] = ri;
        if (slot >= 0) a.st->snap[static_cast<size_t>(slot) * a.n + i] = ri;
        acc[0] += static_cast<double>(ri) * static_cast<double>(zi);
        acc[1] += norm_term(ri, l2);
    }
    double tot[2];
    if (dev::grid_reduce_last<2>(acc, a.parts, a.ticket, tot) && threadIdx.x == 0) {
        SolverState<T>* st = a.st;
        st->rz_old = st->rz;
        st->rz = static_cast<T>(tot[0]);
        st->beta = st->rz / st->rz_old;
        st->norm_r = static_cast<T>(norm_finish(tot[1], l2));
        st->res = st->norm_r / st->norm_b;
        st->nIters = st->iteration;
        st->iteration += 1;
        st->cur_res = static_cast<double>(st->res);
        record_residual(st, st->iteration, st->cur_res);
        if (!isfinite(st->cur_res)) st->status_bits |= kStatusNonFinite;
        const bool fin = solver_finished(*st, st->cur_res);
        st->done = fin ? 1 : 0;
        set_condition(a.cond, fin ? 0u : 1u);
    }
}

// p = z + beta p with z = M r recomputed (conjugate-gradients.hpp:211).
template <typename T>
__global__ void __launch_bounds__(kThreads) cg_p_kernel(CgArgs<T> a) {
    if (a.st->done) return;
    const T beta = a.st->beta;
    const size_t stride = static_cast<size_t>(gridDim.x) * kThreads;
    for (size_t i = static_cast<size_t>(blockIdx.x) * kThreads + threadIdx.x; i < a.n; i += stride)
        a.p[i] = apply_m(a.invD, i, a.r[i]) + beta * a.p[i];
}

// ||b||_1 == 0: x = b (conjugate-gradients.hpp:87-95).
template <typename T>
__global__ void __launch_bounds__(kThreads) copy_if_zero_b_kernel(T* x, const T* b, size_t n,
                                                                  const SolverState<T>* st) {
    if (!st->zero_b) return;
    const size_t stride = static_cast<size_t>(gridDim.x) * kThreads;
    for (size_t i = static_cast<size_t>(blockIdx.x) * kThreads + threadIdx.x; i < n; i += stride)
        x[i] = b[i];
}

// ----------------------------------------------------------- BiCGStab ----

template <typename T>
struct BicgArgs {
    T* x;
    const T* b;
    T* y;    // A x at start
    T* r;
    T* rs;   // r*
    T* p;
    T* s;
    T* Mp;   // == p without preconditioner
    T* Ms;   // == s without preconditioner
    T* AMp;
    T* AMs;
    const T* invD;
    SolverState<T>* st;
    double* parts;
    uint32_t* ticket;
    size_t n;
    unsigned long long cond;
};

// r = b - A x; r* = r; p = r; Mp = M p; ||b||_1, ||r||_1, <r*,r>
// (biconjugate-gradients-stabilized.hpp:61-131).
template <typename T>
__global__ void __launch_bounds__(kThreads) bicg_init_kernel(BicgArgs<T> a) {
    double acc[3] = {0.0, 0.0, 0.0};
    const int l2 = a.st->norm_type;
    const size_t stride = static_cast<size_t>(gridDim.x) * kThreads;
    for (size_t i = static_cast<size_t>(blockIdx.x) * kThreads + threadIdx.x; i < a.n; i += stride) {
        const T bi = a.b[i];
        const T ri = bi - a.y[i];
        a.r[i] = ri;
        a.rs[i] = ri;
        a.p[i] = ri;
        if (a.invD) a.Mp[i] = ri * a.invD[i];
        acc[0] += norm_term(bi, l2);
        acc[1] += norm_term(ri, l2);
        acc[2] += static_cast<double>(ri) * static_cast<double>(ri);
    }
    double tot[3];
    if (dev::grid_reduce_last<3>(acc, a.parts, a.ticket, tot) && threadIdx.x == 0) {
        SolverState<T>* st = a.st;
        st->norm_b = static_cast<T>(norm_finish(tot[0], l2));
        if (st->norm_b <= std::numeric_limits<T>::min()) {
            st->zero_b = 1;
            st->done = 1;
            st->nIters = 0;
            set_condition(a.cond, 0u);
            return;
        }
        st->norm_r = static_cast<T>(norm_finish(tot[1], l2));
        st->res = st->norm_r / st->norm_b;
        st->init_res = static_cast<double>(st->res);
        st->cur_res = st->init_res;
        record_residual(st, 0, st->init_res);
        st->rsr_old = static_cast<T>(tot[2]);
        st->iteration = 0;
        if (solver_finished(*st, st->init_res)) {
            st->nIters = 0;
            st->done = 1;
            set_condition(a.cond, 0u);
        } else {
            set_condition(a.cond, 1u);
        }
    }
}

// s = r - alpha AMp; Ms = M s; ||s||_1 and the first stop test
// (biconjugate-gradients-stabilized.hpp:175-195). On stop, done = 2 asks the
// x kernel to apply x += alpha Mp once and finish.
template <typename T>
__global__ void __launch_bounds__(kThreads) bicg_s_kernel(BicgArgs<T> a) {
    if (a.st->done) return;
    const T alpha = a.st->alpha;
    const int l2 = a.st->norm_type;
    double acc[1] = {0.0};
    const size_t stride = static_cast<size_t>(gridDim.x) * kThreads;
    for (size_t i = static_cast<size_t>(blockIdx.x) * kThreads + threadIdx.x; i < a.n; i += stride) {
        const T si = a.r[i] - alpha * a.AMp[i];
        a.s[i] = si;
        if (a.invD) a.Ms[i] = si * a.invD[i];
        acc[0] += norm_term(si, l2);
    }
    double tot[1];
    if (dev::grid_reduce_last<1>(acc, a.parts, a.ticket, tot) && threadIdx.x == 0) {
        SolverState<T>* st = a.st;
        const T norm_s = static_cast<T>(norm_finish(tot[0], l2));
        st->res = norm_s / st->norm_b;
        st->cur_res = static_cast<double>(st->res);
        if (!isfinite(st->cur_res)) st->status_bits |= kStatusNonFinite;
        if (solver_finished(*st, st->cur_res)) {
            record_residual(st, st->iteration + 1, st->cur_res);  // the s residual it stopped on
            st->nIters = st->iteration;
            st->exit_s = 1;
            st->done = 2;
            set_condition(a.cond, 0u);
        }
    }
}

// x = (x + alpha Mp) + omega Ms; r = s - omega AMs; ||r||_1, <r*,r>; second
// stop test, beta (biconjugate-gradients-stabilized.hpp:213-250).
template <typename T>
__global__ void __launch_bounds__(kThreads) bicg_x_kernel(BicgArgs<T> a) {
    const int done = a.st->done;
    if (done == 1) return;
    const int l2 = a.st->norm_type;
    const T alpha = a.st->alpha;
    const size_t stride = static_cast<size_t>(gridDim.x) * kThreads;
    double acc[2] = {0.0, 0.0};
    if (done == 2) {
        for (size_t i = static_cast<size_t>(blockIdx.x) * kThreads + threadIdx.x; i < a.n; i += stride)
            a.x[i] = a.x[i] + alpha * a.Mp[i];
    } else {
        const T omega = a.st->omega;
        for (size_t i = static_cast<size_t>(blockIdx.x) * kThreads + threadIdx.x; i < a.n; i += stride) {
            const T x1 = a.x[i] + alpha * a.Mp[i];
            a.x[i] = x1 + omega * a.Ms[i];
            const T ri = a.s[i] - omega * a.AMs[i];
            a.r[i] = ri;
            acc[0] += norm_term(ri, l2);
            acc[1] += static_cast<double>(a.rs[i]) * static_cast<double>(ri);
        }
    }
    double tot[2];
    if (dev::grid_reduce_last<2>(acc, a.parts, a.ticket, tot) && threadIdx.x == 0) {
        SolverState<T>* st = a.st;
        if (done == 2) {
            st->done = 1;
            return;
        }
        st->norm_r = static_cast<T>(norm_finish(tot[0], l2));
        st->res = st->norm_r / st->norm_b;
        st->cur_res = static_cast<double>(st->res);
        record_residual(st, st->iteration + 1, st->cur_res);
        if (!isfinite(st->cur_res)) st->status_bits |= kStatusNonFinite;
        if (solver_finished(*st, st->cur_res)) {
            st->nIters = st->iteration;
            st->done = 1;
            set_condition(a.cond, 0u);
            return;
        }
        st->rsr_new = static_cast<T>(tot[1]);
        T beta = st->rsr_new / st->rsr_old;
        beta = beta * st->alpha;
        beta = beta / st->omega;
        st->beta = beta;
        st->rsr_old = st->rsr_new;
        st->iteration += 1;
        st->nIters = st->iteration;
    }
}

// p = (r + beta p) - (beta omega) AMp; Mp = M p
// (biconjugate-gradients-stabilized.hpp:252-262).
template <typename T>
__global__ void __launch_bounds__(kThreads) bicg_p_kernel(BicgArgs<T> a) {
    if (a.st->done) return;
    const T beta = a.st->beta;
    const T bw = beta * a.st->omega;
    const size_t stride = static_cast<size_t>(gridDim.x) * kThreads;
    for (size_t i = static_cast<size_t>(blockIdx.x) * kThreads + threadIdx.x; i < a.n; i += stride) {
        const T p1 = a.r[i] + beta * a.p[i];
        const T pi = p1 - bw * a.AMp[i];
        a.p[i] = pi;
        if (a.invD) a.Mp[i] = pi * a.invD[i];
    }
}

// ------------------------------------------ factorized-inverse PCG ----
// M^-1 = G^T G (G lower triangular on the pattern of tril(A)), applied as two
// SpMVs, so z is held in memory. Per iteration: q = A p with <q,p> fused
// (alpha); x/r update with the stop test; t = G r; z = G^T t with <z,r> fused
// (beta); p = z + beta p.

template <typename T>
struct PcgArgs {
    T* x;
    const T* b;
    T* q;
    T* r;
    T* p;
    T* t;
    T* z;
    SolverState<T>* st;
    double* parts;
    uint32_t* ticket;
    size_t n;
    unsigned long long cond;
    int warm;  // x == 0 and p holds the previous solve's direction
};

// r = b - A x (q holds A x; warm start: x == 0, r = b); ||b||, ||r||; initial
// stop test.
template <typename T>
__global__ void __launch_bounds__(kThreads) pcg_init_kernel(PcgArgs<T> a) {
    double acc[2] = {0.0, 0.0};
    const int l2 = a.st->norm_type;
    const size_t stride = static_cast<size_t>(gridDim.x) * kThreads;
    for (size_t i = static_cast<size_t>(blockIdx.x) * kThreads + threadIdx.x; i < a.n; i += stride) {
        const T bi = a.b[i];
        const T ri = a.warm ? bi : bi - a.q[i];
        a.r[i] = ri;
        acc[0] += norm_term(bi, l2);
        acc[1] += norm_term(ri, l2);
    }
    double tot[2];
    if (dev::grid_reduce_last<2>(acc, a.parts, a.ticket, tot) && threadIdx.x == 0) {
        SolverState<T>* st = a.st;
        st->norm_b = static_cast<T>(norm_finish(tot[0], l2));
        if (st->norm_b == T(0)) {
            st->zero_b = 1;
            st->done = 1;
            st->nIters = 0;
            set_condition(a.cond, 0u);
            return;
        }
        st->norm_r = static_cast<T>(norm_finish(tot[1], l2));
        st->res = st->norm_r / st->norm_b;
        st->init_res = static_cast<double>(st->res);
        st->cur_res = st->init_res;
        st->iteration = 0;
        record_residual(st, 0, st->init_res);
        if (solver_finished(*st, st->init_res)) {
            st->nIters = 0;
            st->done = 1;
            set_condition(a.cond, 0u);
        } else {
            set_condition(a.cond, 1u);
        }
    }
}

template <typename T>
__global__ void __launch_bounds__(kThreads) pcg_copy_kernel(PcgArgs<T> a) {
    if (a.st->done) return;
    const size_t stride = static_cast<size_t>(gridDim.x) * kThreads;
    for (size_t i = static_cast<size_t>(blockIdx.x) * kThreads + threadIdx.x; i < a.n; i += stride)
        a.p[i] = a.z[i];
}

// x += alpha p; r -= alpha q; ||r||; stop test.
template <typename T>
__global__ void __launch_bounds__(kThreads) pcg_update_kernel(PcgArgs<T> a) {
    if (a.st->done) return;
    const T alpha = a.st->alpha;
    const int l2 = a.st->norm_type;
    double acc[1] = {0.0};
    const size_t stride = static_cast<size_t>(gridDim.x) * kThreads;
    for (size_t i = static_cast<size_t>(blockIdx.x) * kThreads + threadIdx.x; i < a.n; i += stride) {
        a.x[i] = a.x[i] + alpha * a.p[i];
        const T ri = a.r[i] - alpha * a.q[i];
        a.r[i] = ri;
        acc[0] += norm_term(ri, l2);
    }
    double tot[1];
    if (dev::grid_reduce_last<1>(acc, a.parts, a.ticket, tot) && threadIdx.x == 0) {
        SolverState<T>* st = a.st;
        st->norm_r = static_cast<T>(norm_finish(tot[0], l2));
        st->res = st->norm_r / st->norm_b;
        st->nIters = st->iteration;
        st->iteration += 1;
        st->cur_res = static_cast<double>(st->res);
        record_residual(st, st->iteration, st->cur_res);
        if (!isfinite(st->cur_res)) st->status_bits |= kStatusNonFinite;
        const bool fin = solver_finished(*st, st->cur_res);
        st->done = fin ? 1 : 0;
        set_condition(a.cond, fin ? 0u : 1u);
    }
}

template <typename T>
__global__ void __launch_bounds__(kThreads) pcg_p_kernel(PcgArgs<T> a) {
    if (a.st->done) return;
    const T beta = a.st->beta;
    const size_t stride = static_cast<size_t>(gridDim.x) * kThreads;
    for (size_t i = static_cast<size_t>(blockIdx.x) * kThreads + threadIdx.x; i < a.n; i += stride)
        a.p[i] = a.z[i] + beta * a.p[i];
}

// ---------------------------------------------------------- driver ----

// Runs prologue / body / epilogue either as one graph with a conditional
// WHILE node around the body (modes 0 and 2) or as host-enqueued chunks of
// bodies that return at once after the device set done (mode 1).
// Loop bodies per trip of the graph's WHILE node. Every body kernel returns
// at once after the device stop test passed, so the extra bodies after the
// last iteration cost a few microseconds, while each trip of the conditional
// node costs about 2.5-3 us. Measured per CG iteration (1, 4, 8 bodies):
// Poisson 512^2 23.2 / 20.7 / 20.3 us, 1024^2 GRF 46.2 / 43.9 / 43.6 us,
// 128^3 diffusion 101.7 / 99.6 / 99.1 us. CLSPARSE_B200_GRAPH_UNROLL
// overrides the default of 4 (1..16).
int graph_unroll() {
    static const int u = [] {
        const char* e = std::getenv("CLSPARSE_B200_GRAPH_UNROLL");
        const int v = e ? std::atoi(e) : 4;
        return v < 1 ? 1 : (v > 16 ? 16 : v);
    }();
    return u;
}

template <typename Pro, typename Body, typename Epi>
clsparseStatus run_solve(clsparseControl c, SolverCache& cache, bool rebuild, const int* d_done,
                         int max_iters, Pro prologue, Body body, Epi epilogue) {
    cudaStream_t s = c->stream;
    if (c->solver_loop_mode != 1) {
        if (rebuild || cache.exec == nullptr) {
            cache.drop_graph();
            cudaStream_t cs = c->capture_stream;
            cudaStream_t bs = nullptr;
            if (cudaStreamCreateWithFlags(&bs, cudaStreamNonBlocking) != cudaSuccess)
                return clsparseOutOfResources;
            bool ok = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal) == cudaSuccess;
            cudaGraph_t g = nullptr;
            cudaStreamCaptureStatus cst;
            const cudaGraphNode_t* deps = nullptr;
            size_t ndeps = 0;
            cudaGraphConditionalHandle h = 0;
            ok = ok && cudaStreamGetCaptureInfo(cs, &cst, nullptr, &g, &deps, &ndeps) == cudaSuccess;
            ok = ok && cudaGraphConditionalHandleCreate(&h, g, 0u, cudaGraphCondAssignDefault) ==
                           cudaSuccess;
            if (ok) prologue(cs, static_cast<unsigned long long>(h));
            ok = ok && cudaStreamGetCaptureInfo(cs, &cst, nullptr, &g, &deps, &ndeps) == cudaSuccess;
            cudaGraphNodeParams cp = {cudaGraphNodeTypeConditional};
            cp.conditional.handle = h;
            cp.conditional.type = cudaGraphCondTypeWhile;
            cp.conditional.size = 1;
            cudaGraphNode_t cn = nullptr;
            ok = ok && cudaGraphAddNode(&cn, g, deps, ndeps, &cp) == cudaSuccess;
            ok = ok && cudaStreamUpdateCaptureDependencies(cs, &cn, 1,
                                                           cudaStreamSetCaptureDependencies) ==
                           cudaSuccess;
            if (ok) {
                ok = cudaStreamBeginCaptureToGraph(bs, cp.conditional.phGraph_out[0], nullptr,
                                                   nullptr, 0, cudaStreamCaptureModeThreadLocal) ==
                     cudaSuccess;
                if (ok) {
                    for (int u = 0; u < graph_unroll(); ++u) body(bs, static_cast<unsigned long long>(h));
                    cudaGraph_t bg = nullptr;
                    ok = cudaStreamEndCapture(bs, &bg) == cudaSuccess;
                }
            }
            if (ok) epilogue(cs);
            cudaGraph_t full = nullptr;
            const bool ended = cudaStreamEndCapture(cs, &full) == cudaSuccess;
            cudaStreamDestroy(bs);
            if (!ok || !ended) {
                if (full) cudaGraphDestroy(full);
                cudaGetLastError();
                return clsparseInvalidKernelExecution;
            }
            cache.graph = full;
            if (cudaGraphInstantiate(&cache.exec, full, 0) != cudaSuccess) {
                cache.drop_graph();
                cudaGetLastError();
                return clsparseInvalidKernelExecution;
            }
        }
        if (cudaGraphLaunch(cache.exec, s) != cudaSuccess) return clsparseInvalidKernelExecution;
        return clsparseSuccess;
    }
    // mode 1: chunks of iterations, checking the device flag between chunks
    prologue(s, 0ull);
    int* h_done = static_cast<int*>(c->pinned) + 1000;
    const int chunk = 16;
    long long ran = 0;
    while (true) {
        for (int k = 0; k < chunk; ++k) body(s, 0ull);
        ran += chunk;
        cudaMemcpyAsync(h_done, d_done, sizeof(int), cudaMemcpyDeviceToHost, s);
        if (cudaStreamSynchronize(s) != cudaSuccess) return clsparseInvalidKernelExecution;
        if (*h_done != 0) break;
        if (max_iters >= 0 && ran > static_cast<long long>(max_iters) + 2 * chunk) break;
    }
    epilogue(s);
    return cudaGetLastError() == cudaSuccess ? clsparseSuccess : clsparseInvalidKernelExecution;
}

template <typename T>
CsrView<T> view_of(const clsparseCsrMatrix* A) {
    return CsrView<T>{dev_ptr<const T>(A->values, A->off_values),
                      dev_ptr<const uint32_t>(A->col_indices, A->off_col_indices),
                      dev_ptr<const uint32_t>(A->row_pointer, A->off_row_pointer), A->num_rows,
                      A->num_cols, A->num_nonzeros, static_cast<const matrix_meta*>(A->meta)};
}

// Shared entry checks of the four solver entry points
// (conjugate-gradients.cpp:18-116, conjugate-gradients.hpp:56-62).
clsparseStatus check_solver_args(const cldenseVector* x, const clsparseCsrMatrix* A,
                                 const cldenseVector* b, clSParseSolverControl sc,
                                 clsparseControl c) {
    clsparseStatus st = check_entry(c);
    if (st != clsparseSuccess) return st;
    if (sc == nullptr) return clsparseInvalidSolverControlObject;
    if (!x || !A || !b) return clsparseInvalidValue;
    if (A->num_cols != b->num_values || A->num_rows != x->num_values) return clsparseInvalidSystemSize;
    if (A->num_rows != A->num_cols) return clsparseInvalidSystemSize;
    if (A->num_rows > 0 && (!A->row_pointer || !x->values || !b->values)) return clsparseInvalidMemObject;
    if (A->num_nonzeros > 0 && (!A->values || !A->col_indices)) return clsparseInvalidMemObject;
    const auto* meta = static_cast<const matrix_meta*>(A->meta);
    if (meta && (meta->rowBlockSize == 0 || meta->num_rows != A->num_rows)) return clsparseStructInvalid;
    return clsparseSuccess;
}

template <typename T>
void init_state(SolverState<T>& h, clSParseSolverControl sc) {
    std::memset(&h, 0, sizeof(h));
    h.relTol = sc->relativeTolerance;
    h.absTol = sc->absoluteTolerance;
    h.maxIters = sc->maxIters;
    h.norm_type = sc->normType & 1;
    h.stop_nonfinite = sc->stopOnNonFinite ? 1 : 0;
    h.nIters = sc->nIters;
    h.one = T(1);
    h.zero = T(0);
    h.hist = sc->history;
    h.hist_cap = sc->history ? static_cast<int>(sc->historyCapacity) : 0;
    h.snap_count = sc->snapshots ? sc->snapshotCount : 0;
    for (int k = 0; k < h.snap_count; ++k) h.snap_iter[k] = sc->snapshotIters[k];
    h.snap = static_cast<T*>(sc->snapshots);
}

// Copies the device state back into the solver control the way the
// reference leaves it after a solve.
template <typename T>
clsparseStatus read_back(clsparseControl c, SolverCache& cache, clSParseSolverControl sc) {
    auto* h = reinterpret_cast<SolverState<T>*>(static_cast<char*>(c->pinned) + 2048);
    cudaMemcpyAsync(h, cache.state.ptr, sizeof(SolverState<T>), cudaMemcpyDeviceToHost, c->stream);
    if (cudaStreamSynchronize(c->stream) != cudaSuccess) return clsparseInvalidKernelExecution;
    if (c->event) cudaEventRecord(c->event, c->stream);
    sc->deviceStatus = static_cast<cl_uint>(h->status_bits);
    sc->historyLength = static_cast<cl_uint>(h->hist_len);
    if (h->status_bits & kStatusBarrierTimeout) return clsparseInvalidKernelExecution;
    if (h->zero_b) {
        // conjugate-gradients.hpp:87-95 resets the tolerances of the control
        sc->nIters = 0;
        sc->absoluteTolerance = 0.0;
        sc->relativeTolerance = 0.0;
        return clsparseSuccess;
    }
    sc->initialResidual = h->init_res;
    sc->currentResidual = h->cur_res;
    sc->nIters = h->nIters;
    return clsparseSuccess;
}

SolverKey make_key(int kind, int vsize, int dsize, clSParseSolverControl sc, clsparseControl c,
                   const clsparseCsrMatrix* A, const cldenseVector* x, const cldenseVector* b) {
    SolverKey k;
    std::memset(&k, 0, sizeof(k));
    k.kind = kind;
    k.dtype = dsize * 16 + vsize + 256 * (sc->normType & 1);
    k.precond = sc->preconditioner == DIAGONAL ? 1 : 0;
    k.ext = c->extended_precision ? 1 : 0;
    k.loop_mode = c->solver_loop_mode;
    k.ptrs[0] = static_cast<const char*>(A->values) + static_cast<size_t>(A->off_values) * vsize;
    k.ptrs[1] = static_cast<const uint32_t*>(A->col_indices) + A->off_col_indices;
    k.ptrs[2] = static_cast<const uint32_t*>(A->row_pointer) + A->off_row_pointer;
    k.ptrs[3] = static_cast<const char*>(x->values) + static_cast<size_t>(x->off_values) * dsize;
    k.ptrs[4] = static_cast<const char*>(b->values) + static_cast<size_t>(b->off_values) * dsize;
    k.ptrs[5] = A->meta;
    k.n = A->num_rows;
    k.nnz = A->num_nonzeros;
    k.meta_words = A->meta ? static_cast<const matrix_meta*>(A->meta)->num_words : 0;
    k.stream = c->stream;
    return k;
}

// Sizes the cache for `nvec` work vectors of n elements and the reduction
// partials of both the SpMV and the vector kernels.
template <typename T>
clsparseStatus prepare_cache(clsparseControl c, SolverCache& cache, const SolverKey& key, int nvec,
                             size_t n, uint32_t spmv_ctas, bool& rebuild) {
    rebuild = !(cache.valid && cache.key == key);
    const size_t vec_bytes = ((n * sizeof(T) + 255) / 256) * 256;
    // [tickets: kTicketBytes][partials]: the SpMV epilogue's two-level
    // reduction needs 2 x (CTAs + 256) partials and 257 counters
    const size_t parts_doubles = std::max<size_t>(3 * kMaxReduceCtas, 2 * (static_cast<size_t>(spmv_ctas) + 256));
    if (cache.vecs.ensure(vec_bytes * nvec + 256) != cudaSuccess ||
        cache.parts.ensure(parts_doubles * sizeof(double) + kTicketBytes + 256) != cudaSuccess ||
        cache.state.ensure(sizeof(SolverState<T>) + 256) != cudaSuccess) {
        cudaGetLastError();
        cache.valid = false;
        return clsparseOutOfResources;
    }
    if (rebuild) {
        // tickets start at zero; kernels leave them at zero
        cudaMemsetAsync(cache.parts.ptr, 0, cache.parts.bytes, c->stream);
        cache.drop_graph();
    }
    cache.key = key;
    cache.valid = true;
    return clsparseSuccess;
}

// Whether the persistent kernel can run this solve: loop mode 2 and a
// CSR-Adaptive meta (with its host word offsets) on every matrix it reads.
bool fused_ok(clsparseControl c, const matrix_meta* m) {
    return c->solver_loop_mode == 2 && m != nullptr && m->num_words >= 2 &&
           m->h_word_nnz.size() == m->num_words && meta_is_default_shape(m);
}

size_t align256(size_t b) { return (b + 255) / 256 * 256; }

// After a persistent solve ended on a barrier timeout, CTAs that had passed
// a barrier may have counted long-row chunks whose other owners had already
// left: the meta's arrival tickets are zeroed so that later SpMVs start clean.
void reset_long_row_tickets(const matrix_meta* m, cudaStream_t s) {
    if (m && m->d_lr_ticket) cudaMemsetAsync(m->d_lr_ticket, 0, m->num_words * sizeof(uint32_t), s);
}

// Launches the persistent solver: sizes the barrier area, makes the per-CTA
// word ranges of A (and G, Gt) when the operands or the grid changed, zeroes
// the barrier counters and launches one cooperative kernel.
template <typename V, typename T, typename VG>
clsparseStatus run_fused(clsparseControl c, SolverCache& cache, bool rebuild, FusedCgArgs<V, T, VG>& fa,
                         const CsrView<V>& Av, const CsrView<VG>* G, const CsrView<VG>* Gt, int pk) {
    const bool ext = c->extended_precision && pk == 0;
    // all CTAs resident, and no more CTAs than A has row-block words
    const uint32_t words = static_cast<uint32_t>(Av.meta->num_words - 1);
    const uint32_t grid = std::min(fused_grid<V, T, VG>(c->sm_count, ext, pk), std::max(1u, words));
    const size_t sync_b = align256(fused_sync_bytes(grid));
    const size_t wb = align256((static_cast<size_t>(grid) + 1) * sizeof(uint32_t));
    if (cache.fused.ensure(sync_b + 3 * wb) != cudaSuccess) {
        cudaGetLastError();
        return clsparseOutOfResources;
    }
    char* base = static_cast<char*>(cache.fused.ptr);
    uint32_t* wA = reinterpret_cast<uint32_t*>(base + sync_b);
    uint32_t* wG = reinterpret_cast<uint32_t*>(base + sync_b + wb);
    uint32_t* wGt = reinterpret_cast<uint32_t*>(base + sync_b + 2 * wb);
    if (rebuild || cache.fused_grid != grid) {
        std::vector<uint32_t> part;
        const CsrView<VG>* mats[2] = {G, Gt};
        uint32_t* dst[2] = {wG, wGt};
        word_partition(Av.meta, grid, part);
        cudaError_t e = cudaMemcpy(wA, part.data(), part.size() * sizeof(uint32_t), cudaMemcpyHostToDevice);
        for (int k = 0; k < 2 && e == cudaSuccess; ++k) {
            if (!mats[k]) continue;
            word_partition(mats[k]->meta, grid, part);
            e = cudaMemcpy(dst[k], part.data(), part.size() * sizeof(uint32_t), cudaMemcpyHostToDevice);
        }
        if (e != cudaSuccess) {
            cache.fused_grid = 0;
            return clsparseInvalidKernelExecution;
        }
        cache.fused_grid = grid;
    }
    if (cudaMemsetAsync(base, 0, kFusedSyncHead, c->stream) != cudaSuccess) return clsparseInvalidKernelExecution;
    fa.sync = fused_sync_at(base);
    // Failure-path test switches: a shorter wait limit, and a first barrier
    // that is never released (every wait then runs out).
    if (const char* e = std::getenv("CLSPARSE_B200_BARRIER_WAIT_NS")) {
        const unsigned long long v = std::strtoull(e, nullptr, 10);
        if (v > 0) fa.sync.wait_ns = v;
    }
    if (const char* e = std::getenv("CLSPARSE_B200_TEST_BARRIER_NEVER_RELEASE")) fa.sync.never_release = std::atoi(e) != 0;
    fa.A = word_mat(Av, wA);
    if (G) fa.G = word_mat(*G, wG);
    if (Gt) fa.Gt = word_mat(*Gt, wGt);
    if (launch_pcg_fused<V, T, VG>(fa, grid, ext, pk, c->stream) != cudaSuccess) {
        cudaGetLastError();
        return clsparseInvalidKernelExecution;
    }
    return clsparseSuccess;
}

// Whether a warm start may continue the cached solve: the cached work
// vectors belong to the same operands.
bool can_continue(const SolverCache& cache, SolverKey key) {
    if (!cache.valid) return false;
    key.warm = cache.key.warm;
    return cache.key == key;
}

template <typename V, typename T>
clsparseStatus cg_solve(cldenseVector* xv, const clsparseCsrMatrix* A, const cldenseVector* bv,
                        clSParseSolverControl sc, clsparseControl c, WarmStart* ws = nullptr) {
    clsparseStatus stt = check_solver_args(xv, A, bv, sc, c);
    if (stt != clsparseSuccess) return stt;
    DeviceGuard guard(c->device);
    const size_t n = A->num_rows;
    // Loop mode 3: a banded matrix runs the reference's CG as one cooperative
    // launch over a diagonal-storage copy (dia.cu); other matrices, and the
    // options that engine does not carry (history, snapshots, extended
    // precision, the refinement's continued solves), stay on the engines below.
    if (c->solver_loop_mode == 3 && std::is_same_v<V, T> && ws == nullptr && n > 0 && !c->extended_precision &&
        sc->history == nullptr && sc->snapshotCount == 0 && dia_enabled()) {
        stt = dia_cg_dropin<T>(xv, A, bv, sc, c);
        if (stt != clsparseNotImplemented) {
            sc->printSummary(stt);
            return stt;
        }
    }
    if (!c->solver_cache) c->solver_cache = std::make_unique<SolverCache>();
    SolverCache& cache = *c->solver_cache;
    const CsrView<V> Av = view_of<V>(A);
    const uint32_t spmv_ctas = spmv_num_ctas(Av.meta, Av.nrows, Av.nnz);
    SolverKey key = make_key(1, sizeof(V), sizeof(T), sc, c, A, xv, bv);
    const bool warm = ws && ws->warm;
    key.warm = warm ? 1 : 0;
    if (warm && !can_continue(cache, key)) return clsparseInvalidValue;
    bool rebuild = false;
    stt = prepare_cache<T>(c, cache, key, 4, n, spmv_ctas, rebuild);
    if (stt != clsparseSuccess) return stt;

    const size_t vb = ((n * sizeof(T) + 255) / 256) * 256;
    char* base = static_cast<char*>(cache.vecs.ptr);
    CgArgs<T> a;
    a.x = dev_ptr<T>(xv->values, xv->off_values);
    a.b = dev_ptr<const T>(bv->values, bv->off_values);
    a.y = reinterpret_cast<T*>(base);
    a.r = reinterpret_cast<T*>(base + vb);
    a.p = reinterpret_cast<T*>(base + 2 * vb);
    T* invD = reinterpret_cast<T*>(base + 3 * vb);
    a.invD = key.precond ? invD : nullptr;
    a.st = static_cast<SolverState<T>*>(cache.state.ptr);
    a.parts = reinterpret_cast<double*>(static_cast<char*>(cache.parts.ptr) + kTicketBytes);
    a.ticket = static_cast<uint32_t*>(cache.parts.ptr);
    a.n = n;
    a.cond = 0;
    a.warm = warm ? 1 : 0;

    auto* hs = reinterpret_cast<SolverState<T>*>(c->pinned);
    init_state(*hs, sc);
    if (warm) hs->rz_old = static_cast<T>(ws->rz);
    cudaMemcpyAsync(a.st, hs, sizeof(SolverState<T>), cudaMemcpyHostToDevice, c->stream);

    const uint32_t vg = vec_grid(n, c->sm_count);
    const bool ext = c->extended_precision;
    SolverState<T>* st = a.st;

    auto prologue = [&](cudaStream_t s, unsigned long long h) {
        CgArgs<T> aa = a;
        aa.cond = h;
        if (aa.invD && !aa.warm)
            extract_inv_diag_kernel<V, T><<<diag_grid(n, c->sm_count), kThreads, 0, s>>>(Av.rp, Av.cols, Av.vals, Av.nrows,
                                                                  invD, st);
        if (!aa.warm) {
            SpmvEpilogue none;
            launch_csrmv<V, T>(Av, &st->one, &st->zero, aa.x, aa.y, ext, none, s);
        }
        cg_init_kernel<T><<<vg, kThreads, 0, s>>>(aa);
        if (aa.warm) cg_p_kernel<T><<<vg, kThreads, 0, s>>>(aa);
    };
    auto body = [&](cudaStream_t s, unsigned long long h) {
        CgArgs<T> aa = a;
        aa.cond = h;
        SpmvEpilogue epi;
        epi.ndots = 1;
        epi.w0 = aa.p;
        epi.partials = aa.parts;
        epi.ticket = aa.ticket;
        epi.op = EpiOp::CgAlpha;
        epi.state = st;
        epi.done = &st->done;
        launch_csrmv<V, T>(Av, &st->one, &st->zero, aa.p, aa.y, ext, epi, s);
        cg_update_kernel<T><<<vg, kThreads, 0, s>>>(aa);
        cg_p_kernel<T><<<vg, kThreads, 0, s>>>(aa);
    };
    auto epilogue = [&](cudaStream_t s) {
        copy_if_zero_b_kernel<T><<<vg, kThreads, 0, s>>>(a.x, a.b, n, st);
    };
    if (n == 0) {
        sc->nIters = 0;
        return clsparseSuccess;
    }
    // residual snapshots are taken by the graph engine's update kernel
    if (fused_ok(c, Av.meta) && !warm && sc->snapshotCount == 0) {
        FusedCgArgs<V, T, T> fa{};
        fa.x = a.x;
        fa.b = a.b;
        fa.q = a.y;
        fa.r = a.r;
        fa.p = a.p;
        fa.invD = a.invD ? invD : nullptr;
        fa.st = st;
        fa.n = static_cast<uint32_t>(n);
        stt = run_fused<V, T, T>(c, cache, rebuild, fa, Av, nullptr, nullptr, 0);
    } else {
        stt = run_solve(c, cache, rebuild, &st->done, sc->maxIters, prologue, body, epilogue);
    }
    if (stt != clsparseSuccess) {
        cache.valid = false;
        cache.drop_graph();
        return stt;
    }
    stt = read_back<T>(c, cache, sc);
    if (sc->deviceStatus & kStatusBarrierTimeout) {
        reset_long_row_tickets(Av.meta, c->stream);
        cache.valid = false;
    }
    if (ws && stt == clsparseSuccess)
        ws->rz = static_cast<double>(reinterpret_cast<SolverState<T>*>(static_cast<char*>(c->pinned) + 2048)->rz_old);
    sc->printSummary(stt);
    return stt;
}

template <typename V, typename T>
clsparseStatus bicg_solve(cldenseVector* xv, const clsparseCsrMatrix* A, const cldenseVector* bv,
                          clSParseSolverControl sc, clsparseControl c) {
    clsparseStatus stt = check_solver_args(xv, A, bv, sc, c);
    if (stt != clsparseSuccess) return stt;
    DeviceGuard guard(c->device);
    const size_t n = A->num_rows;
    // loop mode 3 on a banded matrix: one cooperative launch (see cg_solve)
    if (c->solver_loop_mode == 3 && std::is_same_v<V, T> && n > 0 && !c->extended_precision &&
        sc->history == nullptr && dia_enabled()) {
        stt = dia_bicg_dropin<T>(xv, A, bv, sc, c);
        if (stt != clsparseNotImplemented) {
            sc->printSummary(stt);
            return stt;
        }
    }
    if (!c->solver_cache) c->solver_cache = std::make_unique<SolverCache>();
    SolverCache& cache = *c->solver_cache;
    const CsrView<V> Av = view_of<V>(A);
    const uint32_t spmv_ctas = spmv_num_ctas(Av.meta, Av.nrows, Av.nnz);
    const SolverKey key = make_key(2, sizeof(V), sizeof(T), sc, c, A, xv, bv);
    bool rebuild = false;
    stt = prepare_cache<T>(c, cache, key, 11, n, spmv_ctas, rebuild);
    if (stt != clsparseSuccess) return stt;

    const size_t vb = ((n * sizeof(T) + 255) / 256) * 256;
    char* base = static_cast<char*>(cache.vecs.ptr);
    auto vec = [&](int k) { return reinterpret_cast<T*>(base + static_cast<size_t>(k) * vb); };
    BicgArgs<T> a;
    a.x = dev_ptr<T>(xv->values, xv->off_values);
    a.b = dev_ptr<const T>(bv->values, bv->off_values);
    a.y = vec(0);
    a.r = vec(1);
    a.rs = vec(2);
    a.p = vec(3);
    a.s = vec(4);
    a.AMp = vec(5);
    a.AMs = vec(6);
    T* invD = vec(7);
    const bool pre = key.precond != 0;
    a.Mp = pre ? vec(8) : a.p;
    a.Ms = pre ? vec(9) : a.s;
    a.invD = pre ? invD : nullptr;
    a.st = static_cast<SolverState<T>*>(cache.state.ptr);
    a.parts = reinterpret_cast<double*>(static_cast<char*>(cache.parts.ptr) + kTicketBytes);
    a.ticket = static_cast<uint32_t*>(cache.parts.ptr);
    a.n = n;
    a.cond = 0;

    auto* hs = reinterpret_cast<SolverState<T>*>(c->pinned);
    init_state(*hs, sc);
    cudaMemcpyAsync(a.st, hs, sizeof(SolverState<T>), cudaMemcpyHostToDevice, c->stream);

    const uint32_t vg = vec_grid(n, c->sm_count);
    const bool ext = c->extended_precision;
    SolverState<T>* st = a.st;

    auto prologue = [&](cudaStream_t s, unsigned long long h) {
        BicgArgs<T> aa = a;
        aa.cond = h;
        if (aa.invD)
            extract_inv_diag_kernel<V, T><<<diag_grid(n, c->sm_count), kThreads, 0, s>>>(Av.rp, Av.cols, Av.vals, Av.nrows,
                                                                  invD, st);
        SpmvEpilogue none;
        launch_csrmv<V, T>(Av, &st->one, &st->zero, aa.x, aa.y, ext, none, s);
        bicg_init_kernel<T><<<vg, kThreads, 0, s>>>(aa);
    };
    auto body = [&](cudaStream_t s, unsigned long long h) {
        BicgArgs<T> aa = a;
        aa.cond = h;
        SpmvEpilogue e1;
        e1.ndots = 1;
        e1.w0 = aa.rs;
        e1.partials = aa.parts;
        e1.ticket = aa.ticket;
        e1.op = EpiOp::BicgAlpha;
        e1.state = st;
        e1.done = &st->done;
        launch_csrmv<V, T>(Av, &st->one, &st->zero, aa.Mp, aa.AMp, ext, e1, s);
        bicg_s_kernel<T><<<vg, kThreads, 0, s>>>(aa);
        SpmvEpilogue e2;
        e2.ndots = 2;
        e2.w0 = aa.s;
        e2.dot1_self = true;
        e2.partials = aa.parts;
        e2.ticket = aa.ticket;
        e2.op = EpiOp::BicgOmega;
        e2.state = st;
        e2.done = &st->done;
        launch_csrmv<V, T>(Av, &st->one, &st->zero, aa.Ms, aa.AMs, ext, e2, s);
        bicg_x_kernel<T><<<vg, kThreads, 0, s>>>(aa);
        bicg_p_kernel<T><<<vg, kThreads, 0, s>>>(aa);
    };
    auto epilogue = [&](cudaStream_t s) {
        copy_if_zero_b_kernel<T><<<vg, kThreads, 0, s>>>(a.x, a.b, n, st);
    };
    if (n == 0) {
        sc->nIters = 0;
        return clsparseSuccess;
    }
    stt = run_solve(c, cache, rebuild, &st->done, sc->maxIters, prologue, body, epilogue);
    if (stt != clsparseSuccess) {
        cache.valid = false;
        cache.drop_graph();
        return stt;
    }
    stt = read_back<T>(c, cache, sc);
    sc->printSummary(stt);
    return stt;
}

// PCG with M^-1 = G^T G; G and Gt (its transpose) are CSR with values VG.
template <typename V, typename T, typename VG>
clsparseStatus pcg_factor_solve(cldenseVector* xv, const clsparseCsrMatrix* A, const cldenseVector* bv,
                                clSParseSolverControl sc, const CsrView<VG>& G, const CsrView<VG>& Gt,
                                clsparseControl c, WarmStart* ws = nullptr) {
    clsparseStatus stt = check_solver_args(xv, A, bv, sc, c);
    if (stt != clsparseSuccess) return stt;
    if (G.nrows != A->num_rows || Gt.nrows != A->num_rows) return clsparseInvalidSystemSize;
    DeviceGuard guard(c->device);
    const size_t n = A->num_rows;
    if (!c->solver_cache) c->solver_cache = std::make_unique<SolverCache>();
    SolverCache& cache = *c->solver_cache;
    const CsrView<V> Av = view_of<V>(A);
    const uint32_t spmv_ctas = std::max(spmv_num_ctas(Av.meta, Av.nrows, Av.nnz),
                                        std::max(spmv_num_ctas(G.meta, G.nrows, G.nnz),
                                                 spmv_num_ctas(Gt.meta, Gt.nrows, Gt.nnz)));
    SolverKey key = make_key(3, sizeof(V), sizeof(T), sc, c, A, xv, bv);
    key.ptrs[6] = G.vals;
    key.ptrs[7] = Gt.vals;
    const bool warm = ws && ws->warm;
    key.warm = warm ? 1 : 0;
    if (warm && !can_continue(cache, key)) return clsparseInvalidValue;
    bool rebuild = false;
    stt = prepare_cache<T>(c, cache, key, 5, n, spmv_ctas, rebuild);
    if (stt != clsparseSuccess) return stt;

    const size_t vb = ((n * sizeof(T) + 255) / 256) * 256;
    char* base = static_cast<char*>(cache.vecs.ptr);
    PcgArgs<T> a;
    a.x = dev_ptr<T>(xv->values, xv->off_values);
    a.b = dev_ptr<const T>(bv->values, bv->off_values);
    a.q = reinterpret_cast<T*>(base);
    a.r = reinterpret_cast<T*>(base + vb);
    a.p = reinterpret_cast<T*>(base + 2 * vb);
    a.t = reinterpret_cast<T*>(base + 3 * vb);
    a.z = reinterpret_cast<T*>(base + 4 * vb);
    a.st = static_cast<SolverState<T>*>(cache.state.ptr);
    a.parts = reinterpret_cast<double*>(static_cast<char*>(cache.parts.ptr) + kTicketBytes);
    a.ticket = static_cast<uint32_t*>(cache.parts.ptr);
    a.n = n;
    a.cond = 0;
    a.warm = warm ? 1 : 0;

    auto* hs = reinterpret_cast<SolverState<T>*>(c->pinned);
    init_state(*hs, sc);
    if (warm) hs->rz = static_cast<T>(ws->rz);
    cudaMemcpyAsync(a.st, hs, sizeof(SolverState<T>), cudaMemcpyHostToDevice, c->stream);

    const uint32_t vg = vec_grid(n, c->sm_count);
    const bool ext = c->extended_precision;
    SolverState<T>* st = a.st;
    auto apply_m = [&](cudaStream_t s, const PcgArgs<T>& aa, EpiOp op) {
        SpmvEpilogue plain;
        plain.done = &st->done;
        launch_csrmv<VG, T>(G, &st->one, &st->zero, aa.r, aa.t, false, plain, s);
        SpmvEpilogue e;
        e.ndots = 1;
        e.w0 = aa.r;
        e.partials = aa.parts;
        e.ticket = aa.ticket;
        e.op = op;
        e.state = st;
        e.done = &st->done;
        launch_csrmv<VG, T>(Gt, &st->one, &st->zero, aa.t, aa.z, false, e, s);
    };
    auto prologue = [&](cudaStream_t s, unsigned long long h) {
        PcgArgs<T> aa = a;
        aa.cond = h;
        if (aa.warm) {
            // r = b; z = G^T G r; beta = <z,r> / rz (preset); p = z + beta p
            pcg_init_kernel<T><<<vg, kThreads, 0, s>>>(aa);
            apply_m(s, aa, EpiOp::PcgRz);
            pcg_p_kernel<T><<<vg, kThreads, 0, s>>>(aa);
            return;
        }
        SpmvEpilogue none;
        launch_csrmv<V, T>(Av, &st->one, &st->zero, aa.x, aa.q, ext, none, s);
        pcg_init_kernel<T><<<vg, kThreads, 0, s>>>(aa);
        apply_m(s, aa, EpiOp::PcgRz0);
        pcg_copy_kernel<T><<<vg, kThreads, 0, s>>>(aa);
    };
    auto body = [&](cudaStream_t s, unsigned long long h) {
        PcgArgs<T> aa = a;
        aa.cond = h;
        SpmvEpilogue epi;
        epi.ndots = 1;
        epi.w0 = aa.p;
        epi.partials = aa.parts;
        epi.ticket = aa.ticket;
        epi.op = EpiOp::CgAlpha;
        epi.state = st;
        epi.done = &st->done;
        launch_csrmv<V, T>(Av, &st->one, &st->zero, aa.p, aa.q, ext, epi, s);
        pcg_update_kernel<T><<<vg, kThreads, 0, s>>>(aa);
        apply_m(s, aa, EpiOp::PcgRz);
        pcg_p_kernel<T><<<vg, kThreads, 0, s>>>(aa);
    };
    auto epilogue = [&](cudaStream_t s) {
        copy_if_zero_b_kernel<T><<<vg, kThreads, 0, s>>>(a.x, a.b, n, st);
    };
    if (n == 0) {
        sc->nIters = 0;
        return clsparseSuccess;
    }
    if (fused_ok(c, Av.meta) && fused_ok(c, G.meta) && fused_ok(c, Gt.meta) && !warm) {
        FusedCgArgs<V, T, VG> fa{};
        fa.x = a.x;
        fa.b = a.b;
        fa.q = a.q;
        fa.r = a.r;
        fa.p = a.p;
        fa.t = a.t;
        fa.z = a.z;
        fa.st = st;
        fa.n = static_cast<uint32_t>(n);
        stt = run_fused<V, T, VG>(c, cache, rebuild, fa, Av, &G, &Gt, 1);
    } else {
        stt = run_solve(c, cache, rebuild, &st->done, sc->maxIters, prologue, body, epilogue);
    }
    if (stt != clsparseSuccess) {
        cache.valid = false;
        cache.drop_graph();
        return stt;
    }
    stt = read_back<T>(c, cache, sc);
    if (sc->deviceStatus & kStatusBarrierTimeout) {
        reset_long_row_tickets(Av.meta, c->stream);
        reset_long_row_tickets(G.meta, c->stream);
        reset_long_row_tickets(Gt.meta, c->stream);
        cache.valid = false;
    }
    if (ws && stt == clsparseSuccess)
        ws->rz = static_cast<double>(reinterpret_cast<SolverState<T>*>(static_cast<char*>(c->pinned) + 2048)->rz);
    return stt;
}

}  // namespace

template <typename V, typename T, typename VG>
clsparseStatus pcg_factor_typed(cldenseVector* x, const clsparseCsrMatrix* A, const cldenseVector* b,
                                clSParseSolverControl sc, const CsrView<VG>& G, const CsrView<VG>& Gt,
                                clsparseControl c, WarmStart* ws) {
    return pcg_factor_solve<V, T, VG>(x, A, b, sc, G, Gt, c, ws);
}
template clsparseStatus pcg_factor_typed<float, float, __nv_bfloat16>(
    cldenseVector*, const clsparseCsrMatrix*, const cldenseVector*, clSParseSolverControl,
    const CsrView<__nv_bfloat16>&, const CsrView<__nv_bfloat16>&, clsparseControl, WarmStart*);
template clsparseStatus pcg_factor_typed<__nv_bfloat16, float, __nv_bfloat16>(
    cldenseVector*, const clsparseCsrMatrix*, const cldenseVector*, clSParseSolverControl,
    const CsrView<__nv_bfloat16>&, const CsrView<__nv_bfloat16>&, clsparseControl, WarmStart*);
template clsparseStatus pcg_factor_typed<float, float, float>(cldenseVector*, const clsparseCsrMatrix*,
                                                              const cldenseVector*, clSParseSolverControl,
                                                              const CsrView<float>&, const CsrView<float>&,
                                                              clsparseControl, WarmStart*);
template clsparseStatus pcg_factor_typed<double, double, double>(
    cldenseVector*, const clsparseCsrMatrix*, const cldenseVector*, clSParseSolverControl,
    const CsrView<double>&, const CsrView<double>&, clsparseControl, WarmStart*);

template <typename V, typename T>
clsparseStatus bicg_solve_typed(cldenseVector* x, const clsparseCsrMatrix* A, const cldenseVector* b,
                                clSParseSolverControl sc, clsparseControl c) {
    return bicg_solve<V, T>(x, A, b, sc, c);
}
template clsparseStatus bicg_solve_typed<float, float>(cldenseVector*, const clsparseCsrMatrix*,
                                                       const cldenseVector*, clSParseSolverControl,
                                                       clsparseControl);
template clsparseStatus bicg_solve_typed<__nv_bfloat16, float>(cldenseVector*, const clsparseCsrMatrix*,
                                                               const cldenseVector*, clSParseSolverControl,
                                                               clsparseControl);

template <typename V, typename T>
clsparseStatus cg_solve_typed(cldenseVector* x, const clsparseCsrMatrix* A, const cldenseVector* b,
                              clSParseSolverControl sc, clsparseControl c, WarmStart* ws) {
    return cg_solve<V, T>(x, A, b, sc, c, ws);
}
template clsparseStatus cg_solve_typed<double, double>(cldenseVector*, const clsparseCsrMatrix*,
                                                       const cldenseVector*, clSParseSolverControl,
                                                       clsparseControl, WarmStart*);
template clsparseStatus cg_solve_typed<float, float>(cldenseVector*, const clsparseCsrMatrix*,
                                                     const cldenseVector*, clSParseSolverControl,
                                                     clsparseControl, WarmStart*);
template clsparseStatus cg_solve_typed<__nv_bfloat16, float>(cldenseVector*, const clsparseCsrMatrix*,
                                                             const cldenseVector*, clSParseSolverControl,
                                                             clsparseControl, WarmStart*);

}  // namespace clsp

using namespace clsp;

extern "C" {

clsparseStatus clsparseScsrcg(cldenseVector* x, const clsparseCsrMatrix* A, const cldenseVector* b,
                              clSParseSolverControl solverControl, clsparseControl control) {
    clsp::TraceRange trace_("clsparseScsrcg");
    return cg_solve<float, float>(x, A, b, solverControl, control);
}

clsparseStatus clsparseDcsrcg(cldenseVector* x, const clsparseCsrMatrix* A, const cldenseVector* b,
                              clSParseSolverControl solverControl, clsparseControl control) {
    clsp::TraceRange trace_("clsparseDcsrcg");
    return cg_solve<double, double>(x, A, b, solverControl, control);
}

clsparseStatus clsparseScsrbicgStab(cldenseVector* x, const clsparseCsrMatrix* A,
                                    const cldenseVector* b, clSParseSolverControl solverControl,
                                    clsparseControl control) {
    clsp::TraceRange trace_("clsparseScsrbicgStab");
    return bicg_solve<float, float>(x, A, b, solverControl, control);
}

clsparseStatus clsparseDcsrbicgStab(cldenseVector* x, const clsparseCsrMatrix* A,
                                    const cldenseVector* b, clSParseSolverControl solverControl,
                                    clsparseControl control) {
    clsp::TraceRange trace_("clsparseDcsrbicgStab");
    return bicg_solve<double, double>(x, A, b, solverControl, control);
}

}  // extern "C"
