// Persistent CG / factorized-PCG: the whole solve in ONE cooperative launch.
//
// The graph form of the solvers (solvers.cu) runs three to five kernels per
// iteration; on matrices whose iteration moves a few tens of megabytes the
// launch and drain of each kernel dominate. Here every CTA stays resident for
// the whole solve and the grid meets at a software barrier where a kernel
// boundary used to be:
//
//   * SpMV phases: each CTA walks a static range of CSR-Adaptive row-block
//     words (balanced by nonzeros on the host, spmv_word.cuh does the word);
//     the dot product the solver needs of the result is fused into the row
//     writes, as in the graph form.
//   * vector phases: each CTA updates a contiguous slice of rows.
//   * reductions: each CTA writes its partial sums; the CTA that arrives last
//     at the barrier adds all partials in CTA order (so the result does not
//     depend on timing), publishes the totals and releases the barrier. Every
//     CTA then takes the same scalar steps on identical inputs, so all agree
//     on alpha, beta and the stop decision without another round trip.
//
// The iteration is the reference's operation for operation
// (src/library/solvers/conjugate-gradients.hpp:65-226, the L1 stop test of
// solver-control.hpp:47-64 and its bookkeeping), exactly as the graph form
// does it; the two forms give the same iterates up to reduction order.
//
// Safety: a cooperative launch guarantees that all CTAs are resident. Every
// barrier wait is bounded by the global timer; a wait that runs out sets an
// error flag, every CTA that sees it leaves, and the host reports
// clsparseInvalidKernelExecution with the barrier-timeout status bit.
#include <algorithm>
#include <cstdlib>
#include <vector>

#include "fused.h"
#include "grid_sync.cuh"
#include "spmv_word.cuh"

namespace clsp {
namespace {

// The rows [r0, r1) whose vector entries this CTA updates.
struct RowSlice {
    uint32_t r0, r1;
};

__device__ __forceinline__ RowSlice my_rows(uint32_t n) {
    const uint64_t c = blockIdx.x, G = gridDim.x;
    return RowSlice{static_cast<uint32_t>(c * n / G), static_cast<uint32_t>((c + 1) * n / G)};
}

// ---- row sinks of the SpMV phases ----

// y[row] = value.
template <typename T>
struct StoreSink {
    T* y;
    template <bool EXT>
    __device__ __forceinline__ void put(uint32_t row, dev::Acc<T, EXT> a) {
        y[row] = a.value();
    }
};

// y[row] = value; d += value * w[row].
template <typename T>
struct DotSink {
    T* y;
    const T* w;
    double d;
    template <bool EXT>
    __device__ __forceinline__ void put(uint32_t row, dev::Acc<T, EXT> a) {
        const T v = a.value();
        y[row] = v;
        d += static_cast<double>(v) * static_cast<double>(dev::ld_coherent(w + row));
    }
};

// Runs this CTA's words of M through adaptive_word.
// (Metas of the reference's row-block shape only.)
template <typename V, typename T, bool EXT, int NT, typename XS, typename Sink>
__device__ __forceinline__ void spmv_phase(const WordMat<V>& M, const XS& xs, Sink& sink, WordSmem<T>& sm) {
    const uint32_t wb = M.cta_words[blockIdx.x], we = M.cta_words[blockIdx.x + 1];
    const WordShape shape{kRowsForVector, kLongChunk};
    for (uint32_t w = wb; w < we; ++w) {
        adaptive_word<V, T, EXT, NT, static_cast<int>(kBlkSize)>(w, M.vals, M.cols, M.rp, xs, T(1), M.words,
                                                                 M.word_nnz, M.lo, M.hi, M.vec, M.lr_partial,
                                                                 M.lr_ticket, shape, sm, sink);
        __syncthreads();
    }
}

template <typename T>
__device__ __forceinline__ double norm_term(T v, int l2) {
    const double d = static_cast<double>(v);
    return l2 ? d * d : fabs(d);
}

__device__ __forceinline__ double norm_finish(double acc, int l2) { return l2 ? sqrt(acc) : acc; }

// Writes the CTA-local solver state back (CTA 0 at the end); status bits are
// OR-ed so that bits other CTAs raised in global memory stay.
template <typename T>
__device__ void store_state(SolverState<T>* dst, const SolverState<T>& S) {
    dst->norm_b = S.norm_b;
    dst->rz = S.rz;
    dst->rz_old = S.rz_old;
    dst->yp = S.yp;
    dst->alpha = S.alpha;
    dst->beta = S.beta;
    dst->norm_r = S.norm_r;
    dst->res = S.res;
    dst->init_res = S.init_res;
    dst->cur_res = S.cur_res;
    dst->iteration = S.iteration;
    dst->nIters = S.nIters;
    dst->done = S.done;
    dst->zero_b = S.zero_b;
    atomicOr(&dst->status_bits, S.status_bits);
    atomicMax(&dst->hist_len, S.hist_len);  // only CTA 0 records the history
}

// invD[row] = 1 / A[row,row] for this CTA's rows (first matching entry, as
// the reference's extract_diagonal, src/library/kernels/matrix_utils.cl:65-98).
template <typename V, typename T>
__device__ void extract_inv_diag(const WordMat<V>& A, RowSlice rs, T* __restrict__ invD, int* status) {
    const int lane = threadIdx.x & 31;
    const uint32_t warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    for (uint32_t row = rs.r0 + warp; row < rs.r1; row += nwarps) {
        const uint32_t nb = A.rp[row], ne = A.rp[row + 1];
        bool found = false;
        for (uint32_t base = nb; base < ne && !found; base += 32) {
            const uint32_t j = base + lane;
            const bool m = (j < ne) && (A.cols[j] == row);
            const unsigned ball = __ballot_sync(0xffffffffu, m);
            if (ball) {
                if (lane == __ffs(ball) - 1) {
                    const T v = dev::to_t<T>(A.vals[j]);
                    invD[row] = T(1) / v;
                    if (v == T(0)) atomicOr(status, kStatusZeroDiag);
                }
                found = true;
            }
        }
        if (!found && lane == 0) {
            invD[row] = T(0);
            atomicOr(status, kStatusMissingDiag);
        }
    }
}

template <typename T>
__device__ __forceinline__ T apply_jacobi(const T* invD, uint32_t i, T r) {
    return invD ? r * invD[i] : r;
}

// First stop test after r0 (conjugate-gradients.hpp:73-148); thread 0 only.
template <typename T>
__device__ void init_test(SolverState<T>& S, double nb, double nr, int l2) {
    S.norm_b = static_cast<T>(norm_finish(nb, l2));
    if (S.norm_b == T(0)) {
        S.zero_b = 1;
        S.done = 1;
        S.nIters = 0;
        return;
    }
    S.norm_r = static_cast<T>(norm_finish(nr, l2));
    S.res = S.norm_r / S.norm_b;
    S.init_res = static_cast<double>(S.res);
    S.cur_res = S.init_res;
    S.iteration = 0;
    if (blockIdx.x == 0) record_residual(&S, 0, S.init_res);
    // the stop test sees the iteration count the solver control held before
    // this solve, as the reference's does
    if (solver_finished(S, S.init_res)) {
        S.nIters = 0;
        S.done = 1;
    }
}

// Residual bookkeeping after x/r update (conjugate-gradients.hpp:186-224);
// thread 0 only.
template <typename T>
__device__ void step_test(SolverState<T>& S, double nr, int l2) {
    S.norm_r = static_cast<T>(norm_finish(nr, l2));
    S.res = S.norm_r / S.norm_b;
    S.nIters = S.iteration;
    S.iteration += 1;
    S.cur_res = static_cast<double>(S.res);
    if (blockIdx.x == 0) record_residual(&S, S.iteration, S.cur_res);
    if (!isfinite(S.cur_res)) S.status_bits |= kStatusNonFinite;
    S.done = solver_finished(S, S.cur_res) ? 1 : 0;
}

// Vector phases walk the CTA's rows four per thread at a time, loading all
// inputs of the four before storing anything, so a thread has four loads in
// flight instead of one.
constexpr int kVecUnroll = 4;

// PK = 0: CG with Jacobi (invD != nullptr) or no preconditioner;
// PK = 1: PCG with M^-1 = G^T G (G, Gt with values VG).
//
// Per iteration, PK = 0: [q = A p, <q,p>] exchange(alpha) [x, r update,
// <r, M r>, ||r||] exchange(beta, stop test) [p = M r + beta p] barrier.
// PK = 1: [q = A p, <q,p>] exchange(alpha) [x, r, ||r||] exchange(stop test)
// [t = G r] barrier [z = G^T t, <z,r>] exchange(beta) [p = z + beta p] barrier.
template <typename V, typename T, typename VG, bool EXT, int PK, int NT>
__global__ void __launch_bounds__(NT, 4) pcg_fused_kernel(FusedCgArgs<V, T, VG> a) {
    __shared__ WordSmem<T> sm;
    __shared__ GridSmem gs;
    __shared__ SolverState<T> S;
    if (threadIdx.x == 0) S = *a.st;
    __syncthreads();
    const FusedSync g = a.sync;
    unsigned long long epoch = 0;
    const RowSlice rs = my_rows(a.n);
    const int l2 = S.norm_type;
    // No __restrict__: these vectors are also read by other CTAs' phases.
    T* x = a.x;
    T* r = a.r;
    T* q = a.q;
    T* p = a.p;
    const T* invD = a.invD;

    if constexpr (PK == 0) {
        if (a.invD) extract_inv_diag(a.A, rs, a.invD, &a.st->status_bits);
    }
    {
        // q = A x
        StoreSink<T> sink{q};
        spmv_phase<V, T, EXT, NT>(a.A, DenseX<T, true>{x}, sink, sm);
    }
    if (!grid_sync(g, epoch, gs)) goto fail;
    {
        // r = b - q; (PK 0: p = z = M r); ||b||, ||r||, <r, z>
        double acc[3] = {0.0, 0.0, 0.0};
        for (uint32_t i = rs.r0 + threadIdx.x; i < rs.r1; i += NT) {
            const T bi = a.b[i];
            const T ri = bi - q[i];
            r[i] = ri;
            acc[0] += norm_term(bi, l2);
            acc[1] += norm_term(ri, l2);
            if constexpr (PK == 0) {
                const T zi = apply_jacobi(invD, i, ri);
                p[i] = zi;
                acc[2] += static_cast<double>(ri) * static_cast<double>(zi);
            }
        }
        double tot[3];
        if (!grid_exchange<3>(g, epoch, acc, tot, gs)) goto fail;
        if (threadIdx.x == 0) {
            init_test(S, tot[0], tot[1], l2);
            if constexpr (PK == 0) S.rz = static_cast<T>(tot[2]);
        }
        __syncthreads();
    }
    if (S.done) {
        if (S.zero_b)  // ||b|| == 0: x = b (conjugate-gradients.hpp:87-95)
            for (uint32_t i = rs.r0 + threadIdx.x; i < rs.r1; i += NT) x[i] = a.b[i];
        goto finish;
    }
    if constexpr (PK == 1) {
        // z0 = G^T (G r0), <r0, z0>, p = z0
        {
            StoreSink<T> sink{a.t};
            spmv_phase<VG, T, false, NT>(a.G, DenseX<T, true>{r}, sink, sm);
        }
        if (!grid_sync(g, epoch, gs)) goto fail;
        DotSink<T> sink{a.z, r, 0.0};
        spmv_phase<VG, T, false, NT>(a.Gt, DenseX<T, true>{a.t}, sink, sm);
        double v[1] = {sink.d}, tot[1];
        if (!grid_exchange<1>(g, epoch, v, tot, gs)) goto fail;
        if (threadIdx.x == 0) fin_pcg_rz0(&S, tot[0]);
        for (uint32_t i = rs.r0 + threadIdx.x; i < rs.r1; i += NT) p[i] = a.z[i];
        if (!grid_sync(g, epoch, gs)) goto fail;
    }

    for (;;) {
        // q = A p with <q, p>; alpha
        {
            DotSink<T> sink{q, p, 0.0};
            spmv_phase<V, T, EXT, NT>(a.A, DenseX<T, true>{p}, sink, sm);
            double v[1] = {sink.d}, tot[1];
            if (!grid_exchange<1>(g, epoch, v, tot, gs)) goto fail;
            if (threadIdx.x == 0) fin_cg_alpha(&S, tot[0]);
            __syncthreads();
        }
        const T alpha = S.alpha;
        // x += alpha p; r -= alpha q; (PK 0: z = M r, <r,z>); ||r||
        double acc[2] = {0.0, 0.0};
        for (uint32_t i0 = rs.r0 + threadIdx.x; i0 < rs.r1; i0 += kVecUnroll * NT) {
            T xi[kVecUnroll], pi[kVecUnroll], ri[kVecUnroll], qi[kVecUnroll], di[kVecUnroll];
#pragma unroll
            for (int u = 0; u < kVecUnroll; ++u) {
                const uint32_t i = i0 + u * NT;
                if (i < rs.r1) {
                    xi[u] = x[i];
                    pi[u] = p[i];
                    ri[u] = r[i];
                    qi[u] = q[i];
                    di[u] = (PK == 0 && invD) ? invD[i] : T(1);
                }
            }
#pragma unroll
            for (int u = 0; u < kVecUnroll; ++u) {
                const uint32_t i = i0 + u * NT;
                if (i < rs.r1) {
                    const T xn = xi[u] + alpha * pi[u];
                    const T rn = ri[u] - alpha * qi[u];
                    x[i] = xn;
                    r[i] = rn;
                    if constexpr (PK == 0) {
                        const T zn = invD ? rn * di[u] : rn;
                        acc[0] += static_cast<double>(rn) * static_cast<double>(zn);
                    }
                    acc[1] += norm_term(rn, l2);
                }
            }
        }
        if constexpr (PK == 0) {
            double tot[2];
            if (!grid_exchange<2>(g, epoch, acc, tot, gs)) goto fail;
            if (threadIdx.x == 0) {
                S.rz_old = S.rz;
                S.rz = static_cast<T>(tot[0]);
                S.beta = S.rz / S.rz_old;
                step_test(S, tot[1], l2);
            }
            __syncthreads();
            if (S.done) break;
            // p = M r + beta p (conjugate-gradients.hpp:211)
            const T beta = S.beta;
            for (uint32_t i0 = rs.r0 + threadIdx.x; i0 < rs.r1; i0 += kVecUnroll * NT) {
                T ri[kVecUnroll], pi[kVecUnroll], di[kVecUnroll];
#pragma unroll
                for (int u = 0; u < kVecUnroll; ++u) {
                    const uint32_t i = i0 + u * NT;
                    if (i < rs.r1) {
                        ri[u] = r[i];
                        pi[u] = p[i];
                        di[u] = invD ? invD[i] : T(1);
                    }
                }
#pragma unroll
                for (int u = 0; u < kVecUnroll; ++u) {
                    const uint32_t i = i0 + u * NT;
                    if (i < rs.r1) p[i] = (invD ? ri[u] * di[u] : ri[u]) + beta * pi[u];
                }
            }
        } else {
            double v[1] = {acc[1]}, tot[1];
            if (!grid_exchange<1>(g, epoch, v, tot, gs)) goto fail;
            if (threadIdx.x == 0) step_test(S, tot[0], l2);
            __syncthreads();
            if (S.done) break;
            // z = G^T (G r) with <z, r>; beta; p = z + beta p
            {
                StoreSink<T> sink{a.t};
                spmv_phase<VG, T, false, NT>(a.G, DenseX<T, true>{r}, sink, sm);
            }
            if (!grid_sync(g, epoch, gs)) goto fail;
            DotSink<T> sink{a.z, r, 0.0};
            spmv_phase<VG, T, false, NT>(a.Gt, DenseX<T, true>{a.t}, sink, sm);
            double w[1] = {sink.d}, tot2[1];
            if (!grid_exchange<1>(g, epoch, w, tot2, gs)) goto fail;
            if (threadIdx.x == 0) fin_pcg_rz(&S, tot2[0]);
            __syncthreads();
            const T beta = S.beta;
            for (uint32_t i0 = rs.r0 + threadIdx.x; i0 < rs.r1; i0 += kVecUnroll * NT) {
                T zi[kVecUnroll], pi[kVecUnroll];
#pragma unroll
                for (int u = 0; u < kVecUnroll; ++u) {
                    const uint32_t i = i0 + u * NT;
                    if (i < rs.r1) {
                        zi[u] = a.z[i];
                        pi[u] = p[i];
                    }
                }
#pragma unroll
                for (int u = 0; u < kVecUnroll; ++u) {
                    const uint32_t i = i0 + u * NT;
                    if (i < rs.r1) p[i] = zi[u] + beta * pi[u];
                }
            }
        }
        if (!grid_sync(g, epoch, gs)) goto fail;  // p complete before the next SpMV
    }
finish:
    if (blockIdx.x == 0 && threadIdx.x == 0) store_state(a.st, S);
    return;
fail:
    if (threadIdx.x == 0) atomicOr(&a.st->status_bits, kStatusBarrierTimeout);
}

// CTAs per SM of one kernel instantiation (resident limit), cached.
template <typename Kern>
int resident_per_sm(Kern k, int nt) {
    int b = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k, nt, 0) != cudaSuccess) {
        cudaGetLastError();
        return 1;
    }
    return b > 0 ? b : 1;
}

int ctas_per_sm_cap() {
    static int cap = [] {
        const char* e = std::getenv("CLSPARSE_B200_FUSED_CTAS_PER_SM");
        const int v = e ? std::atoi(e) : 4;
        return v > 0 ? v : 4;
    }();
    return cap;
}

}  // namespace

void word_partition(const matrix_meta* m, uint32_t G, std::vector<uint32_t>& out) {
    const uint32_t W = static_cast<uint32_t>(m->num_words - 1);
    out.assign(G + 1, W);
    out[0] = 0;
    const std::vector<uint32_t>& wn = m->h_word_nnz;
    const uint64_t lo = wn.front(), total = static_cast<uint64_t>(wn.back()) - lo;
    uint32_t w = 0;
    for (uint32_t c = 1; c < G; ++c) {
        const uint64_t target = lo + total * c / G;
        while (w < W && wn[w] < target) ++w;
        out[c] = w;
    }
    out[G] = W;
}

template <typename V>
WordMat<V> word_mat(const CsrView<V>& A, const uint32_t* cta_words) {
    const matrix_meta* m = A.meta;
    WordMat<V> w;
    w.vals = A.vals;
    w.cols = A.cols;
    w.rp = A.rp;
    w.words = m->d_rowBlocks;
    w.word_nnz = m->d_word_nnz;
    w.cta_words = cta_words;
    w.lr_partial = m->d_lr_partial;
    w.lr_ticket = m->d_lr_ticket;
    w.lo = m->nnz_lo;
    w.hi = m->nnz_hi;
    w.vec = ((reinterpret_cast<uintptr_t>(A.vals) | reinterpret_cast<uintptr_t>(A.cols)) & 15u) == 0;
    return w;
}

template WordMat<double> word_mat<double>(const CsrView<double>&, const uint32_t*);
template WordMat<float> word_mat<float>(const CsrView<float>&, const uint32_t*);
template WordMat<__nv_bfloat16> word_mat<__nv_bfloat16>(const CsrView<__nv_bfloat16>&, const uint32_t*);

template <typename V, typename T, typename VG>
uint32_t fused_grid(int sm_count, bool ext, int pk) {
    constexpr int NT = kFusedThreads;
    int per_sm;
    if (pk == 1)
        per_sm = resident_per_sm(pcg_fused_kernel<V, T, VG, false, 1, NT>, NT);
    else if (ext)
        per_sm = resident_per_sm(pcg_fused_kernel<V, T, VG, true, 0, NT>, NT);
    else
        per_sm = resident_per_sm(pcg_fused_kernel<V, T, VG, false, 0, NT>, NT);
    per_sm = std::min(per_sm, ctas_per_sm_cap());
    return static_cast<uint32_t>(std::max(1, sm_count * per_sm));
}

template <typename V, typename T, typename VG>
cudaError_t launch_pcg_fused(const FusedCgArgs<V, T, VG>& a, uint32_t grid, bool ext, int pk, cudaStream_t s) {
    constexpr int NT = kFusedThreads;
    void* args[] = {const_cast<FusedCgArgs<V, T, VG>*>(&a)};
    const void* k;
    if (pk == 1)
        k = reinterpret_cast<const void*>(pcg_fused_kernel<V, T, VG, false, 1, NT>);
    else if (ext)
        k = reinterpret_cast<const void*>(pcg_fused_kernel<V, T, VG, true, 0, NT>);
    else
        k = reinterpret_cast<const void*>(pcg_fused_kernel<V, T, VG, false, 0, NT>);
    return cudaLaunchCooperativeKernel(k, dim3(grid), dim3(NT), args, 0, s);
}

#define CLSP_FUSED_INST(V, T, VG)                                                                    \
    template uint32_t fused_grid<V, T, VG>(int, bool, int);                                          \
    template cudaError_t launch_pcg_fused<V, T, VG>(const FusedCgArgs<V, T, VG>&, uint32_t, bool, int, \
                                                    cudaStream_t);
CLSP_FUSED_INST(double, double, double)
CLSP_FUSED_INST(float, float, float)
CLSP_FUSED_INST(__nv_bfloat16, float, float)
CLSP_FUSED_INST(float, float, __nv_bfloat16)
CLSP_FUSED_INST(__nv_bfloat16, float, __nv_bfloat16)
#undef CLSP_FUSED_INST

}  // namespace clsp
