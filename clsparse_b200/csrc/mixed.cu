// Mixed-precision iterative refinement around CG (clsparseDcsrcgMixed) and
// BiCGStab (clsparseDcsrbicgStabMixed), project extensions with no reference
// counterpart.
//
// Outer loop, all in FP64 on the device: r = b - A x with the FP64 matrix,
// ||r||_2 / ||b||_2 is the stop test. Inner solve: Jacobi-PCG (the library's
// own CG) on A d = r / ||b||_2 with the matrix values rounded to FP32 or BF16
// (column indices, row pointers and the CSR-Adaptive meta are shared with the
// FP64 matrix) and FP32 vectors, accumulated in FP32. Then x += ||b||_2 * d
// in FP64. The inner tolerance is relative (L2) to the inner right-hand side.
//
// The inner solves are not restarts: after the first, each continues the
// previous one's search direction with only the residual replaced by the new
// FP64 true residual ("reliable updates" / residual replacement: G. Sleijpen
// and H. van der Vorst, Computing 56 (1996); H. van der Vorst and Q. Ye, SIAM
// J. Sci. Comput. 22 (2000)). A restarted CG throws away its Krylov space at
// every refinement step and, on ill-conditioned systems, needs about twice
// the FP64 iteration count; the continued one stays close to it.
#include <cmath>
#include <cstring>
#include <type_traits>

#include "device_common.cuh"
#include "dia.h"
#include "internal.h"

namespace clsp {
namespace {

constexpr int kThreads = 256;

uint32_t grid_for(size_t n, int sms) {
    size_t c = (n + kThreads * 4 - 1) / (kThreads * 4);
    size_t cap = static_cast<size_t>(sms) * 8;
    if (cap > static_cast<size_t>(kMaxReduceCtas)) cap = kMaxReduceCtas;
    if (c > cap) c = cap;
    return static_cast<uint32_t>(c ? c : 1);
}

template <typename V>
__global__ void round_values_kernel(const double* __restrict__ src, V* __restrict__ dst, size_t n) {
    const size_t stride = static_cast<size_t>(gridDim.x) * blockDim.x;
    for (size_t i = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride) {
        if constexpr (std::is_same_v<V, __nv_bfloat16>)
            dst[i] = __double2bfloat16(src[i]);
        else
            dst[i] = static_cast<V>(src[i]);
    }
}

// r = b - y; r32 = r * inv_scale (rounded to FP32); out = {sum r^2, sum b^2}.
__global__ void __launch_bounds__(kThreads)
    residual_kernel(const double* __restrict__ b, const double* __restrict__ y, float* __restrict__ r32,
                    double inv_scale, size_t n, double* parts, uint32_t* ticket, double* out) {
    double acc[2] = {0.0, 0.0};
    const size_t stride = static_cast<size_t>(gridDim.x) * kThreads;
    for (size_t i = static_cast<size_t>(blockIdx.x) * kThreads + threadIdx.x; i < n; i += stride) {
        const double bi = b[i];
        const double ri = bi - y[i];
        r32[i] = static_cast<float>(ri * inv_scale);
        acc[0] += ri * ri;
        acc[1] += bi * bi;
    }
    double tot[2];
    if (dev::grid_reduce_last<2>(acc, parts, ticket, tot) && threadIdx.x == 0) {
        out[0] = tot[0];
        out[1] = tot[1];
    }
}

__global__ void update_kernel(double* __restrict__ x, const float* __restrict__ d, double scale, size_t n) {
    const size_t stride = static_cast<size_t>(gridDim.x) * blockDim.x;
    for (size_t i = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride)
        x[i] += scale * static_cast<double>(d[i]);
}

MixedWork& work_of(clsparseControl c) {
    if (!c->mixed_work) {
        c->mixed_work = std::make_unique<MixedWork>();
        cudaMallocHost(&c->mixed_work->pinned, 64);
    }
    return *c->mixed_work;
}

// Learned factor M^-1 = G^T G for the inner solves (null: Jacobi).
struct Factor {
    CsrView<__nv_bfloat16> G, GT;
    clsparseB200Spai net = nullptr;  // owner of the views (metas made on first CSR use)
};

// The inner CG solves on diagonal storage (dia.cu) when A -- and the learned
// factor's G and G^T -- have few distinct column offsets: the low-precision
// copy of A is laid out by diagonal instead of in CSR, and each inner solve
// is one fused cooperative launch.
template <typename V>
struct BandedInner {
    bool on = false;
    DiaMat<V> A;
    DiaMat<__nv_bfloat16> G, GT;
    float* invD = nullptr;
    float* vec[7] = {};  // r0, r1, p0, p1, q, t, z
    int* status = nullptr;
    bool have_p = false;  // a previous solve left a direction to continue
    int pbuf = 0;
    double rz_prev = 0.0;
};

template <typename V>
bool setup_banded(BandedInner<V>& bi, const clsparseCsrMatrix* A, const Factor* factor, MixedWork& w,
                  bool jacobi, clsparseControl c) {
    if (!dia_enabled()) return false;
    if (!w.dia) w.dia = std::make_unique<DiaWork>();
    DiaWork& dw = *w.dia;
    cudaStream_t s = c->stream;
    const uint32_t n = A->num_rows, nnz = A->num_nonzeros;
    const uint32_t* rp = dev_ptr<const uint32_t>(A->row_pointer, A->off_row_pointer);
    const uint32_t* cols = dev_ptr<const uint32_t>(A->col_indices, A->off_col_indices);
    DiaOffsets oa, og, ot;
    if (dia_detect(rp, cols, n, nnz, dw, s, oa) != clsparseSuccess) return false;
    if (factor) {
        if (dia_detect(factor->G.rp, factor->G.cols, n, factor->G.nnz, dw, s, og) != clsparseSuccess ||
            dia_detect(factor->GT.rp, factor->GT.cols, n, factor->GT.nnz, dw, s, ot) != clsparseSuccess)
            return false;
    }
    // padded diagonal counts of the engine's builds; the fallback from the
    // learned factor to Jacobi runs the same A, so A takes the learned class
    int ca = 0, cg = 0;
    dia_classes(oa.nd, factor ? std::max(og.nd, ot.nd) : 0, factor != nullptr, ca, cg);
    if (ca == 0) return false;
    if (dia_build<double, V>(rp, cols, dev_ptr<const double>(A->values, A->off_values), n, oa, ca, dw.A, s, bi.A) !=
        clsparseSuccess)
        return false;
    if (factor && (dia_build<__nv_bfloat16, __nv_bfloat16>(factor->G.rp, factor->G.cols, factor->G.vals, n, og, cg,
                                                           dw.G, s, bi.G) != clsparseSuccess ||
                   dia_build<__nv_bfloat16, __nv_bfloat16>(factor->GT.rp, factor->GT.cols, factor->GT.vals, n, ot,
                                                           cg, dw.GT, s, bi.GT) != clsparseSuccess))
        return false;
    const size_t stride = (static_cast<size_t>(n) + 63) & ~size_t(63);
    if (dw.vecs.ensure(9 * stride * sizeof(float) + 256) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    float* base = static_cast<float*>(dw.vecs.ptr);
    bi.invD = base;
    for (int k = 0; k < 7; ++k) bi.vec[k] = base + (k + 1) * stride;
    bi.status = reinterpret_cast<int*>(base + 9 * stride);
    cudaMemsetAsync(bi.status, 0, sizeof(int), s);
    if constexpr (std::is_same_v<V, __nv_bfloat16>) {
        // BF16 values: the main diagonal in FP32 carrying each row's rounding
        // (row sums kept), so the inner operator stays SPD and within 1 +- 2^-9
        // of A in the energy norm; plain rounding can make a nearly singular
        // diffusion operator indefinite
        if (dia_compensate_diag<V>(rp, cols, dev_ptr<const double>(A->values, A->off_values), n, bi.A,
                                   base + 8 * stride, s) != clsparseSuccess)
            return false;
    }
    if (jacobi) {
        // a zero diagonal entry: the CSR path runs and reports it
        int zero = 0;
        if (dia_jacobi<V>(bi.A, n, bi.invD, bi.status, s) != clsparseSuccess ||
            cudaMemcpyAsync(&zero, bi.status, sizeof(int), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
            cudaStreamSynchronize(s) != cudaSuccess || zero != 0)
            return false;
    }
    bi.on = true;
    return true;
}

// One inner solve on the banded engine, with the bookkeeping of the CSR
// engine's: inner.nIters (iterations - 1), the reached relative residual,
// the device status bits.
template <typename V>
clsparseStatus banded_solve(BandedInner<V>& bi, bool learned, bool jacobi, float* x, const float* b, uint32_t n,
                            double tol, bool warm, _solverControl& inner, MixedWork& w, clsparseControl c) {
    DiaPcgArgs<V, __nv_bfloat16> a;
    a.A = bi.A;
    a.G = bi.G;
    a.GT = bi.GT;
    a.invD = jacobi ? bi.invD : nullptr;
    a.b = b;
    a.x = x;
    a.r[0] = bi.vec[0];
    a.r[1] = bi.vec[1];
    a.p[0] = bi.vec[2];
    a.p[1] = bi.vec[3];
    a.q = bi.vec[4];
    a.t = bi.vec[5];
    a.z = bi.vec[6];
    a.n = n;
    a.gt_diag = 0;
    a.gt_halo = 0;
    for (int d = bi.GT.nd - 1; d >= 0; --d) {  // the first zero offset: the real diagonal, padding comes after
        if (bi.GT.off[d] == 0) a.gt_diag = d;
        if (bi.GT.off[d] > 0) a.gt_halo = std::max<uint32_t>(a.gt_halo, static_cast<uint32_t>(bi.GT.off[d]));
    }
    DiaPcgState st;
    st.tol = tol;
    st.max_iters = inner.maxIters;
    st.warm = (warm && bi.have_p && bi.rz_prev > 0.0) ? 1 : 0;
    st.pbuf = bi.pbuf;
    st.rz_prev = bi.rz_prev;
    const clsparseStatus stt = dia_pcg_solve<V, __nv_bfloat16>(a, learned, *w.dia, c, st);
    if (stt != clsparseSuccess) {
        inner.deviceStatus = static_cast<cl_uint>(st.status);
        return stt;
    }
    inner.nIters = st.iters - 1;
    inner.currentResidual = st.rr0 > 0.0 ? std::sqrt(st.rr / st.rr0) : 0.0;
    inner.deviceStatus = static_cast<cl_uint>(st.status);
    bi.have_p = st.iters > 0 && st.status == 0;
    bi.pbuf = st.pbuf;
    bi.rz_prev = st.rz_prev;
    return clsparseSuccess;
}

enum class Inner { Cg, BiCgStab };

template <typename V>
clsparseStatus refine(cldenseVector* xv, const clsparseCsrMatrix* A, const cldenseVector* bv,
                      clSParseSolverControl sc, double inner_tol, clsparseB200MixedInfo* info,
                      clsparseControl c, const Factor* factor = nullptr, int* fell_back = nullptr,
                      Inner method = Inner::Cg) {
    const size_t n = A->num_rows, nnz = A->num_nonzeros;
    MixedWork& w = work_of(c);
    if (w.lowvals.ensure(nnz * sizeof(V) + 256) != cudaSuccess || w.y.ensure(n * 8 + 256) != cudaSuccess ||
        w.r32.ensure(n * 4 + 256) != cudaSuccess || w.d.ensure(n * 4 + 256) != cudaSuccess ||
        w.parts.ensure((2 * kMaxReduceCtas + 8) * sizeof(double)) != cudaSuccess) {
        cudaGetLastError();
        return clsparseOutOfResources;
    }
    cudaStream_t s = c->stream;
    const double* Avals = dev_ptr<const double>(A->values, A->off_values);
    double* x = dev_ptr<double>(xv->values, xv->off_values);
    const double* b = dev_ptr<const double>(bv->values, bv->off_values);
    V* lv = static_cast<V*>(w.lowvals.ptr);
    BandedInner<V> bi;
    if (method == Inner::Cg)
        setup_banded<V>(bi, A, factor, w, sc->preconditioner == DIAGONAL, c);
    if (!bi.on) round_values_kernel<V><<<grid_for(nnz, c->sm_count), kThreads, 0, s>>>(Avals, lv, nnz);
    Factor csr_factor;
    if (factor != nullptr && !bi.on && factor->net != nullptr && (!factor->G.meta || !factor->GT.meta)) {
        // the CSR inner solves apply G and G^T with their CSR-Adaptive metas
        const clsparseStatus ms = spai_ensure_metas(factor->net, c);
        if (ms != clsparseSuccess) return ms;
        CsrView<float> g32, gt32;
        CsrView<double> g64, gt64;
        csr_factor.net = factor->net;
        if (!spai_factor_views(factor->net, csr_factor.G, csr_factor.GT, g32, gt32, g64, gt64))
            return clsparseStructInvalid;
        factor = &csr_factor;
    }

    // FP64 operator and the low-precision copy sharing its structure and meta
    CsrView<double> A64{Avals, dev_ptr<const uint32_t>(A->col_indices, A->off_col_indices),
                        dev_ptr<const uint32_t>(A->row_pointer, A->off_row_pointer), A->num_rows,
                        A->num_cols, A->num_nonzeros, static_cast<const matrix_meta*>(A->meta)};
    clsparseCsrMatrix Alow = *A;
    Alow.values = lv;
    Alow.off_values = 0;

    double* consts = static_cast<double*>(w.parts.ptr);  // [0]=1, [1]=0, [2..3] results
    uint32_t* ticket = reinterpret_cast<uint32_t*>(consts + 4);
    double* parts = consts + 8;
    const double h_consts[4] = {1.0, 0.0, 0.0, 0.0};
    cudaMemcpyAsync(consts, h_consts, sizeof(h_consts), cudaMemcpyHostToDevice, s);
    cudaMemsetAsync(ticket, 0, 4 * sizeof(uint32_t), s);

    cldenseVector dvec{static_cast<clsparseIdx_t>(n), w.d.ptr, 0};
    cldenseVector rvec{static_cast<clsparseIdx_t>(n), w.r32.ptr, 0};
    _solverControl inner;
    inner.preconditioner = sc->preconditioner;
    inner.normType = 1;
    inner.printMode = QUIET;
    inner.stopOnNonFinite = 1;  // a broken factor costs one inner iteration, not the budget

    const double target = sc->relativeTolerance;
    const int max_inner_total = sc->maxIters;
    double bnorm = -1.0, res = 0.0, prev = 1e300;
    int outer = 0, inner_total = 0, stalls = 0;
    WarmStart ws;              // continuation of the previous inner solve
    bool have_prev = false;    // an inner solve ran whose direction can be continued
    bool prev_factor = false;  // ... and it used the learned factor
    double predicted = 0.0;    // true residual the last inner solve's recursion promises
    double* hres = static_cast<double*>(w.pinned);
    const uint32_t g = grid_for(n, c->sm_count);
    clsparseStatus st = clsparseSuccess;
    bool use_factor = factor != nullptr;
    info->converged = 0;
    for (;;) {
        SpmvEpilogue none;
        if (launch_csrmv<double, double>(A64, consts, consts + 1, x, static_cast<double*>(w.y.ptr), false,
                                         none, s) != cudaSuccess)
            return clsparseInvalidKernelExecution;
        const double inv = bnorm > 0 ? 1.0 / bnorm : 1.0;
        residual_kernel<<<g, kThreads, 0, s>>>(b, static_cast<const double*>(w.y.ptr),
                                               static_cast<float*>(w.r32.ptr), inv, n, parts, ticket,
                                               consts + 2);
        cudaMemcpyAsync(hres, consts + 2, 2 * sizeof(double), cudaMemcpyDeviceToHost, s);
        if (cudaStreamSynchronize(s) != cudaSuccess) return clsparseInvalidKernelExecution;
        if (bnorm < 0) {
            bnorm = std::sqrt(hres[1]);
            if (bnorm == 0.0) {
                cudaMemcpyAsync(x, b, n * sizeof(double), cudaMemcpyDeviceToDevice, s);
                info->outerIterations = 0;
                info->innerIterations = 0;
                info->trueResidual = 0.0;
                info->initialTrueResidual = 0.0;
                info->converged = 1;
                return finish_call(c);
            }
            // first pass computed r without scaling; redo the rounding
            continue;
        }
        res = std::sqrt(hres[0]) / bnorm;
        if (outer == 0) info->initialTrueResidual = res;
        if (res <= target) {
            info->converged = 1;
            break;
        }
        if (inner_total >= max_inner_total) break;
        // The learned factor stalls when an outer step fails to halve the
        // residual or its inner solve broke down: continue with Jacobi.
        const bool breakdown = (inner.deviceStatus & 0x14u) != 0;
        if (use_factor && outer > 0 && (res > 0.5 * prev || breakdown)) {
            use_factor = false;
            if (fell_back) *fell_back = 1;
        } else if (res > 0.5 * prev && ++stalls >= 3) {
            break;  // refinement no longer contracts
        }
        prev = res;
        // inner solve A_low d = r / ||b||, from d = 0
        cudaMemsetAsync(w.d.ptr, 0, n * sizeof(float), s);
        inner.maxIters = max_inner_total - inner_total;
        inner.relativeTolerance = inner_tol;
        inner.absoluteTolerance = 0.0;
        // Continue the previous direction only while the recursion is
        // trustworthy: same method, no breakdown, the inner solve reached its
        // tolerance, and the FP64 true residual is within 2x of what the
        // inner recursive residual predicted. Otherwise restart (p = M r):
        // the residual-replacement criterion of van der Vorst and Ye.
        ws.warm = have_prev && prev_factor == use_factor && !breakdown && res <= 2.0 * predicted;
        inner.nIters = 0;
        inner.deviceStatus = 0;
        if (bi.on)
            st = banded_solve<V>(bi, use_factor, sc->preconditioner == DIAGONAL, static_cast<float*>(w.d.ptr),
                                 static_cast<const float*>(w.r32.ptr), static_cast<uint32_t>(n), inner_tol, ws.warm,
                                 inner, w, c);
        else if (method == Inner::BiCgStab)  // restarted every refinement step
            st = bicg_solve_typed<V, float>(&dvec, &Alow, &rvec, &inner, c);
        else if (use_factor)
            st = pcg_factor_typed<V, float, __nv_bfloat16>(&dvec, &Alow, &rvec, &inner, factor->G, factor->GT,
                                                            c, &ws);
        else
            st = cg_solve_typed<V, float>(&dvec, &Alow, &rvec, &inner, c, &ws);
        if (st != clsparseSuccess) return st;
        have_prev = inner.currentResidual <= inner_tol;
        prev_factor = use_factor;
        predicted = res * inner.currentResidual;
        inner_total += inner.nIters + 1;
        // A correction from an inner solve that went non-finite is dropped: x
        // keeps its last FP64 value and the next step (with Jacobi, if the
        // learned factor caused it) starts from there.
        if ((inner.deviceStatus & 0x10u) == 0)
            update_kernel<<<g, kThreads, 0, s>>>(x, static_cast<const float*>(w.d.ptr), bnorm, n);
        ++outer;
    }
    info->outerIterations = outer;
    info->innerIterations = inner_total;
    info->trueResidual = res;
    sc->nIters = inner_total;
    sc->currentResidual = res;
    sc->initialResidual = info->initialTrueResidual;
    return finish_call(c);
}

}  // namespace
}  // namespace clsp

using namespace clsp;

extern "C" {

clsparseStatus clsparseDcsrcgMixed(cldenseVector* x, const clsparseCsrMatrix* A, const cldenseVector* b,
                                   clSParseSolverControl solverControl, cl_int innerPrecision,
                                   cl_double innerTolerance, clsparseB200MixedInfo* info,
                                   clsparseControl control) {
    clsp::TraceRange trace_("clsparseDcsrcgMixed");
    clsparseStatus st = check_entry(control);
    if (st != clsparseSuccess) return st;
    if (solverControl == nullptr) return clsparseInvalidSolverControlObject;
    if (!x || !A || !b || !info) return clsparseInvalidValue;
    if (A->num_rows != A->num_cols || A->num_rows != x->num_values || A->num_cols != b->num_values)
        return clsparseInvalidSystemSize;
    if (innerPrecision != 0 && innerPrecision != 1) return clsparseInvalidType;
    std::memset(info, 0, sizeof(*info));
    if (A->num_rows == 0) return clsparseSuccess;
    DeviceGuard g(control->device);
    if (innerPrecision == 0)
        return refine<float>(x, A, b, solverControl, innerTolerance, info, control);
    return refine<__nv_bfloat16>(x, A, b, solverControl, innerTolerance, info, control);
}

clsparseStatus clsparseDcsrbicgStabMixed(cldenseVector* x, const clsparseCsrMatrix* A, const cldenseVector* b,
                                         clSParseSolverControl solverControl, cl_int innerPrecision,
                                         cl_double innerTolerance, clsparseB200MixedInfo* info,
                                         clsparseControl control) {
    clsp::TraceRange trace_("clsparseDcsrbicgStabMixed");
    clsparseStatus st = check_entry(control);
    if (st != clsparseSuccess) return st;
    if (solverControl == nullptr) return clsparseInvalidSolverControlObject;
    if (!x || !A || !b || !info) return clsparseInvalidValue;
    if (A->num_rows != A->num_cols || A->num_rows != x->num_values || A->num_cols != b->num_values)
        return clsparseInvalidSystemSize;
    if (innerPrecision != 0 && innerPrecision != 1) return clsparseInvalidType;
    std::memset(info, 0, sizeof(*info));
    if (A->num_rows == 0) return clsparseSuccess;
    DeviceGuard g(control->device);
    if (innerPrecision == 0)
        return refine<float>(x, A, b, solverControl, innerTolerance, info, control, nullptr, nullptr,
                             Inner::BiCgStab);
    return refine<__nv_bfloat16>(x, A, b, solverControl, innerTolerance, info, control, nullptr, nullptr,
                                 Inner::BiCgStab);
}

clsparseStatus clsparseDcsrcgLearned(cldenseVector* x, const clsparseCsrMatrix* A, const cldenseVector* b,
                                     clSParseSolverControl solverControl, clsparseB200Spai spai,
                                     cl_int innerPrecision, cl_double innerTolerance,
                                     clsparseB200MixedInfo* info, cl_int* fellBack, clsparseControl control) {
    clsp::TraceRange trace_("clsparseDcsrcgLearned");
    clsparseStatus st = check_entry(control);
    if (st != clsparseSuccess) return st;
    if (solverControl == nullptr) return clsparseInvalidSolverControlObject;
    if (!x || !A || !b || !info) return clsparseInvalidValue;
    if (A->num_rows != A->num_cols || A->num_rows != x->num_values || A->num_cols != b->num_values)
        return clsparseInvalidSystemSize;
    CsrView<__nv_bfloat16> G16, GT16;
    CsrView<float> G32, GT32;
    CsrView<double> G64, GT64;
    if (!spai_factor_views(spai, G16, GT16, G32, GT32, G64, GT64)) return clsparseStructInvalid;
    if (G16.nrows != A->num_rows) return clsparseInvalidSystemSize;
    std::memset(info, 0, sizeof(*info));
    int fb = 0;
    DeviceGuard g(control->device);
    if (innerPrecision == 2) {
        st = spai_ensure_metas(spai, control);
        if (st != clsparseSuccess) return st;
        spai_factor_views(spai, G16, GT16, G32, GT32, G64, GT64);
        // plain FP64 PCG with M^-1 = G^T G, L2 stop test on the recursive residual
        _solverControl sc = *solverControl;
        sc.normType = 1;
        sc.nIters = 0;
        st = pcg_factor_typed<double, double, double>(x, A, b, &sc, G64, GT64, control);
        if (st != clsparseSuccess) return st;
        info->innerIterations = sc.nIters + 1;
        info->trueResidual = sc.currentResidual;
        info->initialTrueResidual = sc.initialResidual;
        info->converged = sc.currentResidual <= solverControl->relativeTolerance ? 1 : 0;
        solverControl->nIters = sc.nIters;
        solverControl->currentResidual = sc.currentResidual;
        if (fellBack) *fellBack = 0;
        return clsparseSuccess;
    }
    if (innerPrecision != 0 && innerPrecision != 1) return clsparseInvalidType;
    Factor f{G16, GT16, spai};
    if (innerPrecision == 0)
        st = refine<float>(x, A, b, solverControl, innerTolerance, info, control, &f, &fb);
    else
        st = refine<__nv_bfloat16>(x, A, b, solverControl, innerTolerance, info, control, &f, &fb);
    if (fellBack) *fellBack = fb;
    return st;
}

clsparseStatus clsparseB200SolverSetNormType(clSParseSolverControl solverControl, cl_int normType) {
    if (solverControl == nullptr) return clsparseInvalidSolverControlObject;
    if (normType != 1 && normType != 2) return clsparseInvalidValue;
    solverControl->normType = normType == 2 ? 1 : 0;
    return clsparseSuccess;
}

}  // extern "C"
