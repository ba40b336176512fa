// One rank's device work of the row-partitioned CG (multi-GPU): the rank
// owns a contiguous range of rows; its vectors are local, and the vector the
// SpMV reads is an "extended" vector that holds the rank's own entries at
// ownOffset and, around them, the entries of other ranks that its rows
// reference (a halo received from the neighbours, or the whole vector after
// an all-gather). The collectives between the stages (the exchange of the
// extended vector, the all-reduce of the sums) are issued by the caller
// (torch.distributed / NCCL) on the same stream; every stage here is one
// kernel launch, and nothing reads a scalar back to the host.
//
// The iteration is CG in the Chronopoulos-Gear arrangement (A. T.
// Chronopoulos and C. W. Gear, "s-step iterative methods for symmetric linear
// systems", J. Comput. Appl. Math. 25 (1989)): with z = M r and w = A z,
//   gamma = <r, z>, delta = <w, z>, beta = gamma / gamma_old,
//   alpha = gamma / (delta - beta * gamma / alpha_old),
//   p = z + beta p,  s = w + beta s,  x += alpha p,  r -= alpha s,
// which is CG (s = A p) with the three sums of an iteration -- <r,z>, <w,z>
// and the L1 norm of r for the stop test -- formed after one SpMV and
// combined across ranks in ONE all-reduce of three FP64 values, where the
// reference's order (src/library/solvers/conjugate-gradients.hpp:162-226)
// needs <p, A p> before it can update r. The stop test, the residual it
// reports and the iteration count are the reference's:
// residuum = ||r||_1 / ||b||_1 after the update of loop k, finished when
// residuum <= relTol, residuum <= absTol * initial residuum or k >= maxIters
// (solver-control.hpp:47-64), nIters = k (conjugate-gradients.hpp:164,223);
// a zero right-hand side returns x = b (:87-95).
//
// The decisions (alpha, beta, stop) are taken on the device: every CTA of
// the update kernel computes them from the all-reduced sums (bitwise the same
// values on every rank), one thread records them, and once the solve has
// finished every later stage returns at once, so the caller may enqueue
// iterations in chunks and read the state only between chunks.
#include <cuda_runtime.h>
#include <stdint.h>

#include <cmath>
#include <new>

#include "device_common.cuh"
#include "internal.h"

namespace clsp {
namespace {

constexpr int kThreads = 256;

// state[] slots (FP64)
enum : int {
    kNb = 0,      // ||b||_1 (all ranks)
    kInit = 1,    // initial residuum
    kDone = 2,    // 1 once finished
    kIters = 3,   // nIters at the finish
    kCur = 4,     // last residuum
    kAlpha = 5,   // alpha of step j at kAlpha + (j & 1)
    kGamma = 7,   // gamma of step j at kGamma + (j & 1)
    kZeroB = 9,   // 1 when b == 0
    kStateLen = 16
};

// partials[k * G + cta]: 0 <r,z>, 2 ||r||_1, 3 ||b||_1 (update / residual
// kernels), 4 <w,z> (product kernel); red[4] = their totals over the CTAs
// (red[0] <r,z>, red[1] <w,z>, red[2] ||r||_1, red[3] ||b||_1).
constexpr int kSlots = 5;

struct Work {
    const uint32_t* rp;
    const uint32_t* cols;
    const double* vals;
    uint32_t n;        // local rows
    uint32_t own;      // own entries' offset in the extended vectors
    const double* invd;  // nullptr: no preconditioner
    const double* b;
    double* x;
    double* r;
    double* p;
    double* s;
    double* w;
    double* xext;
    double* zext;
    double* partials;
    double* red;
    double* state;
    uint32_t* ticket;
};

__device__ __forceinline__ bool is_done(const Work& a) {
    return *reinterpret_cast<volatile const double*>(a.state + kDone) != 0.0;
}

// Rows handled at once by a group of W lanes: U consecutive rows, whose
// loads are independent, so a group keeps U gathers in flight (short rows
// are latency-bound otherwise: row pointer, then column, then x).
template <int W>
struct RowsPerGroup {
    static constexpr int U = W <= 8 ? 4 : W == 16 ? 2 : 1;
};

// Sums of rows i0 .. i0 + U - 1 of A times v by a group of W lanes (rows at
// or past n are empty); valid in the group's first lane. Every lane of the
// warp calls it.
template <int W, int U>
__device__ __forceinline__ void rows_dot(const Work& a, uint32_t i0, const double* v, uint32_t lane,
                                         double (&acc)[U]) {
    uint32_t e[U], end[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
        const uint32_t i = min(i0 + u, a.n);
        e[u] = __ldg(a.rp + i) + lane;
        end[u] = i0 + u < a.n ? __ldg(a.rp + i + 1) : 0u;
        acc[u] = 0.0;
    }
    bool more = true;
    while (more) {
        more = false;
#pragma unroll
        for (int u = 0; u < U; ++u) {
            if (e[u] < end[u]) {
                acc[u] = fma(dev::ld_stream(a.vals + e[u]), __ldg(v + dev::ld_stream(a.cols + e[u])), acc[u]);
                e[u] += W;
                more |= e[u] < end[u];
            }
        }
    }
#pragma unroll
    for (int u = 0; u < U; ++u)
#pragma unroll
        for (int o = W / 2; o > 0; o >>= 1) acc[u] += __shfl_down_sync(0xffffffffu, acc[u], o, W);
}

// x (local) into the extended vector's own entries.
__global__ void __launch_bounds__(kThreads) load_own_kernel(Work a) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < a.n; i += gridDim.x * blockDim.x)
        a.xext[a.own + i] = a.x[i];
}

// r = b - A xext, z = M r into zext's own entries; partial <r,z>, ||r||_1,
// ||b||_1.
template <int W>
__global__ void __launch_bounds__(kThreads, 8) residual_kernel(Work a) {
    __shared__ double red[32];
    constexpr int U = RowsPerGroup<W>::U;
    constexpr uint32_t kRowsPerCta = (kThreads / W) * U;
    const uint32_t lane = threadIdx.x % W;
    double rz = 0.0, nr = 0.0, nb = 0.0;
    const uint32_t n_pad = (a.n + kRowsPerCta - 1) / kRowsPerCta * kRowsPerCta;
    for (uint32_t i0 = blockIdx.x * kRowsPerCta + (threadIdx.x / W) * U; i0 < n_pad; i0 += gridDim.x * kRowsPerCta) {
        double ax[U];
        rows_dot<W, U>(a, i0, a.xext, lane, ax);
        if (lane == 0) {
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const uint32_t i = i0 + u;
                if (i < a.n) {
                    const double bi = a.b[i];
                    const double ri = bi - ax[u];
                    const double zi = a.invd ? ri * a.invd[i] : ri;
                    a.r[i] = ri;
                    a.zext[a.own + i] = zi;
                    rz = fma(ri, zi, rz);
                    nr += fabs(ri);
                    nb += fabs(bi);
                }
            }
        }
    }
    const uint32_t G = gridDim.x;
    rz = dev::block_sum(rz, red);
    nr = dev::block_sum(nr, red);
    nb = dev::block_sum(nb, red);
    if (threadIdx.x == 0) {
        a.partials[0 * G + blockIdx.x] = rz;
        a.partials[2 * G + blockIdx.x] = nr;
        a.partials[3 * G + blockIdx.x] = nb;
    }
}

// w = A zext, partial <w,z>; the CTA that arrives last adds every slot's
// partials in CTA order into red[].
template <int W>
__global__ void __launch_bounds__(kThreads, 8) product_kernel(Work a) {
    __shared__ double red[32];
    __shared__ bool last;
    if (is_done(a)) {
        if (blockIdx.x == 0 && threadIdx.x < 4) a.red[threadIdx.x] = 0.0;
        return;
    }
    constexpr int U = RowsPerGroup<W>::U;
    constexpr uint32_t kRowsPerCta = (kThreads / W) * U;
    const uint32_t lane = threadIdx.x % W;
    double wz = 0.0;
    const uint32_t n_pad = (a.n + kRowsPerCta - 1) / kRowsPerCta * kRowsPerCta;
    for (uint32_t i0 = blockIdx.x * kRowsPerCta + (threadIdx.x / W) * U; i0 < n_pad; i0 += gridDim.x * kRowsPerCta) {
        double wv[U];
        rows_dot<W, U>(a, i0, a.zext, lane, wv);
        if (lane == 0) {
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const uint32_t i = i0 + u;
                if (i < a.n) {
                    a.w[i] = wv[u];
                    wz = fma(wv[u], a.zext[a.own + i], wz);
                }
            }
        }
    }
    const uint32_t G = gridDim.x;
    wz = dev::block_sum(wz, red);
    if (threadIdx.x == 0) {
        a.partials[4 * G + blockIdx.x] = wz;
        last = dev::ticket_arrive(a.ticket) == G - 1;
    }
    __syncthreads();
    if (!last) return;
    const int slot[4] = {0, 4, 2, 3};
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        double t = 0.0;
        for (uint32_t c = threadIdx.x; c < G; c += blockDim.x) t += __ldcg(a.partials + slot[k] * G + c);
        t = dev::block_sum(t, red);
        if (threadIdx.x == 0) a.red[k] = t;
    }
    if (threadIdx.x == 0) *a.ticket = 0u;
}

// Step j: the stop decision on the sums of step j - 1 (or of the start, j =
// 0), then alpha, beta and the vector updates; partial <r,z>, ||r||_1 of the
// new residual.
__global__ void __launch_bounds__(kThreads) update_kernel(Work a, int j, double rel, double abs_tol, int max_iters) {
    __shared__ double red[32];
    if (is_done(a)) return;
    const double g = a.red[0], d = a.red[1], nr = a.red[2];
    const bool lead = blockIdx.x == 0 && threadIdx.x == 0;
    const double nb = j == 0 ? a.red[3] : a.state[kNb];
    if (j == 0 && nb == 0.0) {
        // zero right-hand side: x = b, nothing iterated
        for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < a.n; i += gridDim.x * blockDim.x) a.x[i] = a.b[i];
        if (lead) {
            a.state[kNb] = 0.0;
            a.state[kInit] = 0.0;
            a.state[kCur] = 0.0;
            a.state[kIters] = 0.0;
            a.state[kZeroB] = 1.0;
            a.state[kDone] = 1.0;
        }
        return;
    }
    const double res = nr / nb;
    const double init = j == 0 ? res : a.state[kInit];
    const int n_iters = j == 0 ? 0 : j - 1;
    if (res <= rel || res <= abs_tol * init || n_iters >= max_iters) {
        if (lead) {
            if (j == 0) {
                a.state[kNb] = nb;
                a.state[kInit] = res;
            }
            a.state[kCur] = res;
            a.state[kIters] = n_iters;
            a.state[kDone] = 1.0;
        }
        return;
    }
    double alpha, beta;
    if (j == 0) {
        beta = 0.0;
        alpha = g / d;
    } else {
        const double g_old = a.state[kGamma + ((j - 1) & 1)];
        const double a_old = a.state[kAlpha + ((j - 1) & 1)];
        beta = g / g_old;
        alpha = g / (d - beta * g / a_old);
    }
    if (lead) {
        if (j == 0) {
            a.state[kNb] = nb;
            a.state[kInit] = res;
        }
        a.state[kCur] = res;
        a.state[kGamma + (j & 1)] = g;
        a.state[kAlpha + (j & 1)] = alpha;
    }
    double rz = 0.0, n1 = 0.0;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < a.n; i += gridDim.x * blockDim.x) {
        const double zi = a.zext[a.own + i];
        const double wi = a.w[i];
        const double pi = j == 0 ? zi : fma(beta, a.p[i], zi);
        const double si = j == 0 ? wi : fma(beta, a.s[i], wi);
        a.p[i] = pi;
        a.s[i] = si;
        a.x[i] = fma(alpha, pi, a.x[i]);
        const double ri = fma(-alpha, si, a.r[i]);
        a.r[i] = ri;
        const double zn = a.invd ? ri * a.invd[i] : ri;
        a.zext[a.own + i] = zn;
        rz = fma(ri, zn, rz);
        n1 += fabs(ri);
    }
    const uint32_t G = gridDim.x;
    rz = dev::block_sum(rz, red);
    n1 = dev::block_sum(n1, red);
    if (threadIdx.x == 0) {
        a.partials[0 * G + blockIdx.x] = rz;
        a.partials[2 * G + blockIdx.x] = n1;
    }
}

// invd[i] = 1 / A[i][own + i]; bad[0] = 1 when a row lacks its diagonal or
// it is zero.
__global__ void __launch_bounds__(kThreads) inv_diag_kernel(Work a, double* invd, int* bad) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < a.n; i += gridDim.x * blockDim.x) {
        double dv = 0.0;
        for (uint32_t e = a.rp[i]; e < a.rp[i + 1]; ++e)
            if (a.cols[e] == a.own + i) dv += a.vals[e];
        if (dv == 0.0) {
            atomicExch(bad, 1);
            invd[i] = 0.0;
        } else {
            invd[i] = 1.0 / dv;
        }
    }
}

__global__ void gather_kernel(double* dst, const double* src, const uint32_t* idx, uint32_t count) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x)
        dst[i] = src[idx[i]];
}

__global__ void bad_columns_kernel(const uint32_t* cols, uint32_t nnz, uint32_t limit, int* bad) {
    for (uint32_t e = blockIdx.x * blockDim.x + threadIdx.x; e < nnz; e += gridDim.x * blockDim.x)
        if (cols[e] >= limit) atomicExch(bad, 1);
}

}  // namespace
}  // namespace clsp

struct _clsparseB200DistCg {
    clsp::Work w{};
    uint32_t next_ext = 0;    // length of the extended vectors
    uint32_t nnz = 0;
    int lanes = 2;            // lanes per row of the SpMV kernels
    uint32_t grid = 1;
    int device = 0;
    clsp::DeviceBuffer buf;   // r p s w invd | xext zext | partials | red state | ticket, flag
    int* d_flag = nullptr;
};

namespace {

using clsp::Work;

clsparseStatus launch_status() {
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? clsparseSuccess : clsparseInvalidKernelExecution;
}

clsparseStatus launch_residual(const _clsparseB200DistCg* h, cudaStream_t s) {
    using namespace clsp;
    switch (h->lanes) {
        case 2: residual_kernel<2><<<h->grid, kThreads, 0, s>>>(h->w); break;
        case 4: residual_kernel<4><<<h->grid, kThreads, 0, s>>>(h->w); break;
        case 8: residual_kernel<8><<<h->grid, kThreads, 0, s>>>(h->w); break;
        case 16: residual_kernel<16><<<h->grid, kThreads, 0, s>>>(h->w); break;
        default: residual_kernel<32><<<h->grid, kThreads, 0, s>>>(h->w); break;
    }
    return launch_status();
}

clsparseStatus launch_product(const _clsparseB200DistCg* h, cudaStream_t s) {
    using namespace clsp;
    switch (h->lanes) {
        case 2: product_kernel<2><<<h->grid, kThreads, 0, s>>>(h->w); break;
        case 4: product_kernel<4><<<h->grid, kThreads, 0, s>>>(h->w); break;
        case 8: product_kernel<8><<<h->grid, kThreads, 0, s>>>(h->w); break;
        case 16: product_kernel<16><<<h->grid, kThreads, 0, s>>>(h->w); break;
        default: product_kernel<32><<<h->grid, kThreads, 0, s>>>(h->w); break;
    }
    return launch_status();
}

}  // namespace

extern "C" {

clsparseStatus clsparseB200DistCgCreate(clsparseB200DistCg* handle, const clsparseCsrMatrix* A, cl_uint extLength,
                                        cl_uint ownOffset, cl_int precond, clsparseControl control) {
    clsp::TraceRange trace_("clsparseB200DistCgCreate");
    using namespace clsp;
    if (handle == nullptr) return clsparseInvalidValue;
    *handle = nullptr;
    if (control == nullptr) return clsparseInvalidControlObject;
    if (A == nullptr || A->row_pointer == nullptr || (A->num_nonzeros > 0 && (A->col_indices == nullptr || A->values == nullptr)))
        return clsparseInvalidMemObject;
    const uint32_t n = A->num_rows;
    if (static_cast<uint64_t>(ownOffset) + n > extLength) return clsparseInvalidSize;
    DeviceGuard g(control->device);
    auto* h = new (std::nothrow) _clsparseB200DistCg();
    if (h == nullptr) return clsparseOutOfResources;
    h->device = control->device;
    h->next_ext = extLength;
    h->nnz = A->num_nonzeros;
    Work& w = h->w;
    w.rp = static_cast<const uint32_t*>(A->row_pointer) + A->off_row_pointer;
    w.cols = static_cast<const uint32_t*>(A->col_indices) + A->off_col_indices;
    w.vals = static_cast<const double*>(A->values) + A->off_values;
    w.n = n;
    w.own = ownOffset;
    const double avg = n ? static_cast<double>(A->num_nonzeros) / n : 0.0;
    h->lanes = avg <= 2.0 ? 2 : avg <= 4.0 ? 4 : avg <= 8.0 ? 8 : avg <= 16.0 ? 16 : 32;
    // one pass over the rows at full occupancy (8 CTAs of 256 threads per SM)
    const uint32_t by_rows = (n + 1023) / 1024;
    h->grid = std::max<uint32_t>(1, std::min<uint32_t>(by_rows, 8u * control->sm_count));
    const size_t nv = n, ne = extLength, G = h->grid;
    const size_t doubles = 5 * nv + 2 * ne + kSlots * G + 4 + kStateLen;
    if (h->buf.ensure(doubles * sizeof(double) + 16) != cudaSuccess) {
        delete h;
        return clsparseOutOfResources;
    }
    double* d = static_cast<double*>(h->buf.ptr);
    w.r = d;
    w.p = d + nv;
    w.s = d + 2 * nv;
    w.w = d + 3 * nv;
    double* invd = d + 4 * nv;
    w.xext = d + 5 * nv;
    w.zext = w.xext + ne;
    w.partials = w.zext + ne;
    w.red = w.partials + kSlots * G;
    w.state = w.red + 4;
    w.ticket = reinterpret_cast<uint32_t*>(w.state + kStateLen);
    h->d_flag = reinterpret_cast<int*>(w.ticket + 1);
    cudaStream_t s = control->stream;
    cudaMemsetAsync(h->buf.ptr, 0, doubles * sizeof(double) + 16, s);
    // columns must index the extended vector; the diagonal must be present
    if (A->num_nonzeros > 0)
        bad_columns_kernel<<<std::max<uint32_t>(1, std::min<uint32_t>((A->num_nonzeros + 255) / 256, 4u * control->sm_count)), 256, 0, s>>>(
            w.cols, A->num_nonzeros, extLength, h->d_flag);
    int bad = 0;
    if (cudaMemcpyAsync(&bad, h->d_flag, sizeof(int), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess) {
        delete h;
        return clsparseInvalidKernelExecution;
    }
    if (bad) {
        delete h;
        return clsparseInvalidValue;
    }
    if (precond == DIAGONAL && n > 0) {
        inv_diag_kernel<<<h->grid, kThreads, 0, s>>>(w, invd, h->d_flag);
        if (cudaMemcpyAsync(&bad, h->d_flag, sizeof(int), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
            cudaStreamSynchronize(s) != cudaSuccess) {
            delete h;
            return clsparseInvalidKernelExecution;
        }
        if (bad) {
            delete h;
            return clsparseInvalidValue;
        }
        w.invd = invd;
    } else {
        w.invd = nullptr;
    }
    *handle = h;
    return clsparseSuccess;
}

clsparseStatus clsparseB200DistCgRelease(clsparseB200DistCg h) {
    if (h == nullptr) return clsparseInvalidValue;
    {
        clsp::DeviceGuard g(h->device);
        h->buf.release();
    }
    delete h;
    return clsparseSuccess;
}

clsparseStatus clsparseB200DistCgBuffers(clsparseB200DistCg h, cl_double** xExt, cl_double** zExt, cl_double** sums) {
    if (h == nullptr) return clsparseInvalidValue;
    if (xExt) *xExt = h->w.xext;
    if (zExt) *zExt = h->w.zext;
    if (sums) *sums = h->w.red;
    return clsparseSuccess;
}

clsparseStatus clsparseB200DistCgStart(clsparseB200DistCg h, cldenseVector* x, const cldenseVector* b,
                                       clsparseControl control) {
    clsp::TraceRange trace_("clsparseB200DistCgStart");
    using namespace clsp;
    if (h == nullptr) return clsparseInvalidValue;
    if (control == nullptr) return clsparseInvalidControlObject;
    if (x == nullptr || b == nullptr || x->values == nullptr || b->values == nullptr) return clsparseInvalidMemObject;
    if (x->num_values != h->w.n || b->num_values != h->w.n) return clsparseInvalidSize;
    DeviceGuard g(control->device);
    h->w.x = static_cast<double*>(x->values) + x->off_values;
    h->w.b = static_cast<const double*>(b->values) + b->off_values;
    cudaStream_t s = control->stream;
    // a fresh solve: clear the state and the sums
    cudaMemsetAsync(h->w.red, 0, (4 + kStateLen) * sizeof(double), s);
    if (h->w.n > 0) load_own_kernel<<<h->grid, kThreads, 0, s>>>(h->w);
    return launch_status();
}

clsparseStatus clsparseB200DistCgResidual(clsparseB200DistCg h, clsparseControl control) {
    clsp::TraceRange trace_("clsparseB200DistCgResidual");
    if (h == nullptr) return clsparseInvalidValue;
    if (control == nullptr) return clsparseInvalidControlObject;
    if (h->w.x == nullptr) return clsparseInvalidValue;
    clsp::DeviceGuard g(control->device);
    return launch_residual(h, control->stream);
}

clsparseStatus clsparseB200DistCgProduct(clsparseB200DistCg h, clsparseControl control) {
    clsp::TraceRange trace_("clsparseB200DistCgProduct");
    if (h == nullptr) return clsparseInvalidValue;
    if (control == nullptr) return clsparseInvalidControlObject;
    if (h->w.x == nullptr) return clsparseInvalidValue;
    clsp::DeviceGuard g(control->device);
    return launch_product(h, control->stream);
}

clsparseStatus clsparseB200DistCgUpdate(clsparseB200DistCg h, cl_int step, clSParseSolverControl solverControl,
                                        clsparseControl control) {
    clsp::TraceRange trace_("clsparseB200DistCgUpdate");
    using namespace clsp;
    if (h == nullptr || step < 0) return clsparseInvalidValue;
    if (control == nullptr) return clsparseInvalidControlObject;
    if (solverControl == nullptr) return clsparseInvalidSolverControlObject;
    if (h->w.x == nullptr) return clsparseInvalidValue;
    DeviceGuard g(control->device);
    update_kernel<<<h->grid, kThreads, 0, control->stream>>>(h->w, step, solverControl->relativeTolerance,
                                                              solverControl->absoluteTolerance,
                                                              solverControl->maxIters);
    return launch_status();
}

clsparseStatus clsparseB200DistCgState(clsparseB200DistCg h, cl_int* done, clSParseSolverControl solverControl,
                                       clsparseControl control) {
    clsp::TraceRange trace_("clsparseB200DistCgState");
    using namespace clsp;
    if (h == nullptr) return clsparseInvalidValue;
    if (control == nullptr) return clsparseInvalidControlObject;
    DeviceGuard g(control->device);
    double st[kStateLen];
    if (cudaMemcpyAsync(st, h->w.state, sizeof(st), cudaMemcpyDeviceToHost, control->stream) != cudaSuccess ||
        cudaStreamSynchronize(control->stream) != cudaSuccess)
        return clsparseInvalidKernelExecution;
    if (done) *done = st[kDone] != 0.0 ? 1 : 0;
    if (solverControl) {
        solverControl->nIters = static_cast<cl_int>(st[kIters]);
        solverControl->initialResidual = st[kInit];
        solverControl->currentResidual = st[kCur];
    }
    return clsparseSuccess;
}

clsparseStatus clsparseB200DistCgGather(cl_double* dst, const cl_double* src, const cl_uint* idx, cl_uint count,
                                        clsparseControl control) {
    using namespace clsp;
    if (control == nullptr) return clsparseInvalidControlObject;
    if (count == 0) return clsparseSuccess;
    if (dst == nullptr || src == nullptr || idx == nullptr) return clsparseInvalidMemObject;
    DeviceGuard g(control->device);
    const uint32_t blocks = std::max<uint32_t>(1, std::min<uint32_t>((count + 255) / 256, 4u * control->sm_count));
    gather_kernel<<<blocks, 256, 0, control->stream>>>(dst, src, idx, count);
    return launch_status();
}

}  // extern "C"
