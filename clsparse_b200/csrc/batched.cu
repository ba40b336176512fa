// Batched Jacobi-CG over many independent SPD systems in one persistent
// launch (clsparseScsrcgBatched), a project extension with no reference
// counterpart.
//
// The systems are stacked block-diagonally in one CSR matrix (rows and columns
// of system s are [off[s], off[s+1])). A persistent kernel keeps one CTA per
// resident slot; each CTA takes the next system from a device work queue
// (atomic counter over the systems ordered by decreasing nonzeros, so the
// largest start first) and runs CG on it to completion: FP32 vectors and FP32
// matrix values, CTA-wide reductions, no grid synchronisation and no host
// round trip. When the recursive FP32 residual meets the tolerance, the CTA
// recomputes the true residual b - A x in FP64; if that check fails, CG
// restarts from the current x with the FP64 residual (refinement) until the
// check passes or the iteration budget is spent. When every system is banded
// (at most kBatchDiags column offsets, all inside its own rows), the products
// come from a per-system diagonal-storage copy laid out at every call: one
// thread per row, the values and the vector entries independent loads
// instead of the row-pointer / column-index / vector chain of CSR, and rows
// whose whole stencil lies inside the system without clamps (C4, 4096 stencil
// systems: 0.349 -> 0.312 -> 0.229 s; the update pass issuing each row's
// loads before its stores: 0.198 s; the vector passes two rows at a time:
// 0.169 s; the product pass too: 0.165 s). Otherwise each system's SpMV uses the
// lanes-per-row width the tuning table gives for its size class. The kernel
// is held to two CTAs per SM (64 registers): the diagonal loop would
// otherwise take 128 registers and halve the resident CTAs (0.51 s).
//
// The whole solve (queue reset, kernel) is captured once into a CUDA graph per
// control and relaunched for repeated solves on the same operands.
#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <numeric>
#include <vector>

#include "device_common.cuh"
#include "internal.h"

namespace clsp {
namespace {

constexpr int kThreads = 512;
constexpr int kWarps = kThreads / 32;

// Diagonals a system may have to be solved from diagonal storage.
constexpr int kBatchDiags = 8;

struct BatchArgs {
    const float* vals;
    const uint32_t* cols;
    const uint32_t* rp;
    float* x;
    const float* b;
    float* r;
    float* p;
    float* q;
    float* invd;
    const uint32_t* off;      // num_systems + 1 row offsets
    const uint32_t* order;    // processing order of the systems
    const uint8_t* lanes;     // lanes per row for each system (1, 2, 4, 8, 16, 32)
    uint32_t* counter;        // work queue head
    int* iters;               // per system: CG iterations
    double* residual;         // per system: FP64 ||b - A x||_2 / ||b||_2 on exit
    int* converged;           // per system: 1 if residual <= tol
    uint32_t nsys;
    int max_iters;
    double tol;
    // Diagonal storage (nullptr: every system's products come from CSR):
    // system s's diagonal d at row r0 + i is dvals[dbase[s] + d * n_s + i],
    // its column offsets doffs[s * kBatchDiags + d] increasing, dnd[s] of them.
    const float* dvals;
    const uint64_t* dbase;
    const int32_t* doffs;
    const uint8_t* dnd;
};

__device__ __forceinline__ double cta_sum(double v, double* red) {
    return dev::block_sum(v, red);
}

// q = A v over the rows of one system, G lanes per row.
template <int G>
__device__ __forceinline__ void sys_spmv(const BatchArgs& a, uint32_t r0, uint32_t r1, const float* v,
                                         float* out) {
    const uint32_t grp = threadIdx.x / G, ln = threadIdx.x & (G - 1);
    const uint32_t groups = kThreads / G;
    for (uint32_t base = r0; base < r1; base += groups) {
        const uint32_t row = base + grp;
        float s = 0.f;
        if (row < r1) {
            const uint32_t nb = a.rp[row], ne = a.rp[row + 1];
            for (uint32_t j = nb + ln; j < ne; j += G) s = fmaf(a.vals[j], v[a.cols[j]], s);
        }
#pragma unroll
        for (int o = G / 2; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o, G);
        if (row < r1 && ln == 0) out[row] = s;
    }
}

__device__ __forceinline__ void spmv_dispatch(const BatchArgs& a, int g, uint32_t r0, uint32_t r1,
                                              const float* v, float* out) {
    switch (g) {
        case 1: sys_spmv<1>(a, r0, r1, v, out); break;
        case 2: sys_spmv<2>(a, r0, r1, v, out); break;
        case 4: sys_spmv<4>(a, r0, r1, v, out); break;
        case 8: sys_spmv<8>(a, r0, r1, v, out); break;
        case 16: sys_spmv<16>(a, r0, r1, v, out); break;
        default: sys_spmv<32>(a, r0, r1, v, out); break;
    }
}

// q = A v over the rows of one system from its diagonal storage: one thread
// per row, products in increasing column order, columns outside the system
// (the block diagonal) contribute nothing. The values and the v entries of
// a row are independent loads (no row-pointer / column-index chain).
__device__ __forceinline__ double sys_spmv_dia(const float* __restrict__ dv, uint32_t ns, uint32_t r0, uint32_t r1,
                                               const int32_t* soff, int nd, const float* v, float* out) {
    double dot = 0.0;
    const int32_t lo = nd > 0 ? soff[0] : 0, hi = nd > 0 ? soff[nd - 1] : 0;
    auto row_sum = [&](uint32_t row) {
        const uint32_t i = row - r0;
        float s = 0.f;
        if (static_cast<int64_t>(row) + lo >= r0 && static_cast<int64_t>(row) + hi < r1) {
            // every column of the row inside the system: no clamps
#pragma unroll
            for (int d = 0; d < kBatchDiags; ++d)
                if (d < nd)
                    s = fmaf(__ldg(dv + static_cast<size_t>(d) * ns + i), v[row + static_cast<uint32_t>(soff[d])], s);
        } else {
#pragma unroll
            for (int d = 0; d < kBatchDiags; ++d) {
                if (d < nd) {
                    const int64_t j = static_cast<int64_t>(row) + soff[d];
                    const bool in = j >= r0 && j < r1;
                    const float av = __ldg(dv + static_cast<size_t>(d) * ns + i);
                    const float xv = v[in ? static_cast<uint32_t>(j) : row];
                    s = fmaf(av, in ? xv : 0.f, s);
                }
            }
        }
        return s;
    };
    // two rows per pass, both rows' loads before the stores (see the update pass)
    for (uint32_t row = r0 + threadIdx.x; row < r1; row += 2 * kThreads) {
        const uint32_t row1 = row + kThreads;
        const bool has1 = row1 < r1;
        const uint32_t rb = has1 ? row1 : row;
        const float s0 = row_sum(row);
        const float s1 = row_sum(rb);
        const float v0 = v[row], v1 = v[rb];
        out[row] = s0;
        dot += static_cast<double>(v0) * s0;
        if (has1) {
            out[row1] = s1;
            dot += static_cast<double>(v1) * s1;
        }
    }
    return dot;  // this thread's part of <v, A v>
}

// r = b - A x in FP64 (the check), written back to r in FP32; returns
// sum r^2 and sum b^2 in every thread.
__device__ __forceinline__ void true_residual(const BatchArgs& a, uint32_t r0, uint32_t r1, double* red,
                                              double& rr, double& bb) {
    double acc_r = 0.0, acc_b = 0.0;
    for (uint32_t row = r0 + threadIdx.x; row < r1; row += kThreads) {
        double s = 0.0;
        for (uint32_t j = a.rp[row]; j < a.rp[row + 1]; ++j)
            s = fma(static_cast<double>(a.vals[j]), static_cast<double>(a.x[a.cols[j]]), s);
        const double bi = a.b[row];
        const double ri = bi - s;
        a.r[row] = static_cast<float>(ri);
        acc_r += ri * ri;
        acc_b += bi * bi;
    }
    rr = cta_sum(acc_r, red);
    bb = cta_sum(acc_b, red);
}

__global__ void __launch_bounds__(kThreads, 2) batched_cg_kernel(BatchArgs a) {
    __shared__ double red[32];
    __shared__ uint32_t slot;
    __shared__ int32_t soff[kBatchDiags];
    for (;;) {
        if (threadIdx.x == 0) slot = atomicAdd(a.counter, 1u);
        __syncthreads();
        const uint32_t k = slot;
        __syncthreads();
        if (k >= a.nsys) break;
        const uint32_t s = a.order[k];
        const uint32_t r0 = a.off[s], r1 = a.off[s + 1];
        const int g = a.lanes[s];
        const float* dv = a.dvals ? a.dvals + a.dbase[s] : nullptr;
        const int nd = a.dvals ? a.dnd[s] : 0;
        if (a.dvals && threadIdx.x < kBatchDiags) soff[threadIdx.x] = a.doffs[s * kBatchDiags + threadIdx.x];

        // Jacobi: inverse diagonal (first diagonal entry of each row; 1 if absent)
        for (uint32_t row = r0 + threadIdx.x; row < r1; row += kThreads) {
            float d = 0.f;
            for (uint32_t j = a.rp[row]; j < a.rp[row + 1]; ++j)
                if (a.cols[j] == row) {
                    d = a.vals[j];
                    break;
                }
            a.invd[row] = d != 0.f ? 1.f / d : 1.f;
        }
        __syncthreads();

        double rr, bb;
        true_residual(a, r0, r1, red, rr, bb);
        const double bnorm = sqrt(bb);
        int it = 0;
        bool ok = bnorm == 0.0 || sqrt(rr) <= a.tol * bnorm;
        double res64 = bnorm == 0.0 ? 0.0 : sqrt(rr) / bnorm;
        while (!ok && it < a.max_iters) {
            // (re)start: z = M r, p = z, rz = <r, z>
            double acc = 0.0;
            for (uint32_t row = r0 + threadIdx.x; row < r1; row += kThreads) {
                const float z = a.r[row] * a.invd[row];
                a.p[row] = z;
                acc += static_cast<double>(a.r[row]) * z;
            }
            double rz = cta_sum(acc, red);
            __syncthreads();
            bool inner_done = false;
            while (!inner_done && it < a.max_iters) {
                if (dv) {
                    // the row's thread also forms its part of <p, q>
                    acc = sys_spmv_dia(dv, r1 - r0, r0, r1, soff, nd, a.p, a.q);
                } else {
                    spmv_dispatch(a, g, r0, r1, a.p, a.q);
                    __syncthreads();
                    acc = 0.0;
                    for (uint32_t row = r0 + threadIdx.x; row < r1; row += kThreads)
                        acc += static_cast<double>(a.p[row]) * a.q[row];
                }
                const double pq = cta_sum(acc, red);  // its barriers also order q's stores
                const float alpha = static_cast<float>(rz / pq);
                double acc_rz = 0.0, acc_rr = 0.0;
                // two rows per pass, all their loads before any store (the
                // vectors are not __restrict__: a store holds back every later
                // load, so one row per pass would wait out each row's loads)
                for (uint32_t row = r0 + threadIdx.x; row < r1; row += 2 * kThreads) {
                    const uint32_t row1 = row + kThreads;
                    const bool has1 = row1 < r1;
                    const uint32_t rb = has1 ? row1 : row;
                    const float xi = fmaf(alpha, a.p[row], a.x[row]);
                    const float ri = fmaf(-alpha, a.q[row], a.r[row]);
                    const float z = ri * a.invd[row];
                    const float xj = fmaf(alpha, a.p[rb], a.x[rb]);
                    const float rj = fmaf(-alpha, a.q[rb], a.r[rb]);
                    const float zj = rj * a.invd[rb];
                    a.x[row] = xi;
                    a.r[row] = ri;
                    acc_rz += static_cast<double>(ri) * z;
                    acc_rr += static_cast<double>(ri) * ri;
                    if (has1) {
                        a.x[row1] = xj;
                        a.r[row1] = rj;
                        acc_rz += static_cast<double>(rj) * zj;
                        acc_rr += static_cast<double>(rj) * rj;
                    }
                }
                const double rz_new = cta_sum(acc_rz, red);
                const double rr_new = cta_sum(acc_rr, red);
                ++it;
                if (!(pq > 0.0) || !isfinite(rz_new)) {
                    inner_done = true;  // breakdown: fall through to the FP64 check
                    break;
                }
                if (sqrt(rr_new) <= a.tol * bnorm) {
                    inner_done = true;
                    break;
                }
                const float beta = static_cast<float>(rz_new / rz);
                rz = rz_new;
                for (uint32_t row = r0 + threadIdx.x; row < r1; row += 2 * kThreads) {
                    const uint32_t row1 = row + kThreads;
                    const bool has1 = row1 < r1;
                    const uint32_t rb = has1 ? row1 : row;
                    const float pi = fmaf(beta, a.p[row], a.r[row] * a.invd[row]);
                    const float pj = fmaf(beta, a.p[rb], a.r[rb] * a.invd[rb]);
                    a.p[row] = pi;
                    if (has1) a.p[row1] = pj;
                }
                __syncthreads();
            }
            __syncthreads();
            true_residual(a, r0, r1, red, rr, bb);
            res64 = sqrt(rr) / bnorm;
            ok = res64 <= a.tol;
            if (!isfinite(res64)) break;
        }
        if (threadIdx.x == 0) {
            a.iters[s] = it;
            a.residual[s] = res64;
            a.converged[s] = ok ? 1 : 0;
        }
        __syncthreads();
    }
}

// One CTA per system: the distinct column offsets col - row of its rows,
// increasing, into doffs[s * kBatchDiags ...] and their count into dnd[s]
// (0 when the system does not qualify); bad[0] = 1 when a system has more
// than kBatchDiags of them, a column outside its own rows, or columns not
// strictly increasing in a row.
__global__ void batch_dia_detect_kernel(const uint32_t* __restrict__ rp, const uint32_t* __restrict__ cols,
                                        const uint32_t* __restrict__ off, int32_t* doffs, uint8_t* dnd, int* bad) {
    constexpr int32_t kEmptySlot = INT32_MIN;  // below any offset of a system of fewer than 2^31 rows
    __shared__ int32_t set[kBatchDiags];
    __shared__ int over;
    const uint32_t s = blockIdx.x;
    const uint32_t r0 = off[s], r1 = off[s + 1];
    if (threadIdx.x < kBatchDiags) set[threadIdx.x] = kEmptySlot;
    if (threadIdx.x == 0) over = 0;
    __syncthreads();
    int mine = 0;
    for (uint32_t row = r0 + threadIdx.x; row < r1; row += blockDim.x) {
        for (uint32_t k = rp[row]; k < rp[row + 1]; ++k) {
            const uint32_t c = cols[k];
            if (c < r0 || c >= r1 || (k > rp[row] && c <= cols[k - 1])) {
                mine = 1;
                continue;
            }
            const int32_t o = static_cast<int32_t>(static_cast<int64_t>(c) - static_cast<int64_t>(row));
            bool placed = false;
            for (int t = 0; t < kBatchDiags && !placed; ++t) {
                const int32_t cur = *reinterpret_cast<volatile int32_t*>(&set[t]);
                if (cur == o) {
                    placed = true;
                } else if (cur == kEmptySlot) {
                    const int32_t old = atomicCAS(&set[t], kEmptySlot, o);
                    placed = old == kEmptySlot || old == o;
                }
            }
            if (!placed) mine = 1;
        }
    }
    if (mine) atomicExch(&over, 1);
    __syncthreads();
    if (threadIdx.x == 0) {
        int32_t v[kBatchDiags];
        int nd = 0;
        for (int t = 0; t < kBatchDiags; ++t)
            if (set[t] != kEmptySlot) v[nd++] = set[t];
        if (over) nd = 0;
        for (int t = 1; t < nd; ++t)  // insertion sort of at most kBatchDiags values
            for (int u = t; u > 0 && v[u - 1] > v[u]; --u) {
                const int32_t w = v[u];
                v[u] = v[u - 1];
                v[u - 1] = w;
            }
        for (int t = 0; t < kBatchDiags; ++t) doffs[s * kBatchDiags + t] = t < nd ? v[t] : 0;
        dnd[s] = static_cast<uint8_t>(nd);
        if (over) atomicExch(bad, 1);
    }
}

// One CTA per system: its CSR values into diagonal storage (dv zeroed before).
__global__ void batch_dia_fill_kernel(const uint32_t* __restrict__ rp, const uint32_t* __restrict__ cols,
                                      const float* __restrict__ vals, const uint32_t* __restrict__ off,
                                      const int32_t* __restrict__ doffs, const uint8_t* __restrict__ dnd,
                                      const uint64_t* __restrict__ dbase, float* dv) {
    const uint32_t s = blockIdx.x;
    const uint32_t r0 = off[s], r1 = off[s + 1], ns = r1 - r0;
    const int nd = dnd[s];
    const int32_t* o = doffs + s * kBatchDiags;
    float* out = dv + dbase[s];
    for (uint32_t row = r0 + threadIdx.x; row < r1; row += blockDim.x) {
        int d = 0;
        for (uint32_t k = rp[row]; k < rp[row + 1]; ++k) {
            const int32_t c = static_cast<int32_t>(static_cast<int64_t>(cols[k]) - static_cast<int64_t>(row));
            while (d < nd && o[d] < c) ++d;  // columns increase, so d only moves forward
            if (d < nd && o[d] == c) out[static_cast<size_t>(d) * ns + (row - r0)] = vals[k];
        }
    }
}

__global__ void gather_bounds_kernel(const uint32_t* rp, const uint32_t* off, uint32_t nsys, uint32_t* bnd) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i <= nsys) bnd[i] = rp[off[i]];
}

int default_lanes(uint32_t n, uint32_t nnz) {
    const uint32_t per = n ? nnz / n : 0;
    if (per >= 24) return 8;
    if (per >= 12) return 4;
    return 2;
}

}  // namespace
}  // namespace clsp

using namespace clsp;

extern "C" {

clsparseStatus clsparseScsrcgBatched(cldenseVector* x, const clsparseCsrMatrix* A, const cldenseVector* b,
                                     const clsparseIdx_t* systemOffsets, cl_int numSystems,
                                     const cl_int* lanesPerRow, clSParseSolverControl solverControl,
                                     clsparseB200BatchResult* result, clsparseControl control) {
    clsp::TraceRange trace_("clsparseScsrcgBatched");
    clsparseStatus st = check_entry(control);
    if (st != clsparseSuccess) return st;
    if (solverControl == nullptr) return clsparseInvalidSolverControlObject;
    if (!x || !A || !b || !systemOffsets || numSystems < 0) return clsparseInvalidValue;
    if (A->num_rows != A->num_cols || x->num_values != A->num_rows || b->num_values != A->num_rows)
        return clsparseInvalidSystemSize;
    const uint32_t nsys = static_cast<uint32_t>(numSystems);
    if (nsys == 0) return clsparseSuccess;
    if (systemOffsets[0] != 0 || systemOffsets[nsys] != A->num_rows) return clsparseInvalidSystemSize;
    for (uint32_t s = 0; s < nsys; ++s)
        if (systemOffsets[s + 1] < systemOffsets[s]) return clsparseInvalidSystemSize;
    DeviceGuard g(control->device);
    const size_t n = A->num_rows;
    if (!control->batch_work) control->batch_work = std::make_unique<BatchWork>();
    BatchWork& w = *control->batch_work;
    cudaStream_t s = control->stream;

    const size_t vb = ((n * 4 + 255) / 256) * 256;
    const size_t meta_bytes = 16 + (nsys + 1) * 4 * 2 + nsys * 4 + nsys + 256;
    const size_t out_bytes = nsys * (4 + 8 + 4) + 64;
    if (w.vecs.ensure(4 * vb + 256) != cudaSuccess || w.meta.ensure(meta_bytes) != cudaSuccess ||
        w.out.ensure(out_bytes) != cudaSuccess) {
        cudaGetLastError();
        return clsparseOutOfResources;
    }
    char* mb = static_cast<char*>(w.meta.ptr);
    uint32_t* d_counter = reinterpret_cast<uint32_t*>(mb);
    uint32_t* d_off = reinterpret_cast<uint32_t*>(mb + 16);
    uint32_t* d_bnd = d_off + (nsys + 1);
    uint32_t* d_order = d_bnd + (nsys + 1);
    uint8_t* d_lanes = reinterpret_cast<uint8_t*>(d_order + nsys);
    const uint32_t* rp = dev_ptr<const uint32_t>(A->row_pointer, A->off_row_pointer);

    // nonzeros per system from the row pointers at the system boundaries
    std::vector<uint32_t> off(systemOffsets, systemOffsets + nsys + 1), bnd(nsys + 1);
    cudaMemcpyAsync(d_off, off.data(), (nsys + 1) * 4, cudaMemcpyHostToDevice, s);
    gather_bounds_kernel<<<(nsys + 256) / 256, 256, 0, s>>>(rp, d_off, nsys, d_bnd);
    cudaMemcpyAsync(bnd.data(), d_bnd, (nsys + 1) * 4, cudaMemcpyDeviceToHost, s);
    if (cudaStreamSynchronize(s) != cudaSuccess) return clsparseInvalidMemObject;

    std::vector<uint32_t> order(nsys);
    std::iota(order.begin(), order.end(), 0u);
    std::stable_sort(order.begin(), order.end(), [&](uint32_t p, uint32_t q) {
        return bnd[p + 1] - bnd[p] > bnd[q + 1] - bnd[q];
    });
    std::vector<uint8_t> lanes(nsys);
    for (uint32_t k = 0; k < nsys; ++k) {
        const uint32_t ns = off[k + 1] - off[k];
        const int l = lanesPerRow ? lanesPerRow[k] : default_lanes(ns, bnd[k + 1] - bnd[k]);
        if (l != 1 && l != 2 && l != 4 && l != 8 && l != 16 && l != 32) return clsparseInvalidValue;
        lanes[k] = static_cast<uint8_t>(l);
    }
    cudaMemcpyAsync(d_order, order.data(), nsys * 4, cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(d_lanes, lanes.data(), nsys, cudaMemcpyHostToDevice, s);

    // Diagonal storage when every system is banded (at most kBatchDiags
    // column offsets inside its own rows): offsets found on the device, the
    // values laid out by diagonal at every call (so values changed in place
    // are seen). CLSPARSE_B200_BATCH_DIA=0 keeps every system on CSR.
    const float* dvals = nullptr;
    const uint64_t* d_dbase = nullptr;
    const int32_t* d_doffs = nullptr;
    const uint8_t* d_dnd = nullptr;
    const char* dia_env = std::getenv("CLSPARSE_B200_BATCH_DIA");
    if (!(dia_env && std::atoi(dia_env) == 0)) {
        const size_t offs_b = ((static_cast<size_t>(nsys) * kBatchDiags * 4 + 255) / 256) * 256;
        const size_t base_b = ((static_cast<size_t>(nsys) * 8 + 255) / 256) * 256;
        const size_t nd_b = ((static_cast<size_t>(nsys) + 255) / 256) * 256;
        if (w.dia_meta.ensure(offs_b + base_b + nd_b + 256) != cudaSuccess) {
            cudaGetLastError();
            return clsparseOutOfResources;
        }
        char* dm = static_cast<char*>(w.dia_meta.ptr);
        int32_t* doffs = reinterpret_cast<int32_t*>(dm);
        uint64_t* dbase = reinterpret_cast<uint64_t*>(dm + offs_b);
        uint8_t* dnd = reinterpret_cast<uint8_t*>(dm + offs_b + base_b);
        int* bad = reinterpret_cast<int*>(dm + offs_b + base_b + nd_b);
        const uint32_t* cols = dev_ptr<const uint32_t>(A->col_indices, A->off_col_indices);
        cudaMemsetAsync(bad, 0, sizeof(int), s);
        batch_dia_detect_kernel<<<nsys, 256, 0, s>>>(rp, cols, d_off, doffs, dnd, bad);
        std::vector<uint8_t> hnd(nsys);
        int hbad = 1;
        cudaMemcpyAsync(hnd.data(), dnd, nsys, cudaMemcpyDeviceToHost, s);
        cudaMemcpyAsync(&hbad, bad, sizeof(int), cudaMemcpyDeviceToHost, s);
        if (cudaStreamSynchronize(s) != cudaSuccess) return clsparseInvalidKernelExecution;
        if (hbad == 0) {
            std::vector<uint64_t> hbase(nsys);
            uint64_t total = 0;
            for (uint32_t k = 0; k < nsys; ++k) {
                hbase[k] = total;
                total += static_cast<uint64_t>(hnd[k]) * (off[k + 1] - off[k]);
            }
            if (w.dia.ensure(total * sizeof(float) + 256) != cudaSuccess) {
                cudaGetLastError();
                return clsparseOutOfResources;
            }
            cudaMemcpyAsync(dbase, hbase.data(), nsys * 8, cudaMemcpyHostToDevice, s);
            cudaMemsetAsync(w.dia.ptr, 0, total * sizeof(float), s);
            batch_dia_fill_kernel<<<nsys, 256, 0, s>>>(rp, cols, dev_ptr<const float>(A->values, A->off_values), d_off,
                                                      doffs, dnd, dbase, static_cast<float*>(w.dia.ptr));
            if (cudaGetLastError() != cudaSuccess) return clsparseInvalidKernelExecution;
            dvals = static_cast<const float*>(w.dia.ptr);
            d_dbase = dbase;
            d_doffs = doffs;
            d_dnd = dnd;
        }
    }

    char* ob = static_cast<char*>(w.out.ptr);
    static_assert(sizeof(BatchArgs) <= sizeof(w.args), "argument record");
    BatchArgs a;
    std::memset(&a, 0, sizeof(a));
    a.vals = dev_ptr<const float>(A->values, A->off_values);
    a.cols = dev_ptr<const uint32_t>(A->col_indices, A->off_col_indices);
    a.rp = rp;
    a.x = dev_ptr<float>(x->values, x->off_values);
    a.b = dev_ptr<const float>(b->values, b->off_values);
    char* vbase = static_cast<char*>(w.vecs.ptr);
    a.r = reinterpret_cast<float*>(vbase);
    a.p = reinterpret_cast<float*>(vbase + vb);
    a.q = reinterpret_cast<float*>(vbase + 2 * vb);
    a.invd = reinterpret_cast<float*>(vbase + 3 * vb);
    a.off = d_off;
    a.order = d_order;
    a.lanes = d_lanes;
    a.counter = d_counter;
    a.residual = reinterpret_cast<double*>(ob);
    a.iters = reinterpret_cast<int*>(ob + nsys * 8);
    a.converged = reinterpret_cast<int*>(ob + nsys * 12);
    a.nsys = nsys;
    a.max_iters = solverControl->maxIters;
    a.tol = solverControl->relativeTolerance;
    a.dvals = dvals;
    a.dbase = d_dbase;
    a.doffs = d_doffs;
    a.dnd = d_dnd;

    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, batched_cg_kernel, kThreads, 0);
    uint32_t grid = static_cast<uint32_t>(control->sm_count * std::max(per_sm, 1));
    grid = std::min(grid, nsys);

    // One graph per operand set: reset the queue, run the persistent kernel.
    const bool same = w.exec && w.grid == grid && std::memcmp(&w.args, &a, sizeof(a)) == 0;
    if (!same) {
        if (w.exec) cudaGraphExecDestroy(w.exec);
        w.exec = nullptr;
        cudaStream_t cs = control->capture_stream;
        cudaGraph_t graph = nullptr;
        if (cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal) != cudaSuccess)
            return clsparseInvalidKernelExecution;
        cudaMemsetAsync(d_counter, 0, 16, cs);
        batched_cg_kernel<<<grid, kThreads, 0, cs>>>(a);
        if (cudaStreamEndCapture(cs, &graph) != cudaSuccess) {
            cudaGetLastError();
            return clsparseInvalidKernelExecution;
        }
        const cudaError_t ie = cudaGraphInstantiate(&w.exec, graph, 0);
        cudaGraphDestroy(graph);
        if (ie != cudaSuccess) {
            w.exec = nullptr;
            cudaGetLastError();
            return clsparseInvalidKernelExecution;
        }
        std::memcpy(&w.args, &a, sizeof(a));
        w.grid = grid;
    }
    if (cudaGraphLaunch(w.exec, s) != cudaSuccess) return clsparseInvalidKernelExecution;

    std::vector<double> res(nsys);
    std::vector<int> its(nsys), conv(nsys);
    cudaMemcpyAsync(res.data(), a.residual, nsys * 8, cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(its.data(), a.iters, nsys * 4, cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(conv.data(), a.converged, nsys * 4, cudaMemcpyDeviceToHost, s);
    if (cudaStreamSynchronize(s) != cudaSuccess) return clsparseInvalidKernelExecution;
    if (control->event) cudaEventRecord(control->event, s);
    int nconv = 0, maxit = 0;
    double worst = 0.0;
    for (uint32_t k = 0; k < nsys; ++k) {
        nconv += conv[k];
        maxit = std::max(maxit, its[k]);
        worst = std::max(worst, res[k]);
        if (result && result->iterations) result->iterations[k] = its[k];
        if (result && result->residuals) result->residuals[k] = res[k];
    }
    if (result) {
        result->systemsConverged = nconv;
        result->maxIterations = maxit;
        result->worstResidual = worst;
    }
    solverControl->nIters = maxit;
    solverControl->currentResidual = worst;
    return clsparseSuccess;
}

}  // extern "C"
