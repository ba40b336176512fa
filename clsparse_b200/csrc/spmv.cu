// CSR sparse matrix-vector product y = alpha*A*x + beta*y for sm_100a, and the
// clsparseScsrmv / clsparseDcsrmv entry points.
//
// Two kernels, chosen as the reference chooses (src/library/blas2/clsparse-csrmv.hpp:103-132):
//
// * csr_adaptive_kernel -- with a meta (row-block words from
//   clsparseCsrMetaCreate) one 256-thread CTA runs per word, in one of three
//   modes decided from the word pair (the CSR-Adaptive scheme of the reference's
//   src/library/kernels/csrmv_adaptive.cl:312-687, rebuilt for B200):
//     STREAM  a block of several short rows (<= 1024 nonzeros in total): the CTA
//             streams alpha*val*x[col] for the whole block into shared memory
//             with coalesced evict-first loads, then reduces every row out of
//             shared memory with groups of up to 32 lanes (warp shuffles, no
//             shared-memory tree).
//     VECTOR  one row (up to 3072 nonzeros): the whole CTA reduces it.
//     LONG    one chunk of 3072 nonzeros of a longer row. Each chunk CTA writes
//             its partial sum to the meta's partial slot and takes an arrival
//             ticket; the CTA that arrives last adds the partials in chunk order
//             and writes y. No CTA waits for another (the reference spin-waits on
//             a flag it flips inside the meta, csrmv_adaptive.cl:596-600), the
//             result does not depend on arrival order, and the meta is left as
//             it was found.
// * csr_vector_kernel -- without a meta, G lanes per row (G = 2..32 from the
//   average row length, as csrmv-vector.hpp:34-49 picks its sub-wave).
//
// beta == 0 overwrites y without reading it on every path (the reference reads
// y on its LONG path; csrmv_adaptive.cl:481-483 skips it on the others).
//
// Both kernels can fuse the dot products a Krylov solver takes of the result
// (<y, w> and <y, y>) and finish them with a deterministic grid reduction.
#include <algorithm>
#include <cstdlib>
#include <string>
#include <type_traits>

#include "device_common.cuh"
#include "internal.h"
#include "pipeline.cuh"
#include "solver_state.cuh"

namespace clsp {

namespace {

constexpr int kThreads = 256;
constexpr uint32_t kLongChunk = kBlkSize * kBlockMultiplier;  // 3072 nonzeros per CTA

template <typename T>
struct EpiDev {
    const T* w0;
    int dot1_self;
    double* partials;
    uint32_t* ticket;
    int op;
    void* state;
    unsigned long long cond;
    const int* done;
};

template <typename T, int K>
struct RowSink {
    T* y;
    const T* w0;
    int dot1_self;
    T beta;
    double d[K > 0 ? K : 1];
    __device__ __forceinline__ void init(T* y_, const EpiDev<T>& e, T beta_) {
        y = y_;
        w0 = e.w0;
        dot1_self = e.dot1_self;
        beta = beta_;
#pragma unroll
        for (int k = 0; k < (K > 0 ? K : 1); ++k) d[k] = 0.0;
    }
    // Final value of one row: adds beta*y (reading y only if beta != 0),
    // stores it and feeds the fused dot products.
    template <bool EXT>
    __device__ __forceinline__ void put(uint32_t row, dev::Acc<T, EXT> a) {
        if (beta != T(0)) a.add_prod(beta, y[row]);
        const T v = a.value();
        y[row] = v;
        if constexpr (K >= 1) d[0] += static_cast<double>(v) * static_cast<double>(w0[row]);
        if constexpr (K >= 2) {
            if (dot1_self) d[1] += static_cast<double>(v) * static_cast<double>(v);
        }
    }
};

template <typename T, int K>
__device__ __forceinline__ void run_epilogue(RowSink<T, K>& sink, const EpiDev<T>& e) {
    if constexpr (K > 0) {
        double tot[K];
        if (dev::grid_reduce_last<K>(sink.d, e.partials, e.ticket, tot)) {
            if (threadIdx.x == 0) {
                auto* st = static_cast<SolverState<T>*>(e.state);
                if (e.op == static_cast<int>(EpiOp::CgAlpha)) fin_cg_alpha(st, tot[0]);
                if (e.op == static_cast<int>(EpiOp::BicgAlpha)) fin_bicg_alpha(st, tot[0]);
                if (e.op == static_cast<int>(EpiOp::PcgRz)) fin_pcg_rz(st, tot[0]);
                if (e.op == static_cast<int>(EpiOp::PcgRz0)) fin_pcg_rz0(st, tot[0]);
                if constexpr (K >= 2) {
                    if (e.op == static_cast<int>(EpiOp::BicgOmega)) fin_bicg_omega(st, tot[0], tot[1]);
                }
            }
        }
    }
}

// Four consecutive nonzeros [e0, e0+4) of the CSR arrays; `mask` marks the
// ones inside the block [nb, ne) being processed (the others are not used).
template <typename T>
struct Quad {
    uint32_t c[4];
    T v[4];
    uint32_t mask;
};

// Loads one quad. When the quad lies inside the matrix's nonzero range
// [lo, hi) and the arrays are 16-byte aligned, the column indices come in one
// 16-byte load and the values in one (FP32) or two (FP64) 16-byte loads;
// otherwise element by element. Nothing outside [lo, hi) is ever read.
template <typename V, typename T>
__device__ __forceinline__ void load_quad(const V* __restrict__ vals, const uint32_t* __restrict__ cols,
                                          uint32_t e0, uint32_t nb, uint32_t ne, uint32_t lo,
                                          uint32_t hi, bool vec, Quad<T>& q) {
    q.mask = 0;
#pragma unroll
    for (int k = 0; k < 4; ++k)
        if (e0 + k >= nb && e0 + k < ne) q.mask |= 1u << k;
    if (vec && e0 >= lo && e0 + 4 <= hi) {
        const uint4 ci = dev::ld_stream(reinterpret_cast<const uint4*>(cols + e0));
        q.c[0] = ci.x;
        q.c[1] = ci.y;
        q.c[2] = ci.z;
        q.c[3] = ci.w;
        if constexpr (std::is_same_v<V, __nv_bfloat16>) {
            const uint2 a = dev::ld_stream(reinterpret_cast<const uint2*>(vals + e0));
            q.v[0] = static_cast<T>(__uint_as_float(a.x << 16));
            q.v[1] = static_cast<T>(__uint_as_float(a.x & 0xffff0000u));
            q.v[2] = static_cast<T>(__uint_as_float(a.y << 16));
            q.v[3] = static_cast<T>(__uint_as_float(a.y & 0xffff0000u));
        } else if constexpr (sizeof(V) == 8) {
            const double2 a = dev::ld_stream(reinterpret_cast<const double2*>(vals + e0));
            const double2 b = dev::ld_stream(reinterpret_cast<const double2*>(vals + e0 + 2));
            q.v[0] = a.x;
            q.v[1] = a.y;
            q.v[2] = b.x;
            q.v[3] = b.y;
        } else {
            const float4 a = dev::ld_stream(reinterpret_cast<const float4*>(vals + e0));
            q.v[0] = a.x;
            q.v[1] = a.y;
            q.v[2] = a.z;
            q.v[3] = a.w;
        }
    } else {
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            if (q.mask & (1u << k)) {
                q.c[k] = dev::ld_stream(cols + e0 + k);
                q.v[k] = dev::ld_val<T>(vals + e0 + k);
            } else {
                q.c[k] = 0;
                q.v[k] = T(0);
            }
        }
    }
}

template <typename T, int N>
__device__ __forceinline__ void gather_quads(const T* __restrict__ x, const Quad<T> (&q)[N], T (&xv)[N][4]) {
#pragma unroll
    for (int j = 0; j < N; ++j)
#pragma unroll
        for (int k = 0; k < 4; ++k) xv[j][k] = (q[j].mask & (1u << k)) ? dev::ld_gather(x + q[j].c[k]) : T(0);
}

// Sum of alpha*a_j*x[col_j] over [cb, ce) by the whole CTA (VECTOR rows and
// LONG chunks). Each round a thread has two quads (8 nonzeros) in flight
// before it gathers x.
template <typename V, typename T, bool EXT, int NT>
__device__ __forceinline__ dev::Acc<T, EXT> range_sum(const V* __restrict__ vals,
                                                      const uint32_t* __restrict__ cols,
                                                      const T* __restrict__ x, T alpha, uint32_t cb,
                                                      uint32_t ce, uint32_t lo, uint32_t hi, bool vec) {
    dev::Acc<T, EXT> a;
    const uint32_t base = cb & ~3u;
    const uint32_t nq = (ce - base + 3) >> 2;
    constexpr int U = 2;
    for (uint32_t g0 = threadIdx.x; g0 < nq; g0 += U * NT) {
        Quad<T> q[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const uint32_t g = g0 + u * NT;
            if (g < nq)
                load_quad(vals, cols, base + 4 * g, cb, ce, lo, hi, vec, q[u]);
            else
                q[u].mask = 0;
        }
        T xv[U][4];
        gather_quads(x, q, xv);
#pragma unroll
        for (int u = 0; u < U; ++u)
#pragma unroll
            for (int k = 0; k < 4; ++k)
                if (q[u].mask & (1u << k)) a.add_prod(alpha * q[u].v[k], xv[u][k]);
    }
    return a;
}

constexpr uint32_t kRpStage = kBlkSize + 1;  // row pointers of a STREAM block kept in shared memory
constexpr uint32_t kStageRow = kBlkSize / 4 + 2;  // quads per block (+1 ragged) + 1 bank skew

// What a 128-position span of a STREAM block hands to the spans after it.
template <typename T>
struct SpanCarry {
    T open;          // sum from the span's last row start to its end (whole span if none)
    T pend;          // first row end in the span: sum from the span start to it
    int open_start;  // position of the span's last row start, -1 if none
    int any;         // the span holds a row start
    int has_pend;    // the span's first row end continues a row from an earlier span
};

// STREAM block without staging products: every thread keeps the products of
// its quads (4 consecutive nonzeros each; a warp covers 128 consecutive
// positions per span) in registers. Row starts are marked in a bitmap over the
// block's positions; each warp runs a segmented scan over its span with warp
// shuffles, rows ending inside the span are written by the lane that sees
// their end, and rows crossing spans are finished from the per-span carries.
// Summation order is fixed, so results are reproducible.
template <typename V, typename T, int K, int NT>
__device__ __forceinline__ void stream_segmented(const V* __restrict__ vals, const uint32_t* __restrict__ cols,
                                                 const uint32_t* __restrict__ rp, const T* __restrict__ x,
                                                 T alpha, uint32_t row, uint32_t nrows, uint32_t nb, uint32_t ne,
                                                 uint32_t lo, uint32_t hi, bool vec, uint32_t* srp,
                                                 uint32_t* bits, uint32_t* rid, SpanCarry<T>* spans,
                                                 RowSink<T, K>& sink) {
    constexpr int QPT = static_cast<int>(kBlkSize) / 4 / NT;
    constexpr int NW = NT / 32;
    constexpr int NREG = QPT * NW;  // regular spans; one more for the ragged quad
    const uint32_t tid = threadIdx.x;
    const uint32_t lane = tid & 31u, warp = tid >> 5;
    const uint32_t base = nb & ~3u;
    const uint32_t nq = (ne - base + 3) >> 2;
    const bool extra = nq > static_cast<uint32_t>(QPT * NT);

    for (uint32_t i = tid; i < kBlkSize / 32 + 8; i += NT) bits[i] = 0u;
    if (tid < static_cast<uint32_t>(NREG + 1)) {
        spans[tid].has_pend = 0;
        spans[tid].any = 0;
        spans[tid].open = T(0);
        spans[tid].open_start = -1;
    }
    Quad<T> q[QPT];
#pragma unroll
    for (int j = 0; j < QPT; ++j) {
        const uint32_t g = tid + j * NT;
        if (g < nq)
            load_quad(vals, cols, base + 4 * g, nb, ne, lo, hi, vec, q[j]);
        else
            q[j].mask = 0;
    }
    Quad<T> qx[1];
    qx[0].mask = 0;
    if (extra && warp == 0 && QPT * NT + lane < nq)
        load_quad(vals, cols, base + 4 * (QPT * NT + lane), nb, ne, lo, hi, vec, qx[0]);
    for (uint32_t i = tid; i <= nrows; i += NT) srp[i] = dev::ld_ro(rp + row + i);
    T xv[QPT][4];
    gather_quads(x, q, xv);
    T xx[1][4];
    gather_quads(x, qx, xx);
    __syncthreads();
    // row starts of the non-empty rows; empty rows are final already
    for (uint32_t r = tid; r < nrows; r += NT) {
        const uint32_t s = srp[r] - base, e = srp[r + 1] - base;
        if (e > s) {
            atomicOr(&bits[s >> 5], 1u << (s & 31u));
            rid[s] = r;
        } else {
            dev::Acc<T, false> z;
            sink.template put<false>(row + r, z);
        }
    }
    __syncthreads();
    auto emit = [&](int pos, T total) {
        dev::Acc<T, false> a;
        a.s = total;
        sink.template put<false>(row + rid[pos], a);
    };
    // segmented scan of one span; p = this lane's four products, qd its quad
    auto span = [&](int S, uint32_t qd, const T (&p)[4]) {
        const uint32_t pos0 = 4u * qd;
        const uint32_t fl = (bits[pos0 >> 5] >> (pos0 & 31u)) & 0xFu;
        T head = T(0), run = T(0);
        int cur = -1;
        bool seen = false;
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            if (fl & (1u << k)) {
                if (!seen) {
                    head = run;
                    seen = true;
                } else {
                    emit(cur, run);  // a row that starts and ends inside this quad
                }
                run = T(0);
                cur = static_cast<int>(pos0) + k;
            }
            run += p[k];
        }
        if (!seen) head = run;
        T v = run;
        int f = seen ? 1 : 0;
        int sp = seen ? cur : -1;
#pragma unroll
        for (int off = 1; off < 32; off <<= 1) {
            const T vu = __shfl_up_sync(0xffffffffu, v, off);
            const int fu = __shfl_up_sync(0xffffffffu, f, off);
            const int su = __shfl_up_sync(0xffffffffu, sp, off);
            if (lane >= static_cast<uint32_t>(off)) {
                if (!f) {
                    v += vu;
                    sp = su;
                }
                f |= fu;
            }
        }
        T rp_ = __shfl_up_sync(0xffffffffu, v, 1);
        int fp = __shfl_up_sync(0xffffffffu, f, 1);
        int spp = __shfl_up_sync(0xffffffffu, sp, 1);
        if (lane == 0) {
            rp_ = T(0);
            fp = 0;
            spp = -1;
        }
        if (seen) {
            const T total = rp_ + head;  // the row ending at this lane's first start
            if (fp) {
                emit(spp, total);
            } else {
                spans[S].pend = total;
                spans[S].has_pend = 1;
            }
        }
        if (lane == 31) {
            spans[S].open = v;
            spans[S].open_start = f ? sp : -1;
            spans[S].any = f;
        }
    };
#pragma unroll
    for (int j = 0; j < QPT; ++j) {
        T p[4];
#pragma unroll
        for (int k = 0; k < 4; ++k)
            p[k] = (q[j].mask & (1u << k)) ? dev::mul_rn(alpha * q[j].v[k], xv[j][k]) : T(0);
        span(j * NW + static_cast<int>(warp), j * NT + tid, p);
    }
    if (extra && warp == 0) {
        T p[4];
#pragma unroll
        for (int k = 0; k < 4; ++k)
            p[k] = (qx[0].mask & (1u << k)) ? dev::mul_rn(alpha * qx[0].v[k], xx[0][k]) : T(0);
        span(NREG, QPT * NT + lane, p);
    }
    __syncthreads();
    // rows that cross spans: the first row end of a span (and the block end)
    const int nspans = NREG + (extra ? 1 : 0);
    if (tid <= static_cast<uint32_t>(nspans)) {
        const int S = static_cast<int>(tid);
        if (S == nspans || spans[S].has_pend) {
            T total = S < nspans ? spans[S].pend : T(0);
            int s = S - 1;
            while (s >= 0 && !spans[s].any) {
                total += spans[s].open;
                --s;
            }
            if (s >= 0 && spans[s].open_start >= 0) emit(spans[s].open_start, total + spans[s].open);
        }
    }
}

template <typename V, typename T, bool EXT, int K, int NT>
__global__ void __launch_bounds__(NT)
    csr_adaptive_kernel(const V* __restrict__ vals, const uint32_t* __restrict__ cols,
                        const uint32_t* __restrict__ rp, const T* __restrict__ x, T* __restrict__ y,
                        const T* __restrict__ alpha_p, const T* __restrict__ beta_p,
                        const uint64_t* __restrict__ words, const uint32_t* __restrict__ word_nnz,
                        uint32_t nblocks, uint32_t lo, uint32_t hi, int vec,
                        double* __restrict__ lr_partial, uint32_t* __restrict__ lr_ticket,
                        EpiDev<T> epi) {
    // Products of a STREAM block, quad-transposed: element e (counted from the
    // block's 16-byte-aligned start) lives at stage[(e & 3) * kStageRow + e / 4],
    // so a warp's stores of one quad slot are contiguous and the row
    // reductions read with few bank conflicts.
    __shared__ T stage[4 * kStageRow];
    __shared__ uint32_t srp[kRpStage];
    __shared__ T red_s[32];
    __shared__ T red_c[32];
    __shared__ bool lr_last;
    // segmented STREAM reduction: row-start bitmap over the block's positions,
    // the block row starting at each flagged position, per-span carries
    constexpr int kSpans = static_cast<int>(kBlkSize) / 128 + 1;
    __shared__ uint32_t seg_bits[kBlkSize / 32 + 8];
    __shared__ uint32_t seg_row[kBlkSize + 8];
    __shared__ SpanCarry<T> spans[kSpans];

    if (epi.done != nullptr && *epi.done) return;

    const T alpha = *alpha_p;
    RowSink<T, K> sink;
    sink.init(y, epi, *beta_p);

    const uint32_t gid = blockIdx.x;
    if (gid < nblocks) {
        // Independent loads: the block's words and the nonzero offsets of
        // their first rows (no dependent row-pointer load).
        const uint64_t w0 = words[gid];
        const uint64_t w1 = words[gid + 1];
        const uint32_t nb = word_nnz[gid];
        const uint32_t ne = word_nnz[gid + 1];
        const uint32_t row = static_cast<uint32_t>(w0 >> 32);
        const uint32_t stop = static_cast<uint32_t>(w1 >> 32);
        const uint32_t low = static_cast<uint32_t>(w0 & ((1u << kWgBits) - 1u));
        const uint32_t nrows = stop - row;
        const uint32_t tid = threadIdx.x;

        if (nrows > kRowsForVector && !EXT && ne - nb <= kBlkSize && nrows < kRpStage) {
            // ---- STREAM, segmented: products stay in registers ----
            stream_segmented<V, T, K, NT>(vals, cols, rp, x, alpha, row, nrows, nb, ne, lo, hi, vec != 0,
                                          srp, seg_bits, seg_row, spans, sink);
        } else if (nrows > kRowsForVector) {
            // ---- STREAM: several short rows, <= kBlkSize nonzeros in total ----
            const uint32_t cnt = ne - nb;
            // A block from clsparseCsrMetaCreate never exceeds the staging
            // buffer; if the row pointers changed after the meta was made, the
            // rows are summed straight from global memory instead.
            const bool staged = cnt <= kBlkSize;
            const bool rp_staged = nrows < kRpStage;
            if (staged) {
                constexpr int QPT = static_cast<int>(kBlkSize) / 4 / NT;
                const uint32_t base = nb & ~3u;
                const uint32_t nq = (ne - base + 3) >> 2;  // <= kBlkSize/4 + 1
                Quad<T> q[QPT];
#pragma unroll
                for (int j = 0; j < QPT; ++j) {
                    const uint32_t g = tid + j * NT;
                    if (g < nq)
                        load_quad(vals, cols, base + 4 * g, nb, ne, lo, hi, vec != 0, q[j]);
                    else
                        q[j].mask = 0;
                }
                if (rp_staged)
                    for (uint32_t i = tid; i <= nrows; i += NT) srp[i] = dev::ld_ro(rp + row + i);
                T xv[QPT][4];
                gather_quads(x, q, xv);
#pragma unroll
                for (int j = 0; j < QPT; ++j) {
                    const uint32_t e0 = base + 4 * (tid + j * NT);
#pragma unroll
                    for (int k = 0; k < 4; ++k)
                        if (q[j].mask & (1u << k))
                            stage[k * kStageRow + (e0 - base) / 4] = dev::mul_rn(alpha * q[j].v[k], xv[j][k]);
                }
                // the quad past QPT*NT, present when the block starts unaligned
                for (uint32_t g = QPT * NT + tid; g < nq; g += NT) {
                    Quad<T> r[1];
                    load_quad(vals, cols, base + 4 * g, nb, ne, lo, hi, vec != 0, r[0]);
                    T rv[1][4];
                    gather_quads(x, r, rv);
#pragma unroll
                    for (int k = 0; k < 4; ++k)
                        if (r[0].mask & (1u << k)) stage[k * kStageRow + g] = dev::mul_rn(alpha * r[0].v[k], rv[0][k]);
                }
            } else if (rp_staged) {
                for (uint32_t i = tid; i <= nrows; i += NT) srp[i] = dev::ld_ro(rp + row + i);
            }
            __syncthreads();
            // Lanes per row: the reference's per-block reduction width, capped at
            // one warp so each row reduces with shuffles inside a warp.
            const uint32_t gw = low == 0 ? 1u : (low > 32u ? 32u : low);
            auto reduce_rows = [&](auto gc) {
                constexpr int G = decltype(gc)::value;
                const uint32_t groups = NT / G;
                const uint32_t grp = tid / G;
                const uint32_t lane = tid & (G - 1);
                for (uint32_t rb = 0; rb < nrows; rb += groups) {
                    const uint32_t r = rb + grp;
                    dev::Acc<T, EXT> a;
                    if (r < nrows) {
                        const uint32_t f = (rp_staged ? srp[r] : dev::ld_ro(rp + row + r)) - nb;
                        const uint32_t l = (rp_staged ? srp[r + 1] : dev::ld_ro(rp + row + r + 1)) - nb;
                        if (staged) {
                            const uint32_t off = nb & 3u;
                            for (uint32_t j = f + lane; j < l; j += G) {
                                const uint32_t e = j + off;
                                a.add(stage[(e & 3u) * kStageRow + (e >> 2)]);
                            }
                        } else {
                            for (uint32_t j = nb + f + lane; j < nb + l; j += G)
                                a.add(dev::mul_rn(alpha * dev::ld_val<T>(vals + j), dev::ld_ro(x + cols[j])));
                        }
                    }
                    dev::group_reduce<G>(a);
                    if (r < nrows && lane == 0) sink.template put<EXT>(row + r, a);
                }
            };
            switch (gw) {
                case 1: reduce_rows(std::integral_constant<int, 1>{}); break;
                case 2: reduce_rows(std::integral_constant<int, 2>{}); break;
                case 4: reduce_rows(std::integral_constant<int, 4>{}); break;
                case 8: reduce_rows(std::integral_constant<int, 8>{}); break;
                case 16: reduce_rows(std::integral_constant<int, 16>{}); break;
                default: reduce_rows(std::integral_constant<int, 32>{}); break;
            }
        } else if (nrows == 1 && low == 0) {
            // ---- VECTOR: one row, the whole CTA ----
            dev::Acc<T, EXT> a = range_sum<V, T, EXT, NT>(vals, cols, x, alpha, nb, ne, lo, hi, vec != 0);
            a = dev::block_reduce_acc(a, red_s, red_c);
            if (tid == 0) sink.template put<EXT>(row, a);
        } else {
            // ---- LONG: chunk `low` of a row split over several CTAs ----
            const uint32_t re = dev::ld_ro(rp + row + 1);
            const uint32_t len = re - nb;
            const uint32_t nchunks = (len + kLongChunk - 1) / kLongChunk;
            if (nchunks >= 2 && low < nchunks) {
                const uint32_t first = gid - low;
                const uint32_t cb = nb + low * kLongChunk;
                const uint32_t ce = min(re, cb + kLongChunk);
                dev::Acc<T, EXT> a = range_sum<V, T, EXT, NT>(vals, cols, x, alpha, cb, ce, lo, hi, vec != 0);
                a = dev::block_reduce_acc(a, red_s, red_c);
                if (tid == 0) {
                    // partial of this chunk; compensation folded in
                    lr_partial[gid] = static_cast<double>(a.value());
                    __threadfence();
                    const uint32_t t = atomicAdd(lr_ticket + first, 1u);
                    lr_last = (t == nchunks - 1);
                }
                __syncthreads();
                if (lr_last && tid == 0) {
                    __threadfence();
                    dev::Acc<T, EXT> tot;
                    for (uint32_t w = 0; w < nchunks; ++w)
                        tot.add(static_cast<T>(__ldcg(lr_partial + first + w)));
                    lr_ticket[first] = 0u;
                    sink.template put<EXT>(row, tot);
                }
            }
        }
    }
    run_epilogue<T, K>(sink, epi);
}

template <typename V, typename T, bool EXT, int G, int K>
__global__ void __launch_bounds__(kThreads)
    csr_vector_kernel(const V* __restrict__ vals, const uint32_t* __restrict__ cols,
                      const uint32_t* __restrict__ rp, const T* __restrict__ x, T* __restrict__ y,
                      const T* __restrict__ alpha_p, const T* __restrict__ beta_p, uint32_t nrows,
                      EpiDev<T> epi) {
    if (epi.done != nullptr && *epi.done) return;
    const T alpha = *alpha_p;
    RowSink<T, K> sink;
    sink.init(y, epi, *beta_p);
    const uint32_t lane = threadIdx.x & (G - 1);
    const uint64_t gtid = static_cast<uint64_t>(blockIdx.x) * kThreads + threadIdx.x;
    const uint32_t grp = static_cast<uint32_t>(gtid / G);
    const uint32_t ngroups = static_cast<uint32_t>(static_cast<uint64_t>(gridDim.x) * kThreads / G);
    for (uint32_t base = 0; base < nrows; base += ngroups) {
        const uint32_t row = base + grp;
        dev::Acc<T, EXT> a;
        if (row < nrows) {
            const uint32_t nb = dev::ld_ro(rp + row);
            const uint32_t ne = dev::ld_ro(rp + row + 1);
            for (uint32_t j = nb + lane; j < ne; j += G)
                a.add_prod(alpha * dev::ld_val<T>(vals + j), dev::ld_ro(x + dev::ld_stream(cols + j)));
        }
        dev::group_reduce<G>(a);
        if (row < nrows && lane == 0) sink.template put<EXT>(row, a);
        if (base > 0xFFFFFFFFu - ngroups) break;
    }
    run_epilogue<T, K>(sink, epi);
}

template <typename T>
EpiDev<T> to_dev(const SpmvEpilogue& e) {
    EpiDev<T> d;
    d.w0 = static_cast<const T*>(e.w0);
    d.dot1_self = e.dot1_self ? 1 : 0;
    d.partials = e.partials;
    d.ticket = e.ticket;
    d.op = static_cast<int>(e.op);
    d.state = e.state;
    d.cond = e.cond;
    d.done = e.done;
    return d;
}

// Sub-warp width of the vector kernel from the average row length
// (reference blas2/csrmv-vector.hpp:34-49 with a 32-wide warp).
uint32_t vector_width(uint32_t nrows, uint32_t nnz) {
    const uint32_t per_row = nrows ? nnz / nrows : 0;
    uint32_t g = 32;
    if (per_row < 32) g = 16;
    if (per_row < 16) g = 8;
    if (per_row < 8) g = 4;
    if (per_row < 4) g = 2;
    return g;
}

uint32_t vector_grid(uint32_t nrows, uint32_t g) {
    const uint64_t threads = static_cast<uint64_t>(nrows) * g;
    uint64_t ctas = (threads + kThreads - 1) / kThreads;
    if (ctas == 0) ctas = 1;
    if (ctas > 0x7fffffffull) ctas = 0x7fffffffull;
    return static_cast<uint32_t>(ctas);
}

template <typename V, typename T, bool EXT, int K>
cudaError_t launch_vector(const CsrView<V>& A, const T* alpha, const T* beta, const T* x, T* y,
                          const EpiDev<T>& e, cudaStream_t s) {
    const uint32_t g = vector_width(A.nrows, A.nnz);
    const uint32_t grid = vector_grid(A.nrows, g);
#define CLSP_VEC(GW)                                                                              \
    csr_vector_kernel<V, T, EXT, GW, K><<<grid, kThreads, 0, s>>>(A.vals, A.cols, A.rp, x, y, alpha, \
                                                               beta, A.nrows, e)
    switch (g) {
        case 2: CLSP_VEC(2); break;
        case 4: CLSP_VEC(4); break;
        case 8: CLSP_VEC(8); break;
        case 16: CLSP_VEC(16); break;
        default: CLSP_VEC(32); break;
    }
#undef CLSP_VEC
    return cudaGetLastError();
}

#include "spmv_tma.cuh"

// Adaptive kernel choice: one CTA per row block (default) or the TMA-staged
// persistent pipeline (CLSPARSE_B200_SPMV_KERNEL=tma), which measured slower
// on the irregular workload (its per-block barriers leave too little work in
// flight per SM).
bool use_tma_kernel() {
    static bool on = [] {
        const char* e = std::getenv("CLSPARSE_B200_SPMV_KERNEL");
        return e && std::string(e) == "tma";
    }();
    return on;
}

template <typename V, typename T, bool EXT, int K>
cudaError_t launch_tma(const CsrView<V>& A, const T* alpha, const T* beta, const T* x, T* y,
                       const EpiDev<T>& e, cudaStream_t s, int* err) {
    using L = tma::Layout<V, T>;
    auto kern = tma::csr_adaptive_tma_kernel<V, T, EXT, K>;
    static int blocks_per_sm = -1;
    static int sms = 0;
    if (blocks_per_sm < 0) {
        cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(L::total));
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        int b = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, kern, tma::kThreads, L::total);
        blocks_per_sm = b > 0 ? b : 1;
    }
    const matrix_meta* m = A.meta;
    const uint32_t nblocks = static_cast<uint32_t>(m->num_words - 1);
    uint64_t grid = static_cast<uint64_t>(sms) * blocks_per_sm;
    if (grid > nblocks) grid = nblocks;
    if (grid == 0) grid = 1;
    const int aligned = ((reinterpret_cast<uintptr_t>(A.vals) | reinterpret_cast<uintptr_t>(A.cols) |
                          reinterpret_cast<uintptr_t>(A.rp)) & 15u) == 0;
    kern<<<static_cast<uint32_t>(grid), tma::kThreads, L::total, s>>>(
        A.vals, A.cols, A.rp, x, y, alpha, beta, m->d_rowBlocks, m->d_word_nnz, nblocks, A.nrows,
        m->nnz_hi, aligned, m->d_lr_partial, m->d_lr_ticket, err, e);
    return cudaGetLastError();
}

// Threads per CTA of the adaptive kernel (128 or 256); CLSPARSE_B200_SPMV_NT
// overrides the default for tuning.
int adaptive_threads() {
    static int nt = [] {
        const char* e = std::getenv("CLSPARSE_B200_SPMV_NT");
        const int v = e ? std::atoi(e) : 128;
        return v == 256 ? 256 : 128;
    }();
    return nt;
}

template <typename V, typename T, bool EXT, int K>
cudaError_t launch_kind(const CsrView<V>& A, const T* alpha, const T* beta, const T* x, T* y,
                        const EpiDev<T>& e, cudaStream_t s) {
    if (A.meta == nullptr) return launch_vector<V, T, EXT, K>(A, alpha, beta, x, y, e, s);
    const uint32_t nblocks = static_cast<uint32_t>(A.meta->num_words - 1);
    uint32_t grid = nblocks;
    if (grid == 0) {
        if (K == 0) return cudaSuccess;
        grid = 1;  // one idle CTA still finishes the fused reduction
    }
    if (use_tma_kernel()) return launch_tma<V, T, EXT, K>(A, alpha, beta, x, y, e, s, A.meta->d_error);
    const int vec = ((reinterpret_cast<uintptr_t>(A.vals) | reinterpret_cast<uintptr_t>(A.cols)) & 15u) == 0;
    const matrix_meta* m = A.meta;
    if (adaptive_threads() == 256)
        csr_adaptive_kernel<V, T, EXT, K, 256><<<grid, 256, 0, s>>>(
            A.vals, A.cols, A.rp, x, y, alpha, beta, m->d_rowBlocks, m->d_word_nnz, nblocks, m->nnz_lo,
            m->nnz_hi, vec, m->d_lr_partial, m->d_lr_ticket, e);
    else
        csr_adaptive_kernel<V, T, EXT, K, 128><<<grid, 128, 0, s>>>(
            A.vals, A.cols, A.rp, x, y, alpha, beta, m->d_rowBlocks, m->d_word_nnz, nblocks, m->nnz_lo,
            m->nnz_hi, vec, m->d_lr_partial, m->d_lr_ticket, e);
    return cudaGetLastError();
}

}  // namespace

uint32_t spmv_num_ctas(const matrix_meta* meta, uint32_t nrows, uint32_t nnz) {
    if (meta) return std::max<uint32_t>(1u, static_cast<uint32_t>(meta->num_words - 1));
    return vector_grid(nrows, vector_width(nrows, nnz));
}

template <typename V, typename T>
cudaError_t launch_csrmv(const CsrView<V>& A, const T* alpha, const T* beta, const T* x, T* y,
                         bool extended, const SpmvEpilogue& epi, cudaStream_t s) {
    const EpiDev<T> e = to_dev<T>(epi);
    if (extended) {
        if (epi.ndots == 0) return launch_kind<V, T, true, 0>(A, alpha, beta, x, y, e, s);
        if (epi.ndots == 1) return launch_kind<V, T, true, 1>(A, alpha, beta, x, y, e, s);
        return launch_kind<V, T, true, 2>(A, alpha, beta, x, y, e, s);
    }
    if (epi.ndots == 0) return launch_kind<V, T, false, 0>(A, alpha, beta, x, y, e, s);
    if (epi.ndots == 1) return launch_kind<V, T, false, 1>(A, alpha, beta, x, y, e, s);
    return launch_kind<V, T, false, 2>(A, alpha, beta, x, y, e, s);
}

template cudaError_t launch_csrmv<float, float>(const CsrView<float>&, const float*, const float*,
                                                const float*, float*, bool, const SpmvEpilogue&,
                                                cudaStream_t);
template cudaError_t launch_csrmv<double, double>(const CsrView<double>&, const double*,
                                                  const double*, const double*, double*, bool,
                                                  const SpmvEpilogue&, cudaStream_t);
template cudaError_t launch_csrmv<__nv_bfloat16, float>(const CsrView<__nv_bfloat16>&, const float*,
                                                        const float*, const float*, float*, bool,
                                                        const SpmvEpilogue&, cudaStream_t);

namespace {

template <typename T>
clsparseStatus csrmv_entry(const clsparseScalar* alpha, const clsparseCsrMatrix* A,
                           const cldenseVector* x, const clsparseScalar* beta, cldenseVector* y,
                           clsparseControl control) {
    clsparseStatus st = check_entry(control);
    if (st != clsparseSuccess) return st;
    if (!alpha || !A || !x || !beta || !y) return clsparseInvalidValue;
    if (x->num_values < A->num_cols || y->num_values < A->num_rows) return clsparseInvalidSize;
    if (A->num_rows == 0) return clsparseSuccess;
    if (!alpha->value || !beta->value || !x->values || !y->values || !A->row_pointer ||
        (A->num_nonzeros > 0 && (!A->values || !A->col_indices)))
        return clsparseInvalidMemObject;
    const auto* meta = static_cast<const matrix_meta*>(A->meta);
    if (meta && meta->rowBlockSize == 0) return clsparseStructInvalid;
    if (meta && meta->num_rows != A->num_rows) return clsparseStructInvalid;
    DeviceGuard g(control->device);
    CsrView<T> v{dev_ptr<const T>(A->values, A->off_values),
                 dev_ptr<const uint32_t>(A->col_indices, A->off_col_indices),
                 dev_ptr<const uint32_t>(A->row_pointer, A->off_row_pointer),
                 A->num_rows, A->num_cols, A->num_nonzeros, meta};
    SpmvEpilogue none;
    cudaError_t e = launch_csrmv<T, T>(v, dev_ptr<const T>(alpha->value, alpha->off_value),
                                    dev_ptr<const T>(beta->value, beta->off_value),
                                    dev_ptr<const T>(x->values, x->off_values),
                                    dev_ptr<T>(y->values, y->off_values), control->extended_precision,
                                    none, control->stream);
    if (e != cudaSuccess) return clsparseInvalidKernelExecution;
    return finish_call(control);
}

}  // namespace

}  // namespace clsp

extern "C" {

clsparseStatus clsparseScsrmv(const clsparseScalar* alpha, const clsparseCsrMatrix* matx,
                              const cldenseVector* x, const clsparseScalar* beta, cldenseVector* y,
                              const clsparseControl control) {
    return clsp::csrmv_entry<float>(alpha, matx, x, beta, y, control);
}

clsparseStatus clsparseDcsrmv(const clsparseScalar* alpha, const clsparseCsrMatrix* matx,
                              const cldenseVector* x, const clsparseScalar* beta, cldenseVector* y,
                              const clsparseControl control) {
    return clsp::csrmv_entry<double>(alpha, matx, x, beta, y, control);
}

}  // extern "C"
