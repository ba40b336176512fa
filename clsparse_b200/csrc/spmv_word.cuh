// One CSR-Adaptive row-block word processed by one CTA: the device code
// shared by the one-CTA-per-word SpMV kernel (spmv.cu) and the persistent
// solver kernels (fused_cg.cu), which walk a static range of words per CTA.
//
// Word modes (the CSR-Adaptive scheme of the reference's
// src/library/kernels/csrmv_adaptive.cl:312-687, rebuilt for B200):
//   STREAM  several short rows (<= 1024 nonzeros in total): products
//           alpha*val*x[col] of the whole block are staged in shared memory
//           with coalesced evict-first loads, then every row is reduced out of
//           shared memory by a group of up to 32 lanes (warp shuffles).
//   VECTOR  one row (up to 3072 nonzeros): the whole CTA reduces it.
//   LONG    one chunk of 3072 nonzeros of a longer row; the chunk CTAs merge
//           through per-word partial slots and an arrival ticket, and the
//           last to arrive writes y. Nobody waits.
#pragma once

#include <type_traits>

#include "device_common.cuh"
#include "internal.h"
#include "solver_state.cuh"

namespace clsp {
namespace {

constexpr uint32_t kLongChunk = kBlkSize * kBlockMultiplier;  // 3072 nonzeros per CTA (default shape)

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
        // two levels pay only on large grids (measured: 14k CTAs -8 % per CG
        // iteration, 1.3k CTAs +7 %)
        const bool last = gridDim.x > 2048 ? dev::grid_reduce_tree<K>(sink.d, e.partials, e.ticket, tot)
                                           : dev::grid_reduce_last<K>(sink.d, e.partials, e.ticket, tot);
        if (last) {
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

// Source of the gathered vector entries x[c]: the dense vector itself
// (read-only path, or coherent when other CTAs of the launch wrote it).
template <typename T, bool COH = false>
struct DenseX {
    const T* x;
    __device__ __forceinline__ T operator()(uint32_t c) const { return dev::ld_x<COH>(x + c); }
};

template <int N, typename T, typename XS>
__device__ __forceinline__ void gather_quads(const XS& xs, const Quad<T> (&q)[N], T (&xv)[N][4]) {
#pragma unroll
    for (int j = 0; j < N; ++j)
#pragma unroll
        for (int k = 0; k < 4; ++k) xv[j][k] = (q[j].mask & (1u << k)) ? xs(q[j].c[k]) : T(0);
}

// Sum of alpha*a_j*x[col_j] over [cb, ce) by the whole CTA (VECTOR rows and
// LONG chunks). Each round a thread has two quads (8 nonzeros) in flight
// before it gathers x.
template <typename V, typename T, bool EXT, int NT, typename XS>
__device__ __forceinline__ dev::Acc<T, EXT> range_sum(const V* __restrict__ vals,
                                                      const uint32_t* __restrict__ cols,
                                                      const XS& x, T alpha, uint32_t cb,
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
        gather_quads<U>(x, q, xv);
#pragma unroll
        for (int u = 0; u < U; ++u)
#pragma unroll
            for (int k = 0; k < 4; ++k)
                if (q[u].mask & (1u << k)) a.add_prod(alpha * q[u].v[k], xv[u][k]);
    }
    return a;
}

// Row-block shape of a meta: BLK (the reference's BLKSIZE) is a template
// parameter of the kernels (shared-memory staging and per-thread quads are
// sized by it); ROWS_FOR_VECTOR and the long-row chunk
// (BLOCK_MULTIPLIER * BLKSIZE) are runtime values.
struct WordShape {
    uint32_t rows_for_vector;
    uint32_t chunk;
};

// Shared memory of one word's processing.
template <typename T, int BLK = static_cast<int>(kBlkSize)>
struct WordSmem {
    static constexpr uint32_t kRpStage = BLK + 1;     // row pointers of a STREAM block
    static constexpr uint32_t kStageRow = BLK / 4 + 2;  // quads per block (+1 ragged) + 1 bank skew
    // Products of a STREAM block, quad-transposed: element e (counted from the
    // block's 16-byte-aligned start) lives at stage[(e & 3) * kStageRow + e / 4],
    // so a warp's stores of one quad slot are contiguous and the row
    // reductions read with few bank conflicts.
    T stage[4 * kStageRow];
    uint32_t srp[kRpStage];
    T red_s[32];
    T red_c[32];
    bool lr_last;
};

// Processes row-block word `gid` (0 <= gid < number of words - 1) with the
// whole CTA (NT threads). x(c) yields the vector entry of column c; every row
// the word finishes goes through sink.put. The caller separates two calls on
// the same shared memory with a barrier.
template <typename V, typename T, bool EXT, int NT, int BLK, typename XS, typename Sink>
__device__ __forceinline__ void adaptive_word(uint32_t gid, const V* __restrict__ vals,
                                              const uint32_t* __restrict__ cols,
                                              const uint32_t* __restrict__ rp, const XS& x,
                                              T alpha, const uint64_t* __restrict__ words,
                                              const uint32_t* __restrict__ word_nnz, uint32_t lo,
                                              uint32_t hi, int vec, double* __restrict__ lr_partial,
                                              uint32_t* __restrict__ lr_ticket, WordShape shape,
                                              WordSmem<T, BLK>& sm, Sink& sink) {
    constexpr uint32_t kRpStage = WordSmem<T, BLK>::kRpStage;
    constexpr uint32_t kStageRow = WordSmem<T, BLK>::kStageRow;
    static_assert(BLK / 4 / NT >= 1, "a block needs at least one quad per thread");
    T* stage = sm.stage;
    uint32_t* srp = sm.srp;
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
    if (nrows > shape.rows_for_vector) {
        // ---- STREAM: several short rows, <= BLK nonzeros in total ----
        const uint32_t cnt = ne - nb;
        // A block from clsparseCsrMetaCreate never exceeds the staging
        // buffer; if the row pointers changed after the meta was made, the
        // rows are summed straight from global memory instead.
        const bool staged = cnt <= static_cast<uint32_t>(BLK);
        const bool rp_staged = nrows < kRpStage;
        if (staged) {
            constexpr int QPT = BLK / 4 / NT;
            const uint32_t base = nb & ~3u;
            const uint32_t nq = (ne - base + 3) >> 2;  // <= BLK/4 + 1
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
            gather_quads<QPT>(x, q, xv);
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
                gather_quads<1>(x, r, rv);
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
                            a.add(dev::mul_rn(alpha * dev::ld_val<T>(vals + j), x(cols[j])));
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
    } else if (nrows >= 1 && low == 0) {
        // ---- VECTOR: up to ROWS_FOR_VECTOR rows, one at a time, the whole CTA
        // (the reference's CSR-Vector branch, csrmv_adaptive.cl:517-610) ----
        for (uint32_t rr = 0; rr < nrows; ++rr) {
            const uint32_t rb = rr == 0 ? nb : dev::ld_ro(rp + row + rr);
            const uint32_t re = rr + 1 == nrows ? ne : dev::ld_ro(rp + row + rr + 1);
            dev::Acc<T, EXT> a = range_sum<V, T, EXT, NT>(vals, cols, x, alpha, rb, re, lo, hi, vec != 0);
            a = dev::block_reduce_acc(a, sm.red_s, sm.red_c);
            if (tid == 0) sink.template put<EXT>(row + rr, a);
        }
    } else {
        // ---- LONG: chunk `low` of a row split over several CTAs ----
        const uint32_t re = dev::ld_ro(rp + row + 1);
        const uint32_t len = re - nb;
        const uint32_t chunk = shape.chunk;
        const uint32_t nchunks = (len + chunk - 1) / chunk;
        if (nchunks >= 2 && low < nchunks) {
            const uint32_t first = gid - low;
            const uint32_t cb = nb + low * chunk;
            const uint32_t ce = min(re, cb + chunk);
            dev::Acc<T, EXT> a = range_sum<V, T, EXT, NT>(vals, cols, x, alpha, cb, ce, lo, hi, vec != 0);
            a = dev::block_reduce_acc(a, sm.red_s, sm.red_c);
            if (tid == 0) {
                // partial of this chunk; compensation folded in
                lr_partial[gid] = static_cast<double>(a.value());
                __threadfence();
                const uint32_t t = atomicAdd(lr_ticket + first, 1u);
                sm.lr_last = (t == nchunks - 1);
            }
            __syncthreads();
            if (sm.lr_last && tid == 0) {
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

}  // namespace
}  // namespace clsp
