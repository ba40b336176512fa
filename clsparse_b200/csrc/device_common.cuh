// Device helpers shared by the SpMV, BLAS-1 and solver kernels: cache-hinted
// loads, compensated accumulation, warp / CTA reductions and the
// deterministic grid reduction that lets the last CTA of a launch finish a
// reduction without a second kernel and without any spin-wait.
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <type_traits>

namespace clsp {
namespace dev {

// Streaming loads for data read exactly once (matrix values and column
// indices): evict-first, so the gathered vector stays in L2.
template <typename T>
__device__ __forceinline__ T ld_stream(const T* p) {
    return __ldcs(p);
}

// Read-only loads through the non-coherent path (gathered vector, row pointers).
template <typename T>
__device__ __forceinline__ T ld_ro(const T* p) {
    return __ldg(p);
}

// Gathered loads of the dense vector x. CLSP_GATHER selects the cache
// treatment: 0 read-only path (default), 1 L2 only, 2 read-only without L1
// allocation.
#ifndef CLSP_GATHER
#define CLSP_GATHER 0
#endif
__device__ __forceinline__ double ld_gather(const double* p) {
#if CLSP_GATHER == 1
    return __ldcg(p);
#elif CLSP_GATHER == 2
    double v;
    asm volatile("ld.global.nc.L1::no_allocate.f64 %0, [%1];" : "=d"(v) : "l"(p));
    return v;
#else
    return __ldg(p);
#endif
}
__device__ __forceinline__ float ld_gather(const float* p) {
#if CLSP_GATHER == 1
    return __ldcg(p);
#elif CLSP_GATHER == 2
    float v;
    asm volatile("ld.global.nc.L1::no_allocate.f32 %0, [%1];" : "=f"(v) : "l"(p));
    return v;
#else
    return __ldg(p);
#endif
}

// Coherent gather for kernels that read a vector other CTAs of the same
// launch wrote before a grid barrier (the persistent solvers): a plain weak
// load, which the barrier's acquire orders, never the non-coherent
// read-only path (whose data must not change while the kernel runs).
__device__ __forceinline__ double ld_coherent(const double* p) {
    double v;
    asm volatile("ld.global.f64 %0, [%1];" : "=d"(v) : "l"(p));
    return v;
}
__device__ __forceinline__ float ld_coherent(const float* p) {
    float v;
    asm volatile("ld.global.f32 %0, [%1];" : "=f"(v) : "l"(p));
    return v;
}

// Gather of x[c]: read-only path, or coherent when COH.
template <bool COH, typename T>
__device__ __forceinline__ T ld_x(const T* p) {
    if constexpr (COH) {
        return ld_coherent(p);
    } else {
        return ld_gather(p);
    }
}

// Loads one matrix value (double, float or bf16) as the arithmetic type T.
template <typename T, typename V>
__device__ __forceinline__ T ld_val(const V* p) {
    if constexpr (std::is_same_v<V, __nv_bfloat16>) {
        const unsigned short u = __ldcs(reinterpret_cast<const unsigned short*>(p));
        return static_cast<T>(__uint_as_float(static_cast<unsigned>(u) << 16));
    } else {
        return static_cast<T>(__ldcs(p));
    }
}

// The same through the read-only (L1-allocating) path, for access patterns in
// which neighbouring threads read the same lines in different iterations
// (one thread per row).
template <typename T, typename V>
__device__ __forceinline__ T ld_val_ro(const V* p) {
    if constexpr (std::is_same_v<V, __nv_bfloat16>) {
        const unsigned short u = __ldg(reinterpret_cast<const unsigned short*>(p));
        return static_cast<T>(__uint_as_float(static_cast<unsigned>(u) << 16));
    } else {
        return static_cast<T>(__ldg(p));
    }
}

// Converts a matrix value held in registers or shared memory to T.
template <typename T, typename V>
__device__ __forceinline__ T to_t(V v) {
    if constexpr (std::is_same_v<V, __nv_bfloat16>) {
        return static_cast<T>(__bfloat162float(v));
    } else {
        return static_cast<T>(v);
    }
}

// Knuth's TwoSum: returns fl(a+b) and adds the exact rounding error to err.
template <typename T>
__device__ __forceinline__ T two_sum(T a, T b, T& err) {
    const T s = a + b;
    const T bp = s - a;
    err += (a - (s - bp)) + (b - bp);
    return s;
}

__device__ __forceinline__ float fma_rn(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ double fma_rn(double a, double b, double c) { return __fma_rn(a, b, c); }
__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }

// Sum accumulator; with EXT it carries a running compensation term
// (compensated dot product in the style of Ogita, Rump and Oishi, "Accurate
// sum and dot product", SIAM J. Sci. Comput. 26(6), 2005), which is the
// extended-precision mode of the reference kernels
// (src/library/kernels/csrmv_adaptive.cl:167-308).
template <typename T, bool EXT>
struct Acc {
    T s = T(0);
    T c = T(0);
    __device__ __forceinline__ void add(T v) {
        if constexpr (EXT) {
            s = two_sum(s, v, c);
        } else {
            s += v;
        }
    }
    __device__ __forceinline__ void add_prod(T a, T b) {
        if constexpr (EXT) {
            const T p = mul_rn(a, b);
            const T e = fma_rn(a, b, -p);
            s = two_sum(s, p, c);
            c += e;
        } else {
            s = fma_rn(a, b, s);
        }
    }
    __device__ __forceinline__ void merge(T os, T oc) {
        if constexpr (EXT) {
            s = two_sum(s, os, c);
            c += oc;
        } else {
            s += os;
        }
    }
    __device__ __forceinline__ T value() const {
        if constexpr (EXT) return s + c;
        return s;
    }
};

// Reduces an accumulator over aligned groups of W lanes (W a power of two
// <= 32). Every lane of the warp must call it. Lane 0 of each group ends with
// the group total.
template <int W, typename T, bool EXT>
__device__ __forceinline__ void group_reduce(Acc<T, EXT>& a) {
#pragma unroll
    for (int off = W / 2; off > 0; off >>= 1) {
        const T os = __shfl_xor_sync(0xffffffffu, a.s, off, W);
        if constexpr (EXT) {
            const T oc = __shfl_xor_sync(0xffffffffu, a.c, off, W);
            a.merge(os, oc);
        } else {
            a.s += os;
        }
    }
}

template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
    return v;
}

// Sums one value per thread over the CTA (blockDim.x a multiple of 32, at
// most 1024). The result is valid in every thread. `scratch` holds >= 32
// elements. The summation order depends only on blockDim, so it is
// reproducible.
template <typename T>
__device__ __forceinline__ T block_sum(T v, T* scratch) {
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const int nwarps = (blockDim.x + 31) >> 5;
    v = warp_sum(v);
    __syncthreads();
    if (lane == 0) scratch[warp] = v;
    __syncthreads();
    T t = (lane < nwarps) ? scratch[lane] : T(0);
    t = warp_sum(t);
    return t;
}

template <typename T, bool EXT>
__device__ __forceinline__ Acc<T, EXT> block_reduce_acc(Acc<T, EXT> a, T* scratch_s, T* scratch_c) {
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const int nwarps = (blockDim.x + 31) >> 5;
    group_reduce<32>(a);
    __syncthreads();
    if (lane == 0) {
        scratch_s[warp] = a.s;
        scratch_c[warp] = a.c;
    }
    __syncthreads();
    Acc<T, EXT> b;
    if (lane < nwarps) {
        b.s = scratch_s[lane];
        b.c = scratch_c[lane];
    }
    group_reduce<32>(b);
    return b;
}

// Deterministic grid-wide sum of K per-thread values of type U (double or
// long long). Each CTA stores its
// partial totals in partials[k * gridDim.x + blockIdx.x], then takes a ticket;
// the CTA that draws the last ticket re-reads all partials in index order and
// returns true with the totals in out[] (valid in every thread of that CTA).
// It also resets the ticket to zero for the next launch. No CTA ever waits
// for another, so there is nothing to deadlock.
// Arrival on a reduction ticket: a release-acquire atomic add at GPU scope.
// The release orders this thread's partial store before the arrival; the
// acquire lets the last arriving CTA read every other CTA's partial (its other
// threads see them after the CTA barrier that follows). Cheaper than a full
// fence before a relaxed atomic.
__device__ __forceinline__ uint32_t ticket_arrive(uint32_t* ticket) {
    uint32_t old;
    asm volatile("atom.acq_rel.gpu.global.add.u32 %0, [%1], 1;" : "=r"(old) : "l"(ticket) : "memory");
    return old;
}

template <int K, typename U = double>
__device__ __forceinline__ bool grid_reduce_last(const U (&v)[K], U* partials, uint32_t* ticket,
                                                 U (&out)[K]) {
    __shared__ U red[32];
    __shared__ bool is_last;
    U tot[K];
#pragma unroll
    for (int k = 0; k < K; ++k) tot[k] = block_sum(v[k], red);
    const uint32_t G = gridDim.x;
    if (threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < K; ++k) partials[(size_t)k * G + blockIdx.x] = tot[k];
        const uint32_t t = ticket_arrive(ticket);
        is_last = (t == G - 1);
    }
    __syncthreads();
    if (!is_last) return false;
#pragma unroll
    for (int k = 0; k < K; ++k) {
        U a = U(0);
        for (uint32_t i = threadIdx.x; i < G; i += blockDim.x) a += __ldcg(partials + (size_t)k * G + i);
        out[k] = block_sum(a, red);
    }
    if (threadIdx.x == 0) *ticket = 0u;
    return true;
}

// Two-level form of grid_reduce_last for launches of many CTAs (the SpMV
// epilogue runs one CTA per row-block word, tens of thousands): the CTAs are
// split into at most kTreeGroups contiguous groups with a counter each; the
// last CTA of a group adds the group's partials in CTA order and arrives at
// the top counter; the last group adds the group sums in order. Arrivals on
// any one counter drop from the grid size to a group's size, and the result
// is still independent of timing.
// tickets: 1 + kTreeGroups zeroed counters (left at zero); partials:
// K * (gridDim.x + kTreeGroups) slots.
constexpr uint32_t kTreeGroups = 256;

template <int K, typename U = double>
__device__ __forceinline__ bool grid_reduce_tree(const U (&v)[K], U* partials, uint32_t* tickets, U (&out)[K]) {
    __shared__ U red[32];
    __shared__ int stage;
    U tot[K];
#pragma unroll
    for (int k = 0; k < K; ++k) tot[k] = block_sum(v[k], red);
    const uint32_t G = gridDim.x;
    const uint32_t gs = (G + kTreeGroups - 1) / kTreeGroups;  // CTAs per group
    const uint32_t ngroups = (G + gs - 1) / gs;
    const uint32_t g = blockIdx.x / gs;
    const uint32_t g0 = g * gs, g1 = min(G, g0 + gs);
    U* gpart = partials + static_cast<size_t>(K) * G;
    if (threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < K; ++k) partials[(size_t)k * G + blockIdx.x] = tot[k];
        const uint32_t t = ticket_arrive(tickets + 1 + g);
        stage = (t == g1 - g0 - 1) ? 1 : 0;
    }
    __syncthreads();
    if (stage == 0) return false;
#pragma unroll
    for (int k = 0; k < K; ++k) {
        U a = U(0);
        for (uint32_t i = g0 + threadIdx.x; i < g1; i += blockDim.x) a += __ldcg(partials + (size_t)k * G + i);
        tot[k] = block_sum(a, red);
    }
    if (threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < K; ++k) gpart[(size_t)k * kTreeGroups + g] = tot[k];
        tickets[1 + g] = 0u;
        const uint32_t t = ticket_arrive(tickets);
        stage = (t == ngroups - 1) ? 2 : 0;
    }
    __syncthreads();
    if (stage != 2) return false;
#pragma unroll
    for (int k = 0; k < K; ++k) {
        U a = U(0);
        for (uint32_t i = threadIdx.x; i < ngroups; i += blockDim.x) a += __ldcg(gpart + (size_t)k * kTreeGroups + i);
        out[k] = block_sum(a, red);
    }
    if (threadIdx.x == 0) *tickets = 0u;
    return true;
}

}  // namespace dev
}  // namespace clsp
