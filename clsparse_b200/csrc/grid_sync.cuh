// Grid-wide exchanges of the persistent solver kernels (one cooperative
// launch per solve, every CTA resident): a deterministic sum of per-CTA
// partials that every CTA obtains bitwise identical, with every wait bounded
// by the global timer. Used by the CSR persistent engine (fused_cg.cu) and
// the banded inner-solve engine (dia.cu).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "device_common.cuh"
#include "fused.h"

namespace clsp {
namespace {

__device__ __forceinline__ uint64_t global_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ unsigned long long ld_relaxed(const unsigned long long* p) {
    unsigned long long v;
    asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void st_release(unsigned long long* p, unsigned long long v) {
    asm volatile("st.release.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

__device__ __forceinline__ void fence_acq_rel() { asm volatile("fence.acq_rel.gpu;" ::: "memory"); }

__device__ __forceinline__ void red_release_add(unsigned long long* p, unsigned long long v) {
    asm volatile("red.release.gpu.global.add.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

__device__ __forceinline__ unsigned long long ld_acquire(const unsigned long long* p) {
    unsigned long long v;
    asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}

struct GridSmem {
    double red[2][4][32];  // per-warp sums of a CTA's values, two buffers by epoch parity
    double fin[4][32];     // per-warp sums of the grid's partials
    int ok;
};

// Sums K values per thread over the CTA, the result in every thread: for
// each value the order of dev::block_sum (warp trees, then a tree over the
// warps' sums), with one barrier for all K values instead of two per value.
// The caller keeps `scratch` from being rewritten while a warp may still read
// it (GridSmem::red alternates by epoch; fin is rewritten only after the
// next exchange's barriers).
template <int K>
__device__ __forceinline__ void block_sum_k(const double (&v)[K], double (&out)[K], double (*scratch)[32]) {
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const int nwarps = (blockDim.x + 31) >> 5;
    double w[K];
#pragma unroll
    for (int k = 0; k < K; ++k) w[k] = dev::warp_sum(v[k]);
    if (lane == 0) {
#pragma unroll
        for (int k = 0; k < K; ++k) scratch[k][warp] = w[k];
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < K; ++k) out[k] = dev::warp_sum(lane < nwarps ? scratch[k][lane] : 0.0);
}

// Grid exchange. Every CTA stores its K partial sums for `epoch` in its slot
// (two buffers, by epoch parity) and adds one to the arrival counter with
// release semantics; thread 0 of every CTA polls the counter with acquire
// loads until all G arrivals of the epoch are in (epoch * G), so no CTA has
// to learn that it came last and release the others. Then every thread reads
// the partials of CTAs tid, tid + NT, ... and a block reduction finishes the
// sums, so every CTA obtains bitwise the same totals, whatever the arrival
// order. K = 0 is a plain barrier. A slot is rewritten two exchanges later
// at the earliest, when every CTA has finished reading it. Measured on B200
// (bare exchange, 512-thread CTAs): 2.1 us at 148 CTAs and 2.8 us at 296,
// against 3.2 / 3.5 us for a ticket with a separate release flag, and 8.2 us
// at 296 for a two-level arrival tree (more dependent round trips). The two
// CTA-wide sums take one barrier each for all K values (block_sum_k): per
// iteration C1 FP64 banded drop-in 11.41 -> 10.99 us, C5 learned inner
// 21.00 -> 20.83 us, the same totals bit for bit.
// Returns false (in every thread) when the grid has to stop: the wait ran out
// (the error flag is then set) or another CTA reported that it did. Under
// the never-release test switch CTA 0 does not count itself, so every wait
// runs out.
template <int K>
__device__ bool grid_exchange(const FusedSync& g, unsigned long long& epoch, const double (&v)[K > 0 ? K : 1],
                              double (&out)[K > 0 ? K : 1], GridSmem& gs) {
    double tot[K > 0 ? K : 1];
    if constexpr (K > 0) {
        block_sum_k<K>(v, tot, gs.red[(epoch + 1) & 1ull]);
    } else {
        __syncthreads();
    }
    ++epoch;
    const uint32_t G = gridDim.x;
    const double* part = g.partials + (epoch & 1ull) * static_cast<size_t>(G) * 4;
    if (threadIdx.x == 0) {
        if constexpr (K > 0) {
            double* mine = g.partials + (epoch & 1ull) * static_cast<size_t>(G) * 4 + static_cast<size_t>(blockIdx.x) * 4;
#pragma unroll
            for (int k = 0; k < K; ++k) mine[k] = tot[k];
        }
        red_release_add(g.arrive, (g.never_release && blockIdx.x == 0) ? 0ull : 1ull);
        const unsigned long long target = epoch * G;
        bool ok = true;
        uint64_t t0 = 0;
        uint32_t spins = 0;
        while (ld_acquire(g.arrive) < target) {
            if ((++spins & 255u) == 0u) {
                if (*reinterpret_cast<volatile int*>(g.err)) {
                    ok = false;
                    break;
                }
                const uint64_t now = global_ns();
                if (t0 == 0) {
                    t0 = now;
                } else if (now - t0 > g.wait_ns) {
                    atomicExch(g.err, 1);
                    ok = false;
                    break;
                }
            }
        }
        gs.ok = ok ? 1 : 0;
    }
    __syncthreads();
    if (!gs.ok) return false;
    if constexpr (K > 0) {
        double acc[K];
#pragma unroll
        for (int k = 0; k < K; ++k) acc[k] = 0.0;
        for (uint32_t i = threadIdx.x; i < G; i += blockDim.x)
#pragma unroll
            for (int k = 0; k < K; ++k) acc[k] += __ldcg(part + static_cast<size_t>(i) * 4 + k);
        block_sum_k<K>(acc, out, gs.fin);
    }
    return true;
}

__device__ __forceinline__ bool grid_sync(const FusedSync& g, unsigned long long& epoch, GridSmem& gs) {
    double none[1] = {0.0}, out[1];
    return grid_exchange<0>(g, epoch, none, out, gs);
}

}  // namespace
}  // namespace clsp
