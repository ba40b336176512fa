// Device-wide in-place inclusive scan of 32-bit counts, in three phases:
// per-block scans of 1024 elements (each thread rewrites only its own
// element) with block totals, an exclusive scan of the block totals by one
// CTA, and the carries added back. Used to turn per-row counts into CSR row
// pointers (format conversions, the learned preconditioner's graph).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace clsp {
namespace scan {
namespace {

__global__ void scan_blocks_kernel(uint32_t* __restrict__ v, uint32_t n, uint32_t* __restrict__ part) {
    __shared__ uint32_t s[1024];
    const uint32_t i = blockIdx.x * 1024u + threadIdx.x;
    s[threadIdx.x] = i < n ? v[i] : 0u;
    __syncthreads();
    for (uint32_t off = 1; off < 1024; off <<= 1) {
        const uint32_t t = threadIdx.x >= off ? s[threadIdx.x - off] : 0u;
        __syncthreads();
        s[threadIdx.x] += t;
        __syncthreads();
    }
    if (i < n) v[i] = s[threadIdx.x];
    if (threadIdx.x == 1023) part[blockIdx.x] = s[1023];
}

__global__ void scan_parts_kernel(uint32_t* __restrict__ part, uint32_t nparts) {
    __shared__ uint32_t s[1024];
    uint32_t carry = 0;
    for (uint32_t b = 0; b < nparts; b += 1024) {
        const uint32_t i = b + threadIdx.x;
        const uint32_t x = i < nparts ? part[i] : 0u;
        s[threadIdx.x] = x;
        __syncthreads();
        for (uint32_t off = 1; off < 1024; off <<= 1) {
            const uint32_t t = threadIdx.x >= off ? s[threadIdx.x - off] : 0u;
            __syncthreads();
            s[threadIdx.x] += t;
            __syncthreads();
        }
        if (i < nparts) part[i] = carry + s[threadIdx.x] - x;
        carry += s[1023];
        __syncthreads();
    }
}

__global__ void scan_add_kernel(uint32_t* __restrict__ v, uint32_t n, const uint32_t* __restrict__ part) {
    const uint32_t i = blockIdx.x * 1024u + threadIdx.x;
    if (i < n) v[i] += part[blockIdx.x];
}

// Scans v[0..n) in place (inclusive); part holds ceil(n / 1024) words.
inline void inclusive_u32(uint32_t* v, uint32_t n, uint32_t* part, cudaStream_t s) {
    if (n == 0) return;
    const uint32_t nparts = (n + 1023) / 1024;
    scan_blocks_kernel<<<nparts, 1024, 0, s>>>(v, n, part);
    scan_parts_kernel<<<1, 1024, 0, s>>>(part, nparts);
    scan_add_kernel<<<nparts, 1024, 0, s>>>(v, n, part);
}

inline uint32_t parts_for(uint32_t n) { return (n + 1023) / 1024; }

}  // namespace
}  // namespace scan
}  // namespace clsp
