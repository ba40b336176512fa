// Banded inner solves of the mixed-precision refinement (project extension,
// no reference counterpart; the reference's CG loop it replaces for these
// matrices is src/library/solvers/conjugate-gradients.hpp:162-226).
//
// Storage. Stencil and banded matrices -- the 5- and 7-point operators of
// the configured workloads and the learned factor G on tril(A) of them --
// have a handful of distinct column offsets j - i. The refinement already
// solves its inner systems on a private low-precision copy of A's values;
// when A has at most kMaxDiags distinct offsets (and fills at least half of
// those diagonals), that copy is laid out by diagonal instead of in CSR:
// values [d][i] for the d-th offset in increasing order, zero where the
// diagonal leaves the matrix, and no column indices or row pointers (DIA
// storage; N. Bell and M. Garland, SC'09). On the 1024^2 five-point matrix
// this is 21 MB of FP32 values against 46 MB for FP32 CSR; G and G^T (three
// diagonals, BF16) are 6.3 MB each. The whole inner iteration's working set
// then fits in the 126 MB L2.
//
// Engine. One cooperative launch per inner solve; every CTA owns a
// contiguous slice of rows and every thread a strided set of them. Grid
// exchanges (grid_sync.cuh) carry the dot products, so every CTA computes
// bitwise the same alpha, beta and stop decision. Vectors written inside the
// launch and read at neighbouring rows by other CTAs are double-buffered
// (p, and r for the learned factor) so that a phase can form a neighbour's
// new value itself instead of waiting for it:
//
//   Jacobi / none (2 exchanges per iteration)
//     A: p_new = z + beta p_old, q = A p_new (neighbours' p_new formed on the
//        fly), <p_new, q>                                  -> exchange: alpha
//     B: x += alpha p_new, r -= alpha q, z = D^-1 r, <r,r>, <r,z>
//                                                   -> exchange: stop, beta
//   learned M^-1 = G^T G (2 exchanges per iteration)
//     A: as above                                          -> exchange: alpha
//     B: x += alpha p_new, r_new = r - alpha q into the other r buffer,
//        z = G^T (G r_new) with the neighbours' (G r_new)_j and their r_new
//        formed on the fly, <r_new, r_new>, ||G r_new||^2 = <r_new, z>
//                                                   -> exchange: stop, beta
//
// Arithmetic: values and vectors FP32 (BF16 values widened), FMA
// accumulation in FP32 in increasing column order, dot products accumulated
// in FP64 -- the precision contract of the CSR inner solves. The stop test
// is the inner solve's: ||r|| <= tol ||r_0|| (L2, recursive residual), or
// maxIters. A continued solve (residual replacement) starts from x = 0 and
// r = b and keeps the previous solve's last direction:
// p = z + (<r,z> / rz_prev) p_prev.
//
// Drop-in solves (solver loop mode 3): clsparse{S,D}csrcg and
// clsparse{S,D}csrbicgStab on a banded matrix run as one cooperative launch
// over a diagonal-storage copy in the solve's own type, in the reference's
// arithmetic (rows in its CSR-Adaptive order, separately rounded operations),
// with its stop tests and solver-control bookkeeping (dia_cg_ref_kernel,
// dia_bicg_ref_kernel below).
//
// Safety: every barrier wait is bounded (grid_sync.cuh); a timeout leaves
// the kernel through every CTA and is reported as the barrier-timeout status.
#include <algorithm>
#include <climits>
#include <cstdlib>
#include <cstring>
#include <limits>
#include <type_traits>
#include <vector>

#include "device_common.cuh"
#include "dia.h"
#include "fused.h"
#include "grid_sync.cuh"
#include "internal.h"
#include "solver_state.cuh"

namespace clsp {
namespace {

constexpr int kSlots = 64;  // hash set of offsets (power of two, > kMaxDiags)
// empty slot: every byte 0x80 (what cudaMemsetAsync writes), below any
// offset j - i a matrix of fewer than 2^31 rows has
constexpr int32_t kEmpty = static_cast<int32_t>(0x80808080u);
// Threads per CTA of the persistent kernel: one CTA per SM at 1024 (measured
// on C5: 22.5 us per learned inner iteration vs 23.1 with two 512-thread CTAs).
#ifndef CLSP_DIA_THREADS
#define CLSP_DIA_THREADS 1024
#endif
constexpr int kDiaThreads = CLSP_DIA_THREADS;
// CTAs per SM (their registers capped to fit): more resident threads with
// fewer registers measured slower -- C5 learned inner iteration 24.7 us at
// 3 x 512 and 33.2 us at 6 x 256 against 21.2 us at 1 x 1024 (spills, and
// more CTAs in every grid exchange).
#ifndef CLSP_DIA_CTAS
#define CLSP_DIA_CTAS (1024 / CLSP_DIA_THREADS)
#endif
constexpr int kDiaCtasPerSm = CLSP_DIA_CTAS;

__device__ __forceinline__ uint32_t slot_of(int32_t o) { return (static_cast<uint32_t>(o) * 2654435761u) >> 26; }

// Inserts o into an open-addressed set of kSlots entries; false when full.
// A plain read finds offsets already present without an atomic.
__device__ bool set_insert(int32_t* table, int32_t o) {
    uint32_t h = slot_of(o);
    for (int probe = 0; probe < kSlots; ++probe) {
        const int32_t cur = *reinterpret_cast<volatile int32_t*>(table + h);
        if (cur == o) return true;
        if (cur == kEmpty) {
            const int32_t old = atomicCAS(table + h, kEmpty, o);
            if (old == kEmpty || old == o) return true;
        }
        h = (h + 1) & (kSlots - 1);
    }
    return false;
}

// The distinct offsets cols[k] - i of a CSR matrix into `table` (kSlots
// entries preset to kEmpty); flags[0] |= 1 when there are more than the set
// holds, |= 2 when a row's columns are not strictly increasing.
__global__ void dia_offsets_kernel(const uint32_t* __restrict__ rp, const uint32_t* __restrict__ cols, uint32_t n,
                                   int32_t* table, int* flags) {
    __shared__ int32_t st[kSlots];
    for (int s = threadIdx.x; s < kSlots; s += blockDim.x) st[s] = kEmpty;
    __syncthreads();
    int bad = 0;
    int32_t last[4] = {kEmpty, kEmpty, kEmpty, kEmpty};  // offsets this thread inserted lately
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t b = rp[i], e = rp[i + 1];
        for (uint32_t k = b; k < e; ++k) {
            const uint32_t c = cols[k];
            if (k > b && c <= cols[k - 1]) bad |= 2;
            const int32_t o = static_cast<int32_t>(static_cast<int64_t>(c) - static_cast<int64_t>(i));
            if (o == last[0] || o == last[1] || o == last[2] || o == last[3]) continue;
            if (!set_insert(st, o)) bad |= 1;
            last[3] = last[2];
            last[2] = last[1];
            last[1] = last[0];
            last[0] = o;
        }
    }
    __syncthreads();
    for (int s = threadIdx.x; s < kSlots; s += blockDim.x)
        if (st[s] != kEmpty && !set_insert(table, st[s])) bad |= 1;
    if (bad) atomicOr(flags, bad);
}

__device__ __forceinline__ float widen(float v) { return v; }
__device__ __forceinline__ float widen(__nv_bfloat16 v) { return __bfloat162float(v); }
__device__ __forceinline__ float widen(double v) { return static_cast<float>(v); }

template <typename VO>
__device__ __forceinline__ VO narrow(double v) {
    if constexpr (std::is_same_v<VO, __nv_bfloat16>)
        return __double2bfloat16(v);
    else
        return static_cast<VO>(v);
}
template <typename VO>
__device__ __forceinline__ VO narrow(__nv_bfloat16 v) {
    if constexpr (std::is_same_v<VO, __nv_bfloat16>)
        return v;
    else
        return static_cast<VO>(__bfloat162float(v));
}
template <typename VO>
__device__ __forceinline__ VO narrow(float v) {
    if constexpr (std::is_same_v<VO, __nv_bfloat16>)
        return __float2bfloat16(v);
    else
        return static_cast<VO>(v);
}

// out[d * n + i] = vals of entry (i, i + off[d]), rounded to VO (out zeroed
// before); the offsets are sorted, so the diagonal is found by a short scan.
template <typename VI, typename VO>
__global__ void dia_fill_kernel(const uint32_t* __restrict__ rp, const uint32_t* __restrict__ cols,
                                const VI* __restrict__ vals, uint32_t n, DiaOffsets offs, VO* __restrict__ out) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t b = rp[i], e = rp[i + 1];
        int d = 0;
        for (uint32_t k = b; k < e; ++k) {
            const int32_t o = static_cast<int32_t>(static_cast<int64_t>(cols[k]) - static_cast<int64_t>(i));
            while (d < offs.nd && offs.off[d] < o) ++d;  // columns increase, so d only moves forward
            if (d < offs.nd && offs.off[d] == o) out[static_cast<size_t>(d) * n + i] = narrow<VO>(vals[k]);
        }
    }
}

// diag32[i] = a_ii + sum_{j != i} (a_ij - round_V(a_ij)) (FP64 sum, FP32
// result); the main diagonal of the V copy (index d0) set to zero.
template <typename V>
__global__ void dia_comp_diag_kernel(const uint32_t* __restrict__ rp, const uint32_t* __restrict__ cols,
                                     const double* __restrict__ vals, uint32_t n, V* __restrict__ main_diag,
                                     float* __restrict__ diag32) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double d = 0.0;
        for (uint32_t k = rp[i]; k < rp[i + 1]; ++k) {
            const double a = vals[k];
            d += cols[k] == i ? a : a - static_cast<double>(widen(narrow<V>(a)));
        }
        diag32[i] = static_cast<float>(d);
        main_diag[i] = narrow<V>(0.0);
    }
}

// invD[i] = 1 / a_ii from the main diagonal of a DIA matrix; status |=
// kStatusZeroDiag where it is zero.
template <typename V>
__global__ void dia_inv_diag_kernel(const V* __restrict__ diag, uint32_t n, float* __restrict__ invD, int* status) {
    bool zero = false;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float v = widen(diag[i]);
        invD[i] = 1.f / v;
        zero |= (v == 0.f);
    }
    if (zero) atomicOr(status, kStatusZeroDiag);
}

// ---- the fused inner PCG

// The rows a CTA owns in every phase: a static contiguous slice, each thread
// a strided set of it. (Handing rows out in chunks from a per-phase counter,
// so that faster CTAs take more, measured slower on B200: C5 learned inner
// iteration 31.9 vs 27.6 us -- the per-chunk barrier and the dependent chunk
// fetch cost more than the wait for the slowest slice at the exchange.)
template <typename F>
__device__ __forceinline__ void for_rows(uint32_t n, F body) {
    const uint64_t c = blockIdx.x, G = gridDim.x;
    const uint32_t r0 = static_cast<uint32_t>(c * n / G), r1 = static_cast<uint32_t>((c + 1) * n / G);
    for (uint32_t i = r0 + threadIdx.x; i < r1; i += kDiaThreads) body(i);
}

// Rows per thread and pass in the Jacobi iteration's phases: 2 walks the
// slice two rows at a time (row i and i + kDiaThreads), all loads of both
// before any store, so a thread keeps two rows' loads in flight. Measured
// per inner iteration: C3 (2.1M rows, FP32) 46.4 -> 37.9 us, C5 (1M rows)
// 17.6 -> 16.3 us; the learned iteration keeps one row per pass (23.0 vs
// 23.5 us with two).
#ifndef CLSP_DIA_U
#define CLSP_DIA_U 2
#endif
// 1: the learned iteration's t = G r pass walks two rows per pass, both
// rows' loads before any global store (C5 learned inner iteration 19.6 ->
// 19.2 us, the same iterates)
#ifndef CLSP_DIA_T_PAIRS
#define CLSP_DIA_T_PAIRS 1
#endif

// Pairs of a CTA's rows: body(i0, i1, has1) with i1 = i0 + kDiaThreads when
// has1 (else i1 = i0, the second row's stores to be skipped).
template <typename F>
__device__ __forceinline__ void for_row_pairs(uint32_t n, F body) {
    const uint64_t c = blockIdx.x, G = gridDim.x;
    const uint32_t r0 = static_cast<uint32_t>(c * n / G), r1 = static_cast<uint32_t>((c + 1) * n / G);
    for (uint32_t i = r0 + threadIdx.x; i < r1; i += 2 * kDiaThreads) {
        const bool has1 = i + kDiaThreads < r1;
        body(i, has1 ? i + kDiaThreads : i, has1);
    }
}

// sum_d M[d][i] * xf(i + off[d]) over the ND diagonals (ND the matrix's
// padded diagonal count), in increasing column order, FP32 FMAs. Every load
// is unconditional -- indices outside the matrix are clamped and their
// product replaced by zero with a select -- so all of a row's loads issue
// before its first FMA waits on one.
// CLAMP false: the caller guarantees that every column i + off[d] lies
// inside the matrix (a CTA whose whole row range is interior), so the row
// needs no clamping or selects -- fewer instructions ahead of its loads
// (C5 learned inner iteration 20.7 -> 19.7 us, Jacobi 15.9 -> 15.6 us, the
// same iterates bit for bit; the drop-in kernels measured no gain from it).
template <int ND, typename V, typename XF, bool CLAMP = true>
__device__ __forceinline__ float dia_row(const DiaMat<V>& M, uint32_t n, uint32_t i, XF xf,
                                         std::integral_constant<bool, CLAMP> = {}) {
    float av[ND], xv[ND];
#pragma unroll
    for (int d = 0; d < ND; ++d) {
        av[d] = widen(__ldg(M.vals + static_cast<size_t>(d) * n + i));
        if constexpr (CLAMP) {
            const int64_t j = static_cast<int64_t>(i) + M.off[d];
            const bool in = j >= 0 && j < static_cast<int64_t>(n);
            const uint32_t jc = in ? static_cast<uint32_t>(j) : i;
            const float v = xf(jc);
            xv[d] = in ? v : 0.f;
        } else {
            xv[d] = xf(i + static_cast<uint32_t>(M.off[d]));
        }
    }
    float s = 0.f;
#pragma unroll
    for (int d = 0; d < ND; ++d) s = fmaf(av[d], xv[d], s);
    if (M.diag32 != nullptr) s = fmaf(__ldg(M.diag32 + i), xf(i), s);
    return s;
}

// z_i = sum_e GT[e][i] t_{i + off_T[e]} for the learned factor, with the
// t_j = (G r)_j of the neighbouring rows formed on the fly from rf (so no
// grid barrier separates t = G r from z = G^T t); ti gets t_i itself (the
// term of G^T's main diagonal, index gt_diag), whose square sums to
// <r, G^T G r> = ||G r||^2.
template <int NDG, typename VG, typename RF>
__device__ __forceinline__ float zt_row(const DiaMat<VG>& G, const DiaMat<VG>& GT, int gt_diag, uint32_t n,
                                        uint32_t i, RF rf, float& ti) {
    float z = 0.f;
    ti = 0.f;
#pragma unroll
    for (int e = 0; e < NDG; ++e) {
        const int64_t j = static_cast<int64_t>(i) + GT.off[e];
        const bool in = j >= 0 && j < static_cast<int64_t>(n);
        const uint32_t jc = in ? static_cast<uint32_t>(j) : i;
        const float gv = widen(__ldg(GT.vals + static_cast<size_t>(e) * n + i));
        const float tj = in ? dia_row<NDG>(G, n, jc, rf) : 0.f;
        z = fmaf(gv, tj, z);
        ti = (e == gt_diag) ? tj : ti;
    }
    return z;
}

// Learned iteration: 1 = three phases (B forms t = G r_new and stores it, C
// forms z = G^T t and ends with a plain barrier), 0 = two phases (B forms z
// with the neighbours' t_j recomputed).
#ifndef CLSP_DIA_SPLIT
#define CLSP_DIA_SPLIT 1
#endif

// Loads of vectors other CTAs wrote earlier in the same launch. The grid
// exchange between two phases orders them (release by the writers, acquire
// by thread 0 of the reader's CTA, then the CTA barrier), so plain weak
// loads observe the new values (CLSP_DIA_LDCG 2, which also leaves the
// compiler free to batch them); 1: L2-only loads, 0: weak loads through
// inline PTX.
#ifndef CLSP_DIA_LDCG
#define CLSP_DIA_LDCG 2
#endif
__device__ __forceinline__ float vld(const float* p) {
#if CLSP_DIA_LDCG == 2
    return *p;
#elif CLSP_DIA_LDCG == 1
    return __ldcg(p);
#else
    return dev::ld_coherent(p);
#endif
}

// Whether rows [lo, hi) of M keep every column i + off[d] inside the matrix.
template <typename V>
__device__ __forceinline__ bool interior_rows(const DiaMat<V>& M, uint32_t n, uint32_t lo, uint32_t hi) {
    if (hi <= lo) return false;
    int32_t mn = 0, mx = 0;
    for (int d = 0; d < M.nd; ++d) {
        mn = min(mn, M.off[d]);
        mx = max(mx, M.off[d]);
    }
    return static_cast<int64_t>(lo) + mn >= 0 && static_cast<int64_t>(hi) - 1 + mx < static_cast<int64_t>(n);
}

template <typename VA, typename VG, int PK, int NDA, int NDG>
__global__ void __launch_bounds__(kDiaThreads, kDiaCtasPerSm) dia_pcg_kernel(DiaPcgArgs<VA, VG> a) {
    __shared__ GridSmem gs;
    const FusedSync g = a.sync;
    unsigned long long epoch = 0;
    const uint32_t n = a.n;
    const uint32_t tid = threadIdx.x;
    // CTAs whose rows keep every neighbour inside the matrix skip the clamps:
    // A over the CTA's slice, G over the slice and G^T's halo after it, G^T
    // over the slice
    const uint32_t sr0 = static_cast<uint32_t>(static_cast<uint64_t>(blockIdx.x) * n / gridDim.x);
    const uint32_t sr1 = static_cast<uint32_t>((static_cast<uint64_t>(blockIdx.x) + 1) * n / gridDim.x);
    const uint32_t shi = static_cast<uint32_t>(std::min<uint64_t>(n, static_cast<uint64_t>(sr1) + a.gt_halo));
    const bool int_a = interior_rows(a.A, n, sr0, sr1);
    const bool int_g = PK == 2 && interior_rows(a.G, n, sr0, shi);
    const bool int_gt = PK == 2 && interior_rows(a.GT, n, sr0, sr1);
    // No __restrict__: these vectors are read at neighbouring rows by other CTAs.
    float* x = a.x;
    float* q = a.q;
    float* t = a.t;
    float* z = a.z;
    const float* b = a.b;
    const float* invD = a.invD;
    const DiaPcgState in = *a.st;
    const double tol2 = in.tol * in.tol;
    int pold = in.pbuf & 1;
    int cur = 0;
    bool use_p = in.warm != 0;
    double rz = 0.0, rr0 = 0.0, rr = 0.0;
    float beta = 0.f;
    int iters = 0, status = 0;

    // ---- r = b, x = 0, z = M r, <r,z>, <r,r>
    {
        double acc[2] = {0.0, 0.0};
        if constexpr (PK >= 1) {
            for_rows(n, [&](uint32_t i) {
                float ti;
                const float zi =
                    zt_row<NDG>(a.G, a.GT, a.gt_diag, n, i, [&](uint32_t k) { return __ldg(b + k); }, ti);
                const float ri = __ldg(b + i);
                a.r[0][i] = ri;
                x[i] = 0.f;
                z[i] = zi;
                acc[0] += static_cast<double>(ti) * ti;  // <r, G^T G r> = ||G r||^2
                acc[1] += static_cast<double>(ri) * ri;
            });
        } else {
            for_rows(n, [&](uint32_t i) {
                const float ri = __ldg(b + i);
                a.r[0][i] = ri;
                x[i] = 0.f;
                const float zi = invD ? ri * __ldg(invD + i) : ri;
                z[i] = zi;
                acc[0] += static_cast<double>(ri) * zi;
                acc[1] += static_cast<double>(ri) * ri;
            });
        }
        double tot[2];
        if (!grid_exchange<2>(g, epoch, acc, tot, gs)) goto fail;
        rz = tot[0];
        rr0 = rr = tot[1];
    }
    if (!(rr0 > 0.0) || in.max_iters <= 0) goto finish;  // b == 0: x = 0
    if (use_p) beta = static_cast<float>(rz / in.rz_prev);

    for (;;) {
        const int pn = pold ^ 1;
        float* P = a.p[pn];
        const float* Po = a.p[pold];
        // ---- A: p_new = z + beta p_old, q = A p_new, <p_new, q>
        {
            double acc[1] = {0.0};
            auto pv = [&](uint32_t j) {
                const float zj = vld(z + j);
                return use_p ? fmaf(beta, vld(Po + j), zj) : zj;
            };
            auto phase_a = [&](auto clamp) {
                // (BF16 values with the FP32 diagonal need more registers: one row per pass)
                if constexpr (CLSP_DIA_U == 2 && PK == 0 && std::is_same_v<VA, float>) {
                    for_row_pairs(n, [&](uint32_t i0, uint32_t i1, bool has1) {
                        const float q0 = dia_row<NDA>(a.A, n, i0, pv, clamp);
                        const float p0 = pv(i0);
                        const float q1 = dia_row<NDA>(a.A, n, i1, pv, clamp);
                        const float p1 = pv(i1);
                        P[i0] = p0;
                        q[i0] = q0;
                        acc[0] += static_cast<double>(p0) * q0;
                        if (has1) {
                            P[i1] = p1;
                            q[i1] = q1;
                            acc[0] += static_cast<double>(p1) * q1;
                        }
                    });
                } else {
                    for_rows(n, [&](uint32_t i) {
                        const float qi = dia_row<NDA>(a.A, n, i, pv, clamp);
                        const float pi = pv(i);
                        P[i] = pi;
                        q[i] = qi;
                        acc[0] += static_cast<double>(pi) * qi;
                    });
                }
            };
            // (the unclamped form of the two-rows pass with seven or more
            // diagonals spills: 128^3 FP32 inner iteration 38.2 -> 41.0 us)
            if constexpr (PK == 2 || NDA <= 5) {
                if (int_a)
                    phase_a(std::false_type{});
                else
                    phase_a(std::true_type{});
            } else {
                phase_a(std::true_type{});
            }
            double pq[1];
            if (!grid_exchange<1>(g, epoch, acc, pq, gs)) goto fail;
            if (!(pq[0] > 0.0)) {  // lost positive curvature (or not finite): stop, the caller restarts
                status |= isfinite(pq[0]) ? kStatusCurvature : kStatusNonFinite;
                break;
            }
            const float alpha = static_cast<float>(rz / pq[0]);
            // ---- B
            if constexpr (PK == 2) {
                // t = G r_new for this CTA's rows and the gt_halo rows after
                // them, into shared memory (t_j needs only q and r, complete
                // since A's exchange), then z = G^T t from there: G^T's
                // offsets are >= 0, so no other CTA's t is needed and one
                // grid exchange per iteration goes away
                extern __shared__ float ts[];
                const uint64_t c = blockIdx.x, G = gridDim.x;
                const uint32_t r0 = static_cast<uint32_t>(c * n / G), r1 = static_cast<uint32_t>((c + 1) * n / G);
                const uint32_t hi = static_cast<uint32_t>(
                    std::min<uint64_t>(n, static_cast<uint64_t>(r1) + a.gt_halo));
                const float* Rc = a.r[cur];
                float* Rn = a.r[cur ^ 1];
                double acc2[2] = {0.0, 0.0};
                auto rnew = [&](uint32_t k) { return fmaf(-alpha, vld(q + k), vld(Rc + k)); };
                auto phase_t = [&](auto clamp) {
#if CLSP_DIA_T_PAIRS
                    // two rows per pass, both rows' loads before any global
                    // store (a store holds back every later load)
                    for (uint32_t i = r0 + tid; i < hi; i += 2 * kDiaThreads) {
                        const uint32_t i1 = i + kDiaThreads;
                        const bool has1 = i1 < hi;
                        const uint32_t ib = has1 ? i1 : i;
                        const float t0 = dia_row<NDG>(a.G, n, i, rnew, clamp);
                        const float t1 = dia_row<NDG>(a.G, n, ib, rnew, clamp);
                        const bool own0 = i < r1, own1 = has1 && i1 < r1;
                        const uint32_t o0 = own0 ? i : r0, o1 = own1 ? i1 : r0;
                        const float xn0 = fmaf(alpha, P[o0], x[o0]);
                        const float rn0 = fmaf(-alpha, q[o0], Rc[o0]);
                        const float xn1 = fmaf(alpha, P[o1], x[o1]);
                        const float rn1 = fmaf(-alpha, q[o1], Rc[o1]);
                        ts[i - r0] = t0;
                        if (has1) ts[i1 - r0] = t1;
                        if (own0) {
                            x[i] = xn0;
                            Rn[i] = rn0;
                            acc2[0] += static_cast<double>(rn0) * rn0;
                            acc2[1] += static_cast<double>(t0) * t0;
                        }
                        if (own1) {
                            x[i1] = xn1;
                            Rn[i1] = rn1;
                            acc2[0] += static_cast<double>(rn1) * rn1;
                            acc2[1] += static_cast<double>(t1) * t1;
                        }
                    }
#else
                    for (uint32_t i = r0 + tid; i < hi; i += kDiaThreads) {
                        const float ti = dia_row<NDG>(a.G, n, i, rnew, clamp);
                        ts[i - r0] = ti;
                        if (i < r1) {
                            // the row's loads before its stores (x, r, q are not
                            // __restrict__: a store would hold back later loads)
                            const float xn = fmaf(alpha, P[i], x[i]);
                            const float rn = fmaf(-alpha, q[i], Rc[i]);
                            x[i] = xn;
                            Rn[i] = rn;
                            acc2[0] += static_cast<double>(rn) * rn;
                            acc2[1] += static_cast<double>(ti) * ti;
                        }
                    }
#endif
                };
                if (int_g)
                    phase_t(std::false_type{});
                else
                    phase_t(std::true_type{});
                __syncthreads();
                auto tl = [&](uint32_t k) { return ts[k - r0]; };
                if (int_gt) {
                    for (uint32_t i = r0 + tid; i < r1; i += kDiaThreads)
                        z[i] = dia_row<NDG>(a.GT, n, i, tl, std::false_type{});
                } else {
                    for (uint32_t i = r0 + tid; i < r1; i += kDiaThreads) z[i] = dia_row<NDG>(a.GT, n, i, tl);
                }
                double tot[2];
                if (!grid_exchange<2>(g, epoch, acc2, tot, gs)) goto fail;
                rr = tot[0];
                cur ^= 1;
                ++iters;
                pold = pn;
                use_p = true;
                if (!isfinite(rr)) {
                    status |= kStatusNonFinite;
                    break;
                }
                if (rr <= tol2 * rr0 || iters >= in.max_iters) break;
                beta = static_cast<float>(tot[1] / rz);
                rz = tot[1];
                continue;
            } else if constexpr (PK == 1) {
                const float* Rc = a.r[cur];
                float* Rn = a.r[cur ^ 1];
                double acc2[2] = {0.0, 0.0};
                auto rnew = [&](uint32_t k) { return fmaf(-alpha, vld(q + k), vld(Rc + k)); };
                for_rows(n, [&](uint32_t i) {
                    float ti;
#if CLSP_DIA_SPLIT
                    ti = dia_row<NDG>(a.G, n, i, rnew);
                    t[i] = ti;
#else
                    const float zi = zt_row<NDG>(a.G, a.GT, a.gt_diag, n, i, rnew, ti);
                    z[i] = zi;
#endif
                    x[i] = fmaf(alpha, P[i], x[i]);
                    const float rn = fmaf(-alpha, q[i], Rc[i]);
                    Rn[i] = rn;
                    acc2[0] += static_cast<double>(rn) * rn;
                    acc2[1] += static_cast<double>(ti) * ti;
                });
                double tot[2];
                if (!grid_exchange<2>(g, epoch, acc2, tot, gs)) goto fail;
                rr = tot[0];
                cur ^= 1;
                ++iters;
                pold = pn;
                use_p = true;
                if (!isfinite(rr)) {
                    status |= kStatusNonFinite;
                    break;
                }
                if (rr <= tol2 * rr0 || iters >= in.max_iters) break;
                beta = static_cast<float>(tot[1] / rz);
                rz = tot[1];
#if CLSP_DIA_SPLIT
                // C: z = G^T t; a plain barrier, <r, z> = ||t||^2 came with B's exchange
                for_rows(n, [&](uint32_t i) { z[i] = dia_row<NDG>(a.GT, n, i, [&](uint32_t k) { return vld(t + k); }); });
                if (!grid_sync(g, epoch, gs)) goto fail;
#endif
                continue;
            } else {
                float* R = a.r[0];
                double acc2[2] = {0.0, 0.0};
#if CLSP_DIA_U == 2
                for_row_pairs(n, [&](uint32_t i0, uint32_t i1, bool has1) {
                    const float x0 = fmaf(alpha, P[i0], x[i0]), x1 = fmaf(alpha, P[i1], x[i1]);
                    const float r0v = fmaf(-alpha, q[i0], R[i0]), r1v = fmaf(-alpha, q[i1], R[i1]);
                    const float z0 = invD ? r0v * __ldg(invD + i0) : r0v;
                    const float z1 = invD ? r1v * __ldg(invD + i1) : r1v;
                    x[i0] = x0;
                    R[i0] = r0v;
                    z[i0] = z0;
                    acc2[0] += static_cast<double>(r0v) * r0v;
                    acc2[1] += static_cast<double>(r0v) * z0;
                    if (has1) {
                        x[i1] = x1;
                        R[i1] = r1v;
                        z[i1] = z1;
                        acc2[0] += static_cast<double>(r1v) * r1v;
                        acc2[1] += static_cast<double>(r1v) * z1;
                    }
                });
#else
                for_rows(n, [&](uint32_t i) {
                    x[i] = fmaf(alpha, P[i], x[i]);
                    const float ri = fmaf(-alpha, q[i], R[i]);
                    R[i] = ri;
                    const float zi = invD ? ri * __ldg(invD + i) : ri;
                    z[i] = zi;
                    acc2[0] += static_cast<double>(ri) * ri;
                    acc2[1] += static_cast<double>(ri) * zi;
                });
#endif
                double tot[2];
                if (!grid_exchange<2>(g, epoch, acc2, tot, gs)) goto fail;
                rr = tot[0];
                ++iters;
                pold = pn;
                use_p = true;
                if (!isfinite(rr)) {
                    status |= kStatusNonFinite;
                    break;
                }
                if (rr <= tol2 * rr0 || iters >= in.max_iters) break;
                beta = static_cast<float>(tot[1] / rz);
                rz = tot[1];
                continue;
            }
        }
    }
finish:
    if (blockIdx.x == 0 && tid == 0) {
        a.st->iters = iters;
        a.st->rr0 = rr0;
        a.st->rr = rr;
        a.st->rz_prev = rz;  // the denominator that formed the last direction
        a.st->pbuf = pold;   // the buffer holding it
        a.st->xbuf = cur;    // the buffer holding the last residual
        atomicOr(&a.st->status, status);
    }
    return;
fail:
    if (tid == 0) atomicOr(&a.st->status, kStatusBarrierTimeout);
}

// ---- the drop-in CG (clsparse{S,D}csrcg, solver loop mode 3)

// In/out block of one drop-in solve.
struct DiaCgState {
    // in: the solver control
    double rel_tol = 0.0, abs_tol = 0.0;
    int max_iters = 0;
    int n_iters_in = 0;  // nIters the control held before the solve (the first stop test sees it)
    int l2 = 0;          // 0: ||.||_1 stop test as the reference, 1: ||.||_2
    int stop_nonfinite = 0;
    // out
    int n_iters = 0;
    int zero_b = 0;      // ||b|| == 0: x = b, nothing else done
    int zero_diag = 0;   // Jacobi with a zero on the main diagonal: nothing written to x
    int status = 0;      // kStatusCurvature / kStatusNonFinite / kStatusBarrierTimeout
    double init_res = 0.0, cur_res = 0.0;
};

// Rows [r0, r1) whose CSR-Adaptive block reduces a row over g > 1 lanes.
struct LaneRange {
    uint32_t r0, r1, g;
};
constexpr int kMaxLaneRanges = 8;

template <typename T>
struct DiaCgArgs {
    using value_type = T;
    DiaMat<T> A;
    // CSR arrays of A, for the rows of lane ranges
    const uint32_t* rp;
    const uint32_t* cols;
    const T* vals;
    LaneRange lanes[kMaxLaneRanges];
    int nlanes;
    // A symmetric bit for bit with its offsets symmetric and no padding
    // diagonals (the kernel's SYM form): the value of lower diagonal d at row
    // i is read as A[j][i] from its upper partner ND - 1 - d at row
    // j = i + off[d], and the lower diagonals are not read at all
    int nd_real;
    int d0;         // index of the main diagonal (Jacobi)
    T* invD;        // Jacobi: 1 / a_ii, formed in the prologue; nullptr: no preconditioner
    const T* b;
    T* x;           // initial guess in, solution out
    T* r;
    T* p[2];        // direction of iteration k in p[k & 1]
    T* q;           // A p
    T* z;           // M r (== r without preconditioner)
    uint32_t n;
    FusedSync sync;
    DiaCgState* st;
};

// Separately rounded products and sums (no contraction into FMAs): the
// arithmetic of the reference's kernels as compiled for its CPU runs.
__device__ __forceinline__ double add_rn(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ float add_rn(float a, float b) { return __fadd_rn(a, b); }
using dev::mul_rn;

// sum_d A[d][i] * xf(i + off[d]) in T: products rounded, then summed one by
// one in increasing column order from zero -- the order of a CSR-Adaptive
// STREAM block that reduces each row on one lane
// (src/library/kernels/csrmv_adaptive.cl:312-420); the zeros of entries a
// CSR row does not hold add nothing. Loads are unconditional with
// out-of-matrix columns clamped and their products zero; a mirrored
// diagonal's value is read from the upper one at the column's row.
template <int ND, bool SYM, typename Args, typename XF>
__device__ __forceinline__ typename Args::value_type dia_row_seq(const Args& a, uint32_t i, XF xf) {
    using T = typename Args::value_type;
    const uint32_t n = a.n;
    T av[ND], xv[ND];
#pragma unroll
    for (int d = 0; d < ND; ++d) {
        const int64_t j = static_cast<int64_t>(i) + a.A.off[d];
        const bool in = j >= 0 && j < static_cast<int64_t>(n);
        const uint32_t jc = in ? static_cast<uint32_t>(j) : i;
        T v;
        if (SYM && a.A.off[d] < 0)
            v = __ldg(a.A.vals + static_cast<size_t>(ND - 1 - d) * n + jc);
        else
            v = __ldg(a.A.vals + static_cast<size_t>(d) * n + i);
        const T xj = xf(jc);
        av[d] = in ? v : T(0);
        xv[d] = in ? xj : T(0);
    }
    T s = T(0);
#pragma unroll
    for (int d = 0; d < ND; ++d) s = add_rn(s, mul_rn(av[d], xv[d]));
    return s;
}

// Row i of a CSR-Adaptive STREAM block that reduces a row over g lanes (g a
// power of two): lane l sums the row's products l, l + g, ... one by one,
// then the lanes combine pairwise at distances g/2, ..., 1. A banded row
// holds at most kMaxDiags entries, so lanes from kMaxDiags on hold zero.
template <typename T, typename XF>
__device__ __noinline__ T csr_row_lanes(const uint32_t* rp, const uint32_t* cols, const T* vals, uint32_t i,
                                        uint32_t g, XF xf) {
    T v[kMaxDiags];
#pragma unroll
    for (int l = 0; l < kMaxDiags; ++l) v[l] = T(0);
    g = g > static_cast<uint32_t>(kMaxDiags) ? static_cast<uint32_t>(kMaxDiags) : g;
    const uint32_t b = rp[i], e = rp[i + 1];
    for (uint32_t k = b; k < e; ++k) {
        const uint32_t l = (k - b) & (g - 1);
        v[l] = add_rn(v[l], mul_rn(__ldg(vals + k), xf(cols[k])));
    }
    for (uint32_t off = g / 2; off > 0; off >>= 1)
        for (uint32_t l = 0; l < off; ++l) v[l] = add_rn(v[l], v[l + off]);
    return v[0];
}

// q_i = (A xf)_i in the reference's order for row i.
template <int ND, bool SYM, typename Args, typename XF>
__device__ __forceinline__ typename Args::value_type cg_row(const Args& a, uint32_t i, XF xf) {
    for (int k = 0; k < a.nlanes; ++k)
        if (i >= a.lanes[k].r0 && i < a.lanes[k].r1) return csr_row_lanes(a.rp, a.cols, a.vals, i, a.lanes[k].g, xf);
    return dia_row_seq<ND, SYM>(a, i, xf);
}

// The reference's CG (src/library/solvers/conjugate-gradients.hpp:73-226) as
// one cooperative launch over a matrix stored by diagonal. Scalars in T as
// the reference's clsparse::scalar<T>, reductions accumulated in FP64:
//   prologue: r = b - A x, z = M r, p = z; ||b||, ||r||, <r,z>   -> exchange
//             ||b|| == 0: x = b, stop; res = ||r|| / ||b||; stop test with
//             the control's previous nIters
//   A: p_k = z + beta p_{k-1} (k > 0; a neighbour's p_k formed on the fly
//      from its z and p_{k-1}), q = A p_k, <q,p_k>          -> exchange: alpha
//   B: x += alpha p_k, r -= alpha q, z = M r; <r,z>, ||r||   -> exchange:
//      beta = <r,z>_new / <r,z>_old, res, nIters = k, stop test
// The exchanges are bounded waits; a timeout leaves every CTA and sets
// kStatusBarrierTimeout.
template <typename T, int ND, bool SYM>
__global__ void __launch_bounds__(kDiaThreads, kDiaCtasPerSm) dia_cg_ref_kernel(DiaCgArgs<T> a) {
    __shared__ GridSmem gs;
    const FusedSync g = a.sync;
    unsigned long long epoch = 0;
    const uint32_t n = a.n;
    const bool lead = blockIdx.x == 0 && threadIdx.x == 0;
    // No __restrict__: these vectors are read at neighbouring rows by other CTAs.
    T* x = a.x;
    T* r = a.r;
    T* q = a.q;
    T* z = a.z;
    T* invD = a.invD;
    const T* b = a.b;
    const DiaCgState in = *a.st;
    const int l2 = in.l2;
    auto term = [l2](T v) {
        const double d = static_cast<double>(v);
        return l2 ? mul_rn(d, d) : fabs(d);
    };
    auto finish_norm = [l2](double s) { return l2 ? sqrt(s) : s; };

    // ---- prologue
    double tot0[4];
    {
        double acc[4] = {0.0, 0.0, 0.0, 0.0};
        T* p0 = a.p[0];
        for_rows(n, [&](uint32_t i) {
            const T y = cg_row<ND, SYM>(a, i, [&](uint32_t j) { return x[j]; });
            const T bi = __ldg(b + i);
            const T ri = add_rn(bi, -y);
            T zi = ri;
            if (invD != nullptr) {
                const T d = __ldg(a.A.vals + static_cast<size_t>(a.d0) * n + i);
                const T inv = T(1) / d;
                invD[i] = inv;
                zi = mul_rn(ri, inv);
                acc[3] += d == T(0) ? 1.0 : 0.0;
                z[i] = zi;
            }
            r[i] = ri;
            p0[i] = zi;
            acc[0] = add_rn(acc[0], term(bi));
            acc[1] = add_rn(acc[1], term(ri));
            acc[2] = add_rn(acc[2], mul_rn(static_cast<double>(ri), static_cast<double>(zi)));
        });
        if (!grid_exchange<4>(g, epoch, acc, tot0, gs)) goto fail;
    }
    if (tot0[3] > 0.0) {
        if (lead) a.st->zero_diag = 1;
        return;
    }
    {
        const T norm_b = static_cast<T>(finish_norm(tot0[0]));
        if (norm_b == T(0)) {
            for_rows(n, [&](uint32_t i) { x[i] = __ldg(b + i); });
            if (lead) {
                a.st->zero_b = 1;
                a.st->n_iters = 0;
            }
            return;
        }
        const T norm_r0 = static_cast<T>(finish_norm(tot0[1]));
        const double init_res = static_cast<double>(norm_r0 / norm_b);
        auto finished = [&](double res, int n_iters) {
            return res <= in.rel_tol || res <= in.abs_tol * init_res || n_iters >= in.max_iters ||
                   (in.stop_nonfinite && !isfinite(res));
        };
        T rz = static_cast<T>(tot0[2]);
        T beta = T(0);
        double cur_res = init_res;
        int n_iters = 0, status = 0;
        bool done = finished(init_res, in.n_iters_in);
        for (int k = 0; !done; ++k) {
            T* pk = a.p[k & 1];
            const T* pprev = a.p[(k + 1) & 1];
            // ---- A: p_k, q = A p_k, <q, p_k>
            double pq[1] = {0.0};
            if (k == 0) {
                for_rows(n, [&](uint32_t i) {
                    const T pi = pk[i];
                    const T qi = cg_row<ND, SYM>(a, i, [&](uint32_t j) { return pk[j]; });
                    q[i] = qi;
                    pq[0] = add_rn(pq[0], mul_rn(static_cast<double>(qi), static_cast<double>(pi)));
                });
            } else {
                auto pdir = [&](uint32_t j) { return add_rn(z[j], mul_rn(beta, pprev[j])); };
                for_rows(n, [&](uint32_t i) {
                    const T pi = pdir(i);
                    const T qi = cg_row<ND, SYM>(a, i, pdir);
                    pk[i] = pi;
                    q[i] = qi;
                    pq[0] = add_rn(pq[0], mul_rn(static_cast<double>(qi), static_cast<double>(pi)));
                });
            }
            double tq[1];
            if (!grid_exchange<1>(g, epoch, pq, tq, gs)) goto fail;
            const T yp = static_cast<T>(tq[0]);
            const T alpha = rz / yp;
            if (!(yp > T(0))) status |= kStatusCurvature;
            // ---- B: x += alpha p_k, r -= alpha q, z = M r; <r,z>, ||r||
            double acc[2] = {0.0, 0.0};
            for_rows(n, [&](uint32_t i) {
                // every load of the row before its first store (the vectors
                // are not __restrict__, so a store would hold back later loads)
                const T xi = add_rn(x[i], mul_rn(alpha, pk[i]));
                const T ri = add_rn(r[i], -mul_rn(alpha, q[i]));
                const T zi = invD != nullptr ? mul_rn(ri, invD[i]) : ri;
                x[i] = xi;
                r[i] = ri;
                if (invD != nullptr) z[i] = zi;
                acc[0] = add_rn(acc[0], mul_rn(static_cast<double>(ri), static_cast<double>(zi)));
                acc[1] = add_rn(acc[1], term(ri));
            });
            double tb[2];
            if (!grid_exchange<2>(g, epoch, acc, tb, gs)) goto fail;
            const T rz_old = rz;
            rz = static_cast<T>(tb[0]);
            beta = rz / rz_old;
            const T res = static_cast<T>(finish_norm(tb[1])) / norm_b;
            n_iters = k;
            cur_res = static_cast<double>(res);
            if (!isfinite(cur_res)) status |= kStatusNonFinite;
            done = finished(cur_res, n_iters);
        }
        if (lead) {
            a.st->n_iters = n_iters;
            a.st->init_res = init_res;
            a.st->cur_res = cur_res;
            atomicOr(&a.st->status, status);
        }
        return;
    }
fail:
    if (threadIdx.x == 0) atomicOr(&a.st->status, kStatusBarrierTimeout);
}

// ---- the drop-in BiCGStab (clsparse{S,D}csrbicgStab, solver loop mode 3)

template <typename T>
struct DiaBicgArgs {
    using value_type = T;
    DiaMat<T> A;
    const uint32_t* rp;
    const uint32_t* cols;
    const T* vals;
    LaneRange lanes[kMaxLaneRanges];
    int nlanes;
    int nd_real;
    int d0;
    T* invD;        // Jacobi: 1 / a_ii, formed in the prologue; nullptr: no preconditioner
    const T* b;
    T* x;
    T* r;
    T* rs;          // r*
    T* p[2];        // direction of iteration k in p[k & 1]
    T* AMp[2];      // A M p_k in AMp[k & 1]
    T* Mp;          // M p_k (== p_k without preconditioner)
    T* s;
    T* Ms;          // M s (== s without preconditioner)
    T* AMs;
    uint32_t n;
    FusedSync sync;
    DiaCgState* st;
};

// The reference's BiCGStab (src/library/solvers/biconjugate-gradients-
// stabilized.hpp:61-266) as one cooperative launch, in the arithmetic and row
// order of the drop-in CG above. Per iteration k:
//   1: p_k = (r + beta p_{k-1}) - (beta omega) AMp_{k-1}, Mp = M p_k (a
//      neighbour's M p_k formed on the fly), AMp_k = A Mp, <r*, AMp_k>
//                                                         -> exchange: alpha
//   2: s = r - alpha AMp_k, Ms = M s (a neighbour's formed on the fly),
//      AMs = A Ms; ||s||, <AMs, s>, <AMs, AMs>           -> exchange: the
//      stop test on s (then x += alpha Mp and stop), omega
//   3: x = (x + alpha Mp) + omega Ms, r = s - omega AMs; ||r||, <r*, r>
//                                       -> exchange: stop test, beta
// The reference tests ||s|| before forming A M s; here A M s is formed in the
// same pass and dropped when the test stops the solve. The stop tests of the
// first iteration see the nIters the control held before the solve.
template <typename T, int ND, bool SYM>
__global__ void __launch_bounds__(kDiaThreads, kDiaCtasPerSm) dia_bicg_ref_kernel(DiaBicgArgs<T> a) {
    __shared__ GridSmem gs;
    const FusedSync g = a.sync;
    unsigned long long epoch = 0;
    const uint32_t n = a.n;
    const bool lead = blockIdx.x == 0 && threadIdx.x == 0;
    T* x = a.x;
    T* r = a.r;
    T* rs = a.rs;
    T* s = a.s;
    T* Ms = a.Ms;
    T* AMs = a.AMs;
    T* Mp = a.Mp;
    T* invD = a.invD;
    const T* b = a.b;
    const DiaCgState in = *a.st;
    const int l2 = in.l2;
    auto term = [l2](T v) {
        const double d = static_cast<double>(v);
        return l2 ? mul_rn(d, d) : fabs(d);
    };
    auto finish_norm = [l2](double v) { return l2 ? sqrt(v) : v; };
    auto dot = [](T u, T v) { return mul_rn(static_cast<double>(u), static_cast<double>(v)); };
    auto apply_m = [invD](T v, uint32_t j) { return invD != nullptr ? mul_rn(v, invD[j]) : v; };

    // ---- prologue: r = b - A x, r* = r, p = r, Mp = M p
    double tot0[4];
    {
        double acc[4] = {0.0, 0.0, 0.0, 0.0};
        T* p0 = a.p[0];
        for_rows(n, [&](uint32_t i) {
            const T y = cg_row<ND, SYM>(a, i, [&](uint32_t j) { return x[j]; });
            const T bi = __ldg(b + i);
            const T ri = add_rn(bi, -y);
            T mi = ri;
            if (invD != nullptr) {
                const T d = __ldg(a.A.vals + static_cast<size_t>(a.d0) * n + i);
                const T inv = T(1) / d;
                invD[i] = inv;
                mi = mul_rn(ri, inv);
                acc[3] += d == T(0) ? 1.0 : 0.0;
                Mp[i] = mi;
            }
            r[i] = ri;
            rs[i] = ri;
            p0[i] = ri;
            acc[0] = add_rn(acc[0], term(bi));
            acc[1] = add_rn(acc[1], term(ri));
            acc[2] = add_rn(acc[2], dot(ri, ri));
        });
        if (!grid_exchange<4>(g, epoch, acc, tot0, gs)) goto fail;
    }
    if (tot0[3] > 0.0) {
        if (lead) a.st->zero_diag = 1;
        return;
    }
    {
        const T norm_b = static_cast<T>(finish_norm(tot0[0]));
        if (norm_b <= std::numeric_limits<T>::min()) {
            for_rows(n, [&](uint32_t i) { x[i] = __ldg(b + i); });
            if (lead) {
                a.st->zero_b = 1;
                a.st->n_iters = 0;
            }
            return;
        }
        const double init_res = static_cast<double>(static_cast<T>(finish_norm(tot0[1])) / norm_b);
        auto finished = [&](double res, int n_iters) {
            return res <= in.rel_tol || res <= in.abs_tol * init_res || n_iters >= in.max_iters ||
                   (in.stop_nonfinite && !isfinite(res));
        };
        T rsr_old = static_cast<T>(tot0[2]);
        T beta = T(0), omega = T(0);
        double cur_res = init_res;
        int n_iters = in.n_iters_in, status = 0;
        bool done = finished(init_res, n_iters);
        if (done) n_iters = 0;
        for (int k = 0; !done; ++k) {
            T* pk = a.p[k & 1];
            const T* pprev = a.p[(k + 1) & 1];
            T* amp = a.AMp[k & 1];
            const T* amp_prev = a.AMp[(k + 1) & 1];
            // with no preconditioner M p_k is p_k itself
            T* mp = invD != nullptr ? Mp : pk;
            // ---- 1: p_k, M p_k, AMp_k = A M p_k, <r*, AMp_k>
            double acc1[1] = {0.0};
            {
                const T bw = mul_rn(beta, omega);
                auto pdir = [&](uint32_t j) {
                    return add_rn(add_rn(r[j], mul_rn(beta, pprev[j])), -mul_rn(bw, amp_prev[j]));
                };
                if (k == 0) {
                    for_rows(n, [&](uint32_t i) {
                        const T ai = cg_row<ND, SYM>(a, i, [&](uint32_t j) { return mp[j]; });
                        const T rsi = rs[i];
                        amp[i] = ai;
                        acc1[0] = add_rn(acc1[0], dot(ai, rsi));
                    });
                } else {
                    for_rows(n, [&](uint32_t i) {
                        const T pi = pdir(i);
                        const T mi = apply_m(pi, i);
                        const T ai = cg_row<ND, SYM>(a, i, [&](uint32_t j) { return apply_m(pdir(j), j); });
                        const T rsi = rs[i];
                        pk[i] = pi;
                        if (invD != nullptr) Mp[i] = mi;
                        amp[i] = ai;
                        acc1[0] = add_rn(acc1[0], dot(ai, rsi));
                    });
                }
            }
            double t1[1];
            if (!grid_exchange<1>(g, epoch, acc1, t1, gs)) goto fail;
            const T rs_amp = static_cast<T>(t1[0]);
            const T alpha = rsr_old / rs_amp;
            if (rs_amp == T(0)) status |= kStatusBicgBreakdown;
            // ---- 2: s, M s, AMs = A M s; ||s||, <AMs, s>, <AMs, AMs>
            double acc2[3] = {0.0, 0.0, 0.0};
            {
                auto sdir = [&](uint32_t j) { return add_rn(r[j], -mul_rn(alpha, amp[j])); };
                for_rows(n, [&](uint32_t i) {
                    const T si = sdir(i);
                    const T msi = apply_m(si, i);
                    const T ai = cg_row<ND, SYM>(a, i, [&](uint32_t j) { return apply_m(sdir(j), j); });
                    s[i] = si;
                    if (invD != nullptr) Ms[i] = msi;
                    AMs[i] = ai;
                    acc2[0] = add_rn(acc2[0], term(si));
                    acc2[1] = add_rn(acc2[1], dot(ai, si));
                    acc2[2] = add_rn(acc2[2], dot(ai, ai));
                });
            }
            double t2[3];
            if (!grid_exchange<3>(g, epoch, acc2, t2, gs)) goto fail;
            {
                const T res_s = static_cast<T>(finish_norm(t2[0])) / norm_b;
                cur_res = static_cast<double>(res_s);
                if (!isfinite(cur_res)) status |= kStatusNonFinite;
                if (finished(cur_res, n_iters)) {
                    // biconjugate-gradients-stabilized.hpp:183-195: x += alpha M p
                    for_rows(n, [&](uint32_t i) { x[i] = add_rn(x[i], mul_rn(alpha, mp[i])); });
                    n_iters = k;
                    break;
                }
            }
            const T amss = static_cast<T>(t2[1]);
            const T amsams = static_cast<T>(t2[2]);
            omega = amss / amsams;
            if (omega == T(0)) status |= kStatusBicgBreakdown;
            // ---- 3: x, r; ||r||, <r*, r>
            double acc3[2] = {0.0, 0.0};
            {
                const T* msv = invD != nullptr ? Ms : s;
                for_rows(n, [&](uint32_t i) {
                    const T x1 = add_rn(x[i], mul_rn(alpha, mp[i]));
                    const T xi = add_rn(x1, mul_rn(omega, msv[i]));
                    const T ri = add_rn(s[i], -mul_rn(omega, AMs[i]));
                    const T rsi = rs[i];
                    x[i] = xi;
                    r[i] = ri;
                    acc3[0] = add_rn(acc3[0], term(ri));
                    acc3[1] = add_rn(acc3[1], dot(rsi, ri));
                });
            }
            double t3[2];
            if (!grid_exchange<2>(g, epoch, acc3, t3, gs)) goto fail;
            const T res = static_cast<T>(finish_norm(t3[0])) / norm_b;
            cur_res = static_cast<double>(res);
            if (!isfinite(cur_res)) status |= kStatusNonFinite;
            if (finished(cur_res, n_iters)) {
                n_iters = k;
                break;
            }
            const T rsr_new = static_cast<T>(t3[1]);
            beta = rsr_new / rsr_old;
            beta = beta * alpha;
            beta = beta / omega;
            rsr_old = rsr_new;
            n_iters = k + 1;
        }
        if (lead) {
            a.st->n_iters = n_iters;
            a.st->init_res = init_res;
            a.st->cur_res = cur_res;
            atomicOr(&a.st->status, status);
        }
        return;
    }
fail:
    if (threadIdx.x == 0) atomicOr(&a.st->status, kStatusBarrierTimeout);
}

template <typename VA, typename VG, int PK, int NDA, int NDG>
int dia_grid(int sm_count, size_t smem) {
    int b = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, dia_pcg_kernel<VA, VG, PK, NDA, NDG>, kDiaThreads,
                                                      smem) != cudaSuccess) {
        cudaGetLastError();
        b = 1;
    }
    return std::max(1, sm_count) * std::max(1, std::min(b, kDiaCtasPerSm));
}

// smem: dynamic shared memory of the launch (the local-t learned form).
template <typename VA, typename VG, int PK, int NDA, int NDG>
cudaError_t dia_launch(DiaPcgArgs<VA, VG>& a, int sm_count, cudaStream_t s, uint32_t& grid, size_t smem = 0) {
    const void* k = reinterpret_cast<const void*>(dia_pcg_kernel<VA, VG, PK, NDA, NDG>);
    if (smem > 0) {
        const cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                   static_cast<int>(smem));
        if (e != cudaSuccess) return e;
    }
    grid = static_cast<uint32_t>(dia_grid<VA, VG, PK, NDA, NDG>(sm_count, smem));
    void* args[] = {&a};
    return cudaLaunchCooperativeKernel(k, dim3(grid), dim3(kDiaThreads), args, smem, s);
}

// Padded diagonal counts the kernel is built for: A alone (Jacobi / none),
// and (A, G) pairs for the learned factor (G and G^T padded alike).
constexpr int kClassA[] = {3, 5, 7, 9, kMaxDiags};
constexpr int kPairs[][2] = {{5, 3}, {7, 4}, {9, 5}, {kMaxDiags, kMaxDiags}};

size_t align256(size_t b) { return (b + 255) & ~size_t(255); }

}  // namespace

bool dia_enabled() {
    const char* e = std::getenv("CLSPARSE_B200_DIA");
    return !(e && e[0] == '0' && e[1] == '\0');
}

clsparseStatus dia_detect(const uint32_t* rp, const uint32_t* cols, uint32_t n, uint32_t nnz, DiaWork& w,
                          cudaStream_t s, DiaOffsets& offs) {
    offs.nd = 0;
    if (n == 0 || nnz == 0) return clsparseInvalidValue;
    if (w.table.ensure(kSlots * sizeof(int32_t) + 64) != cudaSuccess) {
        cudaGetLastError();
        return clsparseOutOfResources;
    }
    int32_t* table = static_cast<int32_t*>(w.table.ptr);
    int* flags = reinterpret_cast<int*>(table + kSlots);
    cudaMemsetAsync(table, 0x80, kSlots * sizeof(int32_t), s);  // kEmpty in every slot
    cudaMemsetAsync(flags, 0, sizeof(int), s);
    const uint32_t grid = std::min<uint32_t>((n + 255) / 256, 1184);
    dia_offsets_kernel<<<grid, 256, 0, s>>>(rp, cols, n, table, flags);
    int32_t h[kSlots + 1];
    if (cudaGetLastError() != cudaSuccess ||
        cudaMemcpyAsync(h, table, sizeof(h), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess)
        return clsparseInvalidKernelExecution;
    if (h[kSlots] != 0) return clsparseInvalidValue;
    std::vector<int32_t> o;
    for (int k = 0; k < kSlots; ++k)
        if (h[k] != kEmpty) o.push_back(h[k]);
    if (o.empty() || o.size() > static_cast<size_t>(kMaxDiags)) return clsparseInvalidValue;
    // at least half of the stored diagonal entries hold matrix entries
    if (static_cast<uint64_t>(nnz) * 2 < static_cast<uint64_t>(o.size()) * n) return clsparseInvalidValue;
    std::sort(o.begin(), o.end());
    offs.nd = static_cast<int>(o.size());
    for (int d = 0; d < offs.nd; ++d) offs.off[d] = o[d];
    return clsparseSuccess;
}

template <typename VI, typename VO>
clsparseStatus dia_build(const uint32_t* rp, const uint32_t* cols, const VI* vals, uint32_t n,
                         const DiaOffsets& offs, int nd_pad, DeviceBuffer& buf, cudaStream_t s, DiaMat<VO>& out) {
    if (nd_pad < offs.nd || nd_pad > kMaxDiags) return clsparseInvalidValue;
    const size_t bytes = static_cast<size_t>(nd_pad) * n * sizeof(VO);
    if (buf.ensure(bytes + 256) != cudaSuccess) {
        cudaGetLastError();
        return clsparseOutOfResources;
    }
    VO* v = static_cast<VO*>(buf.ptr);
    cudaMemsetAsync(v, 0, bytes, s);
    const uint32_t grid = std::min<uint32_t>((n + 255) / 256, 1184);
    dia_fill_kernel<VI, VO><<<grid, 256, 0, s>>>(rp, cols, vals, n, offs, v);
    if (cudaGetLastError() != cudaSuccess) return clsparseInvalidKernelExecution;
    out.vals = v;
    out.nd = nd_pad;  // padded diagonals: offset 0, values 0
    for (int d = 0; d < kMaxDiags; ++d) out.off[d] = d < offs.nd ? offs.off[d] : 0;
    return clsparseSuccess;
}

// Index of the main diagonal among a DIA matrix's offsets: the first zero
// offset (padding diagonals, also at offset 0, come after the real ones).
template <typename V>
int main_diag_index(const DiaMat<V>& A) {
    int d0 = -1;
    for (int d = A.nd - 1; d >= 0; --d)
        if (A.off[d] == 0) d0 = d;
    return d0;
}

template <typename VA>
clsparseStatus dia_jacobi(const DiaMat<VA>& A, uint32_t n, float* invD, int* status, cudaStream_t s) {
    const uint32_t grid = std::min<uint32_t>((n + 255) / 256, 1184);
    if (A.diag32 != nullptr) {
        dia_inv_diag_kernel<float><<<grid, 256, 0, s>>>(A.diag32, n, invD, status);
        return cudaGetLastError() == cudaSuccess ? clsparseSuccess : clsparseInvalidKernelExecution;
    }
    const int d0 = main_diag_index(A);
    if (d0 < 0) return clsparseInvalidValue;  // no main diagonal: the CSR path reports it
    dia_inv_diag_kernel<VA><<<grid, 256, 0, s>>>(A.vals + static_cast<size_t>(d0) * n, n, invD, status);
    return cudaGetLastError() == cudaSuccess ? clsparseSuccess : clsparseInvalidKernelExecution;
}

template <typename V>
clsparseStatus dia_compensate_diag(const uint32_t* rp, const uint32_t* cols, const double* vals, uint32_t n,
                                   DiaMat<V>& A, float* diag32, cudaStream_t s) {
    const int d0 = main_diag_index(A);
    if (d0 < 0 || diag32 == nullptr) return clsparseInvalidValue;
    V* main_diag = const_cast<V*>(A.vals) + static_cast<size_t>(d0) * n;
    const uint32_t grid = std::min<uint32_t>((n + 255) / 256, 1184);
    dia_comp_diag_kernel<V><<<grid, 256, 0, s>>>(rp, cols, vals, n, main_diag, diag32);
    if (cudaGetLastError() != cudaSuccess) return clsparseInvalidKernelExecution;
    A.diag32 = diag32;
    return clsparseSuccess;
}

void dia_classes(int nda, int ndg, bool learned, int& ca, int& cg) {
    ca = cg = 0;
    if (!learned) {
        for (int c : kClassA)
            if (nda <= c) {
                ca = c;
                return;
            }
        return;
    }
    for (const auto& p : kPairs)
        if (nda <= p[0] && ndg <= p[1]) {
            ca = p[0];
            cg = p[1];
            return;
        }
}

namespace {

// One inner solve as one cooperative launch.
// Shared memory of the local-t learned form (t for a CTA's rows and the
// gt_halo rows after them), or 0 when that form does not apply: an offset of
// G^T below zero, more than kLocalTMaxSmem bytes, or CLSPARSE_B200_DIA_LOCAL_T=0.
constexpr size_t kLocalTMaxSmem = 160 * 1024;
template <typename VA, typename VG>
size_t local_t_smem(const DiaPcgArgs<VA, VG>& a, int sm_count) {
    const char* env = std::getenv("CLSPARSE_B200_DIA_LOCAL_T");
    if (env && std::atoi(env) == 0) return 0;
    for (int e = 0; e < a.GT.nd; ++e)
        if (a.GT.off[e] < 0) return 0;
    const uint64_t G = static_cast<uint64_t>(std::max(1, sm_count));  // one CTA per SM
    const uint64_t rows = (a.n + G - 1) / G + a.gt_halo;
    const size_t bytes = static_cast<size_t>(rows) * sizeof(float);
    return bytes <= kLocalTMaxSmem ? bytes : 0;
}

template <typename VA, typename VG>
clsparseStatus dia_persistent_solve(DiaPcgArgs<VA, VG> a, bool learned, DiaWork& w, clsparseControl c,
                                    DiaPcgState& st) {
    cudaStream_t s = c->stream;
    const uint32_t max_grid = static_cast<uint32_t>(std::max(1, c->sm_count) * std::max(2, kDiaCtasPerSm));
    const size_t sync_b = align256(fused_sync_bytes(max_grid));
    if (w.sync.ensure(sync_b + align256(sizeof(DiaPcgState))) != cudaSuccess) {
        cudaGetLastError();
        return clsparseOutOfResources;
    }
    char* base = static_cast<char*>(w.sync.ptr);
    DiaPcgState* dst = reinterpret_cast<DiaPcgState*>(base + sync_b);
    st.status = 0;
    cudaMemsetAsync(base, 0, kFusedSyncHead, s);
    cudaMemcpyAsync(dst, &st, sizeof(st), cudaMemcpyHostToDevice, s);
    a.sync = fused_sync_at(base);
    // failure-path test switches, as for the CSR persistent engine
    if (const char* e = std::getenv("CLSPARSE_B200_BARRIER_WAIT_NS")) {
        const unsigned long long v = std::strtoull(e, nullptr, 10);
        if (v > 0) a.sync.wait_ns = v;
    }
    if (const char* e = std::getenv("CLSPARSE_B200_TEST_BARRIER_NEVER_RELEASE")) a.sync.never_release = std::atoi(e) != 0;
    a.st = dst;
    const int sms = c->sm_count;
    uint32_t grid = 0;
    cudaError_t e = cudaErrorInvalidValue;
    const int na = a.A.nd, ng = a.G.nd;
    if (!learned) {
        if (na == 3) e = dia_launch<VA, VG, 0, 3, 3>(a, sms, s, grid);
        else if (na == 5) e = dia_launch<VA, VG, 0, 5, 3>(a, sms, s, grid);
        else if (na == 7) e = dia_launch<VA, VG, 0, 7, 3>(a, sms, s, grid);
        else if (na == 9) e = dia_launch<VA, VG, 0, 9, 3>(a, sms, s, grid);
        else if (na == kMaxDiags) e = dia_launch<VA, VG, 0, kMaxDiags, 3>(a, sms, s, grid);
    } else if (local_t_smem(a, sms) > 0) {
        // t kept per CTA in shared memory: two grid exchanges per iteration
        const size_t sm = local_t_smem(a, sms);
        if (na == 5 && ng == 3) e = dia_launch<VA, VG, 2, 5, 3>(a, sms, s, grid, sm);
        else if (na == 7 && ng == 4) e = dia_launch<VA, VG, 2, 7, 4>(a, sms, s, grid, sm);
        else if (na == 9 && ng == 5) e = dia_launch<VA, VG, 2, 9, 5>(a, sms, s, grid, sm);
        else if (na == kMaxDiags && ng == kMaxDiags) e = dia_launch<VA, VG, 2, kMaxDiags, kMaxDiags>(a, sms, s, grid, sm);
    } else {
        if (na == 5 && ng == 3) e = dia_launch<VA, VG, 1, 5, 3>(a, sms, s, grid);
        else if (na == 7 && ng == 4) e = dia_launch<VA, VG, 1, 7, 4>(a, sms, s, grid);
        else if (na == 9 && ng == 5) e = dia_launch<VA, VG, 1, 9, 5>(a, sms, s, grid);
        else if (na == kMaxDiags && ng == kMaxDiags) e = dia_launch<VA, VG, 1, kMaxDiags, kMaxDiags>(a, sms, s, grid);
    }
    if (e != cudaSuccess || grid > max_grid) {
        cudaGetLastError();
        return clsparseInvalidKernelExecution;
    }
    if (cudaMemcpyAsync(&st, dst, sizeof(st), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess)
        return clsparseInvalidKernelExecution;
    if (st.status & kStatusBarrierTimeout) return clsparseInvalidKernelExecution;
    return clsparseSuccess;
}

}  // namespace

template <typename VA, typename VG>
clsparseStatus dia_pcg_solve(DiaPcgArgs<VA, VG> a, bool learned, DiaWork& w, clsparseControl c,
                             DiaPcgState& st) {
    return dia_persistent_solve<VA, VG>(a, learned, w, c, st);
}

namespace {

// flag |= 1 when A[i][i + off_l] (diagonal dl, off_l < 0) differs bitwise
// from A[i + off_l][i] (diagonal du at -off_l) for a row i inside the matrix.
template <typename T>
__global__ void dia_sym_check_kernel(const T* __restrict__ vals, uint32_t n, int dl, int du, int32_t off_l,
                                     int* flag) {
    using U = std::conditional_t<sizeof(T) == 8, unsigned long long, unsigned int>;
    bool bad = false;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int64_t j = static_cast<int64_t>(i) + off_l;
        if (j < 0) continue;
        const T lo = vals[static_cast<size_t>(dl) * n + i];
        const T up = vals[static_cast<size_t>(du) * n + static_cast<size_t>(j)];
        U bl, bu;
        memcpy(&bl, &lo, sizeof(U));
        memcpy(&bu, &up, sizeof(U));
        bad |= bl != bu;
    }
    if (bad) atomicOr(flag, 1);
}

// Whether the drop-in CG runs its SYM form: A symmetric bit for bit with
// symmetric offsets (off[d] = -off[nd - 1 - d]), at most 5 diagonals (the
// form's register budget), and -- unless CLSPARSE_B200_DIA_SYM=1 asks for it
// whenever A qualifies (=0: never) -- a working set (the diagonals and the
// seven work vectors) above half of L2. Measured per iteration on B200: the
// 1024^2 five-point FP64 matrix (96 MB) 30.0 -> 26.5 us; where the working
// set stays in L2 the extra index arithmetic costs more than the bytes it
// saves (512^2 FP64: 11.6 -> 12.0 us, 1024^2 FP32: 19.3 -> 21.9 us).
// Diagonal classes the SYM form runs for. On the 128^3 seven-point matrix it
// measured slower (FP64 74.8 vs 70.8 us per iteration, FP32 48.9 vs 42.8):
// the mirrored reads at -16384 rows fall in another CTA's slice, L2 instead
// of L1.
constexpr int kSymMaxDiags = 5;

template <typename T>
clsparseStatus dia_symmetric(const DiaMat<T>& M, const DiaOffsets& offs, uint32_t n, int nd_pad, size_t l2_bytes,
                             DiaWork& w, cudaStream_t s, bool& sym) {
    sym = false;
    const char* env = std::getenv("CLSPARSE_B200_DIA_SYM");
    const int mode = env ? std::atoi(env) : -1;
    if (mode == 0 || nd_pad > kSymMaxDiags || offs.nd != nd_pad) return clsparseSuccess;
    const size_t working = static_cast<size_t>(nd_pad + 7) * n * sizeof(T);
    if (mode != 1 && (l2_bytes == 0 || 2 * working <= l2_bytes)) return clsparseSuccess;
    const int nd = offs.nd;
    for (int d = 0; d < nd; ++d)
        if (offs.off[d] != -offs.off[nd - 1 - d]) return clsparseSuccess;
    if (nd < 2) return clsparseSuccess;
    int* flag = reinterpret_cast<int*>(static_cast<int32_t*>(w.table.ptr) + kSlots) + 1;
    cudaMemsetAsync(flag, 0, sizeof(int), s);
    const uint32_t grid = std::min<uint32_t>((n + 255) / 256, 1184);
    for (int d = 0; offs.off[d] < 0; ++d)
        dia_sym_check_kernel<T><<<grid, 256, 0, s>>>(M.vals, n, d, nd - 1 - d, offs.off[d], flag);
    int h = 1;
    if (cudaGetLastError() != cudaSuccess ||
        cudaMemcpyAsync(&h, flag, sizeof(int), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess)
        return clsparseInvalidKernelExecution;
    sym = h == 0;
    return clsparseSuccess;
}

// The cooperative kernel of a drop-in solve for an argument block.
template <typename T, int ND, bool SYM>
const void* dropin_kernel(const DiaCgArgs<T>*) {
    return reinterpret_cast<const void*>(dia_cg_ref_kernel<T, ND, SYM>);
}
template <typename T, int ND, bool SYM>
const void* dropin_kernel(const DiaBicgArgs<T>*) {
    return reinterpret_cast<const void*>(dia_bicg_ref_kernel<T, ND, SYM>);
}

template <typename T, int ND, bool SYM, typename Args>
cudaError_t dropin_launch(Args& a, int sm_count, cudaStream_t s, uint32_t max_grid) {
    const void* k = dropin_kernel<T, ND, SYM>(&a);
    int b = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k, kDiaThreads, 0) != cudaSuccess) {
        cudaGetLastError();
        return cudaErrorInvalidConfiguration;
    }
    if (b < 1) return cudaErrorInvalidConfiguration;
    const uint32_t grid = static_cast<uint32_t>(std::max(1, sm_count) * std::min(b, kDiaCtasPerSm));
    if (grid > max_grid) return cudaErrorInvalidConfiguration;
    void* args[] = {&a};
    return cudaLaunchCooperativeKernel(k, dim3(grid), dim3(kDiaThreads), args, 0, s);
}

// The drop-in solves (clsparse{S,D}csrcg with BICG false, clsparse{S,D}csrbicgStab
// with BICG true) on the banded engine.
template <typename T, bool BICG>
clsparseStatus dia_dropin(cldenseVector* xv, const clsparseCsrMatrix* A, const cldenseVector* bv,
                          clSParseSolverControl sc, clsparseControl c) {
    using Args = std::conditional_t<BICG, DiaBicgArgs<T>, DiaCgArgs<T>>;
    const uint32_t n = static_cast<uint32_t>(A->num_rows);
    const uint32_t nnz = static_cast<uint32_t>(A->num_nonzeros);
    if (n == 0 || nnz == 0) return clsparseNotImplemented;
    // The reference's solvers multiply with csrmv_adaptive when the matrix has
    // a meta (csrmv_general otherwise: the graph engine runs that order). Its
    // STREAM blocks reduce a row on one lane except in a few blocks (the last
    // one, with few rows): those row ranges are taken over as CSR rows with
    // their lane count. A block of another kind, or more such ranges than
    // kMaxLaneRanges, leaves the solve to the graph engine.
    const auto* meta = static_cast<const matrix_meta*>(A->meta);
    if (meta == nullptr || meta->h_rowBlocks.size() < meta->num_words || meta->num_words < 2)
        return clsparseNotImplemented;
    LaneRange lanes[kMaxLaneRanges];
    int nlanes = 0;
    for (size_t w = 0; w + 1 < meta->num_words; ++w) {
        const uint64_t w0 = meta->h_rowBlocks[w], w1 = meta->h_rowBlocks[w + 1];
        const uint32_t r0 = static_cast<uint32_t>(w0 >> 32), r1 = static_cast<uint32_t>(w1 >> 32);
        if (r1 - r0 <= meta->rows_for_vector) return clsparseNotImplemented;  // not a STREAM block
        const uint32_t low = static_cast<uint32_t>(w0 & ((1u << kWgBits) - 1u));
        const uint32_t g = low == 0 ? 1u : std::min(low, 32u);
        if (g == 1) continue;
        if ((g & (g - 1)) != 0 || nlanes == kMaxLaneRanges) return clsparseNotImplemented;
        if (nlanes > 0 && lanes[nlanes - 1].r1 == r0 && lanes[nlanes - 1].g == g)
            lanes[nlanes - 1].r1 = r1;
        else
            lanes[nlanes++] = LaneRange{r0, r1, g};
    }
    cudaStream_t s = c->stream;
    if (!c->dia_cg) c->dia_cg = std::make_unique<DiaWork>();
    DiaWork& w = *c->dia_cg;
    const uint32_t* rp = dev_ptr<const uint32_t>(A->row_pointer, A->off_row_pointer);
    const uint32_t* cols = dev_ptr<const uint32_t>(A->col_indices, A->off_col_indices);
    const T* vals = dev_ptr<const T>(A->values, A->off_values);
    DiaOffsets offs;
    clsparseStatus stt = dia_detect(rp, cols, n, nnz, w, s, offs);
    if (stt == clsparseInvalidValue) return clsparseNotImplemented;  // not banded
    if (stt != clsparseSuccess) return stt;
    int ca = 0, cg = 0;
    dia_classes(offs.nd, 0, false, ca, cg);
    const bool jac = sc->preconditioner == DIAGONAL;
    bool has_main = false;
    for (int d = 0; d < offs.nd; ++d) has_main |= offs.off[d] == 0;
    if (ca == 0 || (jac && !has_main)) return clsparseNotImplemented;
    // BiCGStab forms a neighbour's M p and M s from three to four vectors
    // each: it pays while the diagonals and the eleven work vectors stay in
    // L2. Measured per iteration on B200 against the graph engine (FP64):
    // 512^2 five-point (33 MB) 25.0 vs 34.0 us; 1024^2 five-point (134 MB)
    // 82.6 vs 81.6; 128^3 seven-point (288 MB) 191 vs 161. Larger systems
    // run the graph engine.
    if (BICG && static_cast<size_t>(ca + 11) * n * sizeof(T) > c->l2_bytes) return clsparseNotImplemented;
    DiaMat<T> M;
    stt = dia_build<T, T>(rp, cols, vals, n, offs, ca, w.A, s, M);
    if (stt != clsparseSuccess) return stt;
    bool sym = false;
    if (!BICG) {
        stt = dia_symmetric<T>(M, offs, n, ca, c->l2_bytes, w, s, sym);
        if (stt != clsparseSuccess) return stt;
    }

    // work vectors -- CG: invD, r, p[0], p[1], q, z; BiCGStab: invD, r, r*,
    // p[0], p[1], AMp[0], AMp[1], Mp, s, Ms, AMs
    const int nvec = BICG ? 11 : 6;
    const size_t vb = align256(static_cast<size_t>(n) * sizeof(T));
    const uint32_t max_grid = static_cast<uint32_t>(std::max(1, c->sm_count) * kDiaCtasPerSm);
    const size_t sync_b = align256(fused_sync_bytes(max_grid));
    if (w.vecs.ensure(nvec * vb) != cudaSuccess ||
        w.sync.ensure(sync_b + align256(sizeof(DiaCgState))) != cudaSuccess) {
        cudaGetLastError();
        return clsparseOutOfResources;
    }
    char* vbase = static_cast<char*>(w.vecs.ptr);
    auto vec = [&](int k) { return reinterpret_cast<T*>(vbase + static_cast<size_t>(k) * vb); };
    Args a{};
    a.A = M;
    a.rp = rp;
    a.cols = cols;
    a.vals = vals;
    for (int k = 0; k < nlanes; ++k) a.lanes[k] = lanes[k];
    a.nlanes = nlanes;
    a.nd_real = offs.nd;
    a.d0 = main_diag_index(M);
    a.invD = jac ? vec(0) : nullptr;
    a.b = dev_ptr<const T>(bv->values, bv->off_values);
    a.x = dev_ptr<T>(xv->values, xv->off_values);
    a.r = vec(1);
    a.n = n;
    if constexpr (BICG) {
        a.rs = vec(2);
        a.p[0] = vec(3);
        a.p[1] = vec(4);
        a.AMp[0] = vec(5);
        a.AMp[1] = vec(6);
        a.Mp = vec(7);
        a.s = vec(8);
        a.Ms = jac ? vec(9) : a.s;
        a.AMs = vec(10);
    } else {
        a.p[0] = vec(2);
        a.p[1] = vec(3);
        a.q = vec(4);
        a.z = jac ? vec(5) : a.r;
    }

    char* base = static_cast<char*>(w.sync.ptr);
    DiaCgState h;
    h.rel_tol = sc->relativeTolerance;
    h.abs_tol = sc->absoluteTolerance;
    h.max_iters = sc->maxIters;
    h.n_iters_in = sc->nIters;
    h.l2 = sc->normType & 1;
    h.stop_nonfinite = sc->stopOnNonFinite ? 1 : 0;
    a.st = reinterpret_cast<DiaCgState*>(base + sync_b);
    cudaMemsetAsync(base, 0, kFusedSyncHead, s);
    cudaMemcpyAsync(a.st, &h, sizeof(h), cudaMemcpyHostToDevice, s);
    a.sync = fused_sync_at(base);
    // failure-path test switches, as for the other persistent solvers
    if (const char* e = std::getenv("CLSPARSE_B200_BARRIER_WAIT_NS")) {
        const unsigned long long v = std::strtoull(e, nullptr, 10);
        if (v > 0) a.sync.wait_ns = v;
    }
    if (const char* e = std::getenv("CLSPARSE_B200_TEST_BARRIER_NEVER_RELEASE")) a.sync.never_release = std::atoi(e) != 0;

    const int sms = c->sm_count;
    cudaError_t e = cudaErrorInvalidValue;
    if (sym) {
        if constexpr (!BICG) {
            if (ca == 3) e = dropin_launch<T, 3, true>(a, sms, s, max_grid);
            else if (ca == 5) e = dropin_launch<T, 5, true>(a, sms, s, max_grid);
        }
    } else {
        if (ca == 3) e = dropin_launch<T, 3, false>(a, sms, s, max_grid);
        else if (ca == 5) e = dropin_launch<T, 5, false>(a, sms, s, max_grid);
        else if (ca == 7) e = dropin_launch<T, 7, false>(a, sms, s, max_grid);
        else if (ca == 9) e = dropin_launch<T, 9, false>(a, sms, s, max_grid);
        else if (ca == kMaxDiags) e = dropin_launch<T, kMaxDiags, false>(a, sms, s, max_grid);
    }
    if (e != cudaSuccess) {
        cudaGetLastError();
        return clsparseInvalidKernelExecution;
    }
    if (cudaMemcpyAsync(&h, a.st, sizeof(h), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess)
        return clsparseInvalidKernelExecution;
    if (c->event) cudaEventRecord(c->event, s);
    sc->deviceStatus = static_cast<cl_uint>(h.status);
    sc->historyLength = 0;
    if (h.status & kStatusBarrierTimeout) return clsparseInvalidKernelExecution;
    if (h.zero_diag) return clsparseNotImplemented;  // x untouched; the graph engine reports the zero
    if (h.zero_b) {
        // conjugate-gradients.hpp:87-95 (biconjugate-gradients-stabilized.hpp
        // alike) resets the tolerances of the control
        sc->nIters = 0;
        sc->absoluteTolerance = 0.0;
        sc->relativeTolerance = 0.0;
        return clsparseSuccess;
    }
    sc->initialResidual = h.init_res;
    sc->currentResidual = h.cur_res;
    sc->nIters = h.n_iters;
    return clsparseSuccess;
}

}  // namespace

template <typename T>
clsparseStatus dia_cg_dropin(cldenseVector* xv, const clsparseCsrMatrix* A, const cldenseVector* bv,
                             clSParseSolverControl sc, clsparseControl c) {
    return dia_dropin<T, false>(xv, A, bv, sc, c);
}

template <typename T>
clsparseStatus dia_bicg_dropin(cldenseVector* xv, const clsparseCsrMatrix* A, const cldenseVector* bv,
                               clSParseSolverControl sc, clsparseControl c) {
    return dia_dropin<T, true>(xv, A, bv, sc, c);
}

template clsparseStatus dia_cg_dropin<float>(cldenseVector*, const clsparseCsrMatrix*, const cldenseVector*,
                                             clSParseSolverControl, clsparseControl);
template clsparseStatus dia_cg_dropin<double>(cldenseVector*, const clsparseCsrMatrix*, const cldenseVector*,
                                              clSParseSolverControl, clsparseControl);
template clsparseStatus dia_bicg_dropin<float>(cldenseVector*, const clsparseCsrMatrix*, const cldenseVector*,
                                               clSParseSolverControl, clsparseControl);
template clsparseStatus dia_bicg_dropin<double>(cldenseVector*, const clsparseCsrMatrix*, const cldenseVector*,
                                                clSParseSolverControl, clsparseControl);

#define CLSP_DIA_INST(VA, VG)                                                                                 \
    template clsparseStatus dia_pcg_solve<VA, VG>(DiaPcgArgs<VA, VG>, bool, DiaWork&, clsparseControl,       \
                                                  DiaPcgState&);
CLSP_DIA_INST(float, __nv_bfloat16)
CLSP_DIA_INST(__nv_bfloat16, __nv_bfloat16)
#undef CLSP_DIA_INST

template clsparseStatus dia_build<double, float>(const uint32_t*, const uint32_t*, const double*, uint32_t,
                                                 const DiaOffsets&, int, DeviceBuffer&, cudaStream_t, DiaMat<float>&);
template clsparseStatus dia_build<double, __nv_bfloat16>(const uint32_t*, const uint32_t*, const double*, uint32_t,
                                                         const DiaOffsets&, int, DeviceBuffer&, cudaStream_t,
                                                         DiaMat<__nv_bfloat16>&);
template clsparseStatus dia_build<__nv_bfloat16, __nv_bfloat16>(const uint32_t*, const uint32_t*,
                                                                const __nv_bfloat16*, uint32_t, const DiaOffsets&,
                                                                int, DeviceBuffer&, cudaStream_t,
                                                                DiaMat<__nv_bfloat16>&);
template clsparseStatus dia_compensate_diag<float>(const uint32_t*, const uint32_t*, const double*, uint32_t,
                                                    DiaMat<float>&, float*, cudaStream_t);
template clsparseStatus dia_compensate_diag<__nv_bfloat16>(const uint32_t*, const uint32_t*, const double*, uint32_t,
                                                            DiaMat<__nv_bfloat16>&, float*, cudaStream_t);
template clsparseStatus dia_jacobi<float>(const DiaMat<float>&, uint32_t, float*, int*, cudaStream_t);
template clsparseStatus dia_jacobi<__nv_bfloat16>(const DiaMat<__nv_bfloat16>&, uint32_t, float*, int*,
                                                  cudaStream_t);

}  // namespace clsp
