// Learned factorized sparse approximate inverse (project extension, no
// reference counterpart): a 4-layer message-passing network over the graph
// of an SPD matrix A emits a lower-triangular G on the pattern of tril(A)
// with a softplus-positive diagonal, so M^-1 = G^T G is SPD. The forward and
// backward passes, the loss and the optimiser are the kernels of this file;
// training runs on the GPU.
//
// Scaling: the network sees A_hat = D^-1/2 A D^-1/2 (unit diagonal) and emits
// G_hat; the preconditioner factor is G = G_hat D^-1/2.
//
// Network (hidden width H = 64, message passing over the off-diagonal
// pattern of A, which is symmetric):
//   h0_i  = relu(W_in f_i + b_in)                 f_i = [1, sum_j|a_hat_ij|, deg_i/8, 0]
//   layer l = 1..4:
//     u_j  = U_l h_j
//     s_i  = sum_{j != i} relu(u_j + a_hat_ij w_l + c_l)
//     h_i <- h_i + relu(V_l [h_i ; s_i] + d_l)
//   g_hat_ii = softplus(w_d . h_i + b_d)
//   g_hat_ij = w_o . relu(P h_i + Q h_j + a_hat_ij r + t) + b_o   (j < i, a_ij != 0)
// Weights are kept in FP32 for the optimiser and used as BF16 in the
// forward and backward passes (products accumulated in FP32); a debug switch
// uses the FP32 copies instead (gradient checks). In the BF16 forward pass the
// dense layers U_l, V_l, P and Q run on the tcgen05 tensor cores
// (linear_fwd_umma: BF16 operands in shared memory, FP32 accumulator in
// tensor memory).
//
// Loss: the Kaporin condition-number bound of G_hat A_hat G_hat^T,
//   L_K = log(tr(G_hat A_hat G_hat^T) / n) - (2/n) sum_i log g_hat_ii,
// whose minimiser on a fixed pattern is the classical FSAI factor, plus
// lambda times the mean over residual probes r (CG residual histories) of
//   ||G_hat^T G_hat A_hat r - r||^2 / ||r||^2.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <initializer_list>
#include <cstring>
#include <random>
#include <type_traits>
#include <vector>

#include "device_common.cuh"
#include "internal.h"
#include "pipeline.cuh"
#include "scan.cuh"

namespace clsp {
namespace gnn {

constexpr int H = 64;      // hidden width
constexpr int HO = 32;     // width of the edge output MLP
constexpr int NF = 4;      // node input features
constexpr int NL = 4;      // message-passing layers
constexpr int kMaxTrainP = 32;  // max entries per row of tril(A) for training (local blocks B_i are m x m)

// ---- flat parameter layout ----
struct Offsets {
    int w_in, b_in;
    int U[NL], w[NL], c[NL], V[NL], d[NL];
    int P, Q, r, t, w_o, b_o, w_d, b_d;
    int total;
};

inline Offsets layout() {
    Offsets o;
    int k = 0;
    auto take = [&](int n) {
        const int s = k;
        k += n;
        return s;
    };
    o.w_in = take(H * NF);
    o.b_in = take(H);
    for (int l = 0; l < NL; ++l) {
        o.U[l] = take(H * H);
        o.w[l] = take(H);
        o.c[l] = take(H);
        o.V[l] = take(H * 2 * H);
        o.d[l] = take(H);
    }
    o.P = take(HO * H);
    o.Q = take(HO * H);
    o.r = take(HO);
    o.t = take(HO);
    o.w_o = take(HO);
    o.b_o = take(1);
    o.w_d = take(H);
    o.b_d = take(1);
    o.total = k;
    return o;
}

__device__ __forceinline__ float bfr(float v) {  // round a weight through BF16
    return __bfloat162float(__float2bfloat16(v));
}

// Y[n x M] = act(X1 W1^T + X2 W2^T + b) (+ R), W = [W1 | W2] row-major M x (K1+K2).
// act: 0 none, 1 relu. Rows tiled 32 per CTA; weights staged in shared memory.
template <int M, int K1, int K2>
__global__ void __launch_bounds__(256)
    linear_fwd(const float* __restrict__ X1, const float* __restrict__ X2, const float* __restrict__ W,
               const float* __restrict__ b, const float* __restrict__ R, float* __restrict__ Y,
               float* __restrict__ A, size_t n, int act, int bf16) {
    constexpr int K = K1 + K2;
    constexpr int ROWS = 16;
    __shared__ float sw[M * K];
    __shared__ float sx[ROWS][K + 1];
    for (int i = threadIdx.x; i < M * K; i += 256) sw[i] = bf16 ? bfr(W[i]) : W[i];
    const size_t r0 = static_cast<size_t>(blockIdx.x) * ROWS;
    for (int i = threadIdx.x; i < ROWS * K; i += 256) {
        const int rr = i / K, kk = i % K;
        const size_t row = r0 + rr;
        float v = 0.f;
        if (row < n) v = kk < K1 ? X1[row * K1 + kk] : X2[row * K2 + (kk - K1)];
        sx[rr][kk] = v;
    }
    __syncthreads();
    for (int o = threadIdx.x; o < ROWS * M; o += 256) {
        const int rr = o / M, m = o % M;
        const size_t row = r0 + rr;
        if (row >= n) continue;
        float z = b ? b[m] : 0.f;
#pragma unroll 8
        for (int kk = 0; kk < K; ++kk) z = fmaf(sx[rr][kk], sw[m * K + kk], z);
        const float a = act ? fmaxf(z, 0.f) : z;
        if (A) A[row * M + m] = a;
        Y[row * M + m] = R ? R[row * M + m] + a : a;
    }
}

// ---- tcgen05 tensor-core form of the dense layers (BF16 inference) ----
//
// Y[n x M] = act(X W^T + b) (+ R) with X = [X1 | X2] and W rounded to BF16 and
// FP32 accumulation, on the sm_100 tensor cores: one 128 x M x 16 UMMA
// (tcgen05.mma, kind::f16) per 16 columns of K, issued by one thread, the
// 128 x M FP32 accumulator in tensor memory. A persistent CTA of 4 warps
// stages the weights once, then per 128-row tile of X: stages the tile as
// BF16 in shared memory, issues the MMAs, waits on their commit barrier, and
// each warp reads its 32 accumulator rows (TMEM lanes) for the epilogue (bias,
// ReLU, residual). Operands are K-major without swizzle: core matrices of
// 8 rows x 16 bytes, stored contiguously, the 8-row groups K*16 bytes apart
// (SBO) and the two K-halves of one MMA 128 bytes apart (LBO).
namespace umma {

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Shared-memory matrix descriptor (no swizzle, descriptor version 1).
__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    return static_cast<uint64_t>((saddr >> 4) & 0x3FFFu) | (static_cast<uint64_t>((lbo >> 4) & 0x3FFFu) << 16) |
           (static_cast<uint64_t>((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// Instruction descriptor of kind::f16: D FP32, A and B BF16, both K-major.
template <int TM, int TN>
__host__ __device__ constexpr uint32_t idesc_bf16() {
    return (1u << 4) | (1u << 7) | (1u << 10) | (static_cast<uint32_t>(TN >> 3) << 17) |
           (static_cast<uint32_t>(TM >> 4) << 24);
}

// Element offset of (row, k) in the K-major core-matrix layout of a BF16
// operand with K columns.
template <int K>
__device__ __forceinline__ int core_off(int row, int k) {
    return (row >> 3) * (K * 8) + (k >> 3) * 64 + (row & 7) * 8 + (k & 7);
}

template <int M, int K>
__host__ __device__ constexpr size_t smem_bytes() {
    return static_cast<size_t>(128 * K + M * K) * 2 + M * 4 + 16;
}

}  // namespace umma

__device__ int g_umma_error;  // set when a commit-barrier wait ran out

template <int M, int K1, int K2>
__global__ void __launch_bounds__(128)
    linear_fwd_umma(const float* __restrict__ X1, const float* __restrict__ X2, const float* __restrict__ W,
                    const float* __restrict__ b, const float* __restrict__ R, float* __restrict__ Y,
                    float* __restrict__ A, size_t n, int act) {
    constexpr int K = K1 + K2;
    constexpr int TR = 128;                            // rows per tile = UMMA M
    constexpr uint32_t kCols = M < 32 ? 32 : M;        // TMEM columns: a power of two >= 32
    static_assert(K % 16 == 0 && M % 16 == 0 && M >= 16 && M <= 256 && (M & (M - 1)) == 0, "UMMA shape");
    extern __shared__ __align__(1024) unsigned char dsm[];
    __nv_bfloat16* sa = reinterpret_cast<__nv_bfloat16*>(dsm);  // TR x K
    __nv_bfloat16* sw = sa + TR * K;                             // M x K
    float* sbias = reinterpret_cast<float*>(sw + M * K);
    uint64_t* bar = reinterpret_cast<uint64_t*>(sbias + M);
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bar + 1);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         umma::smem_u32(tmem_slot)),
                     "r"(kCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (threadIdx.x == 0) {
        pipe::mbar_init(bar, 1);
        pipe::fence_barrier_init();
    }
    for (int i = threadIdx.x; i < M * K; i += TR) sw[umma::core_off<K>(i / K, i % K)] = __float2bfloat16_rn(W[i]);
    static_assert(K1 % 8 == 0 && K2 % 8 == 0, "a core-matrix row never straddles X1 and X2");
    constexpr int C = K / 8;  // 16-byte core-matrix rows per tile row
    for (int i = threadIdx.x; i < M; i += TR) sbias[i] = b ? b[i] : 0.f;
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = *tmem_slot;
    const uint32_t sa_addr = umma::smem_u32(sa), sw_addr = umma::smem_u32(sw);
    constexpr uint32_t idesc = umma::idesc_bf16<TR, M>();
    const size_t ntiles = (n + TR - 1) / TR;
    uint32_t phase = 0;
    bool issued = false;  // an MMA commit may still be pending on the barrier
    for (size_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const size_t r0 = tile * TR;
        // one 16-byte core-matrix row (8 columns) per thread and pass; eight
        // consecutive threads fill the 8 rows of one core matrix (128
        // contiguous bytes, no bank conflict)
        for (int idx = threadIdx.x; idx < TR * C; idx += TR) {
            const int chunk = (idx >> 3) % C;
            const int rr = (idx & 7) + 8 * ((idx >> 3) / C);
            const size_t row = r0 + rr;
            const int k0 = chunk * 8;
            float4 lo = make_float4(0.f, 0.f, 0.f, 0.f), hi = lo;
            if (row < n) {
                const float* src = k0 < K1 ? X1 + row * K1 + k0 : X2 + row * K2 + (k0 - K1);
                lo = *reinterpret_cast<const float4*>(src);
                hi = *reinterpret_cast<const float4*>(src + 4);
            }
            __nv_bfloat162 q[4] = {__floats2bfloat162_rn(lo.x, lo.y), __floats2bfloat162_rn(lo.z, lo.w),
                                   __floats2bfloat162_rn(hi.x, hi.y), __floats2bfloat162_rn(hi.z, hi.w)};
            *reinterpret_cast<uint4*>(sa + (rr >> 3) * (K * 8) + chunk * 64 + (rr & 7) * 8) =
                *reinterpret_cast<const uint4*>(q);
        }
        // the generic-proxy stores must be visible to the tensor core's reads
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        if (threadIdx.x == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
#pragma unroll
            for (int s = 0; s < K / 16; ++s) {
                const uint64_t ad = umma::smem_desc(sa_addr + s * 256, 128, K * 16);
                const uint64_t bd = umma::smem_desc(sw_addr + s * 256, 128, K * 16);
                asm volatile(
                    "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                    "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem),
                    "l"(ad), "l"(bd), "r"(idesc), "r"(s)
                    : "memory");
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                             umma::smem_u32(bar))
                         : "memory");
        }
        issued = true;
        const bool waited = pipe::mbar_wait(bar, phase, nullptr);
        if (__syncthreads_or(!waited)) {  // the whole CTA leaves together
            if (threadIdx.x == 0) atomicExch(&g_umma_error, 1);
            break;
        }
        issued = false;
        phase ^= 1u;
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const size_t row = r0 + warp * 32 + lane;
#pragma unroll
        for (int c0 = 0; c0 < M; c0 += 16) {
            uint32_t v[16];
            asm volatile(
                "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, "
                "[%16];"
                : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]),
                  "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]),
                  "=r"(v[14]), "=r"(v[15])
                : "r"(tmem + (static_cast<uint32_t>(warp * 32) << 16) + static_cast<uint32_t>(c0)));
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            if (row < n) {
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    float a[4];
#pragma unroll
                    for (int j = 0; j < 4; ++j) {
                        const float z = __uint_as_float(v[4 * q + j]) + sbias[c0 + 4 * q + j];
                        a[j] = act ? fmaxf(z, 0.f) : z;
                    }
                    const size_t off = row * M + c0 + 4 * q;
                    const float4 av = make_float4(a[0], a[1], a[2], a[3]);
                    if (A) *reinterpret_cast<float4*>(A + off) = av;
                    float4 yv = av;
                    if (R) {
                        const float4 rv = *reinterpret_cast<const float4*>(R + off);
                        yv = make_float4(rv.x + av.x, rv.y + av.y, rv.z + av.z, rv.w + av.w);
                    }
                    *reinterpret_cast<float4*>(Y + off) = yv;
                }
            }
        }
        // accumulator read and shared operand consumed before the next tile
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncthreads();
    }
    if (issued && threadIdx.x == 0) pipe::mbar_wait(bar, phase, nullptr);  // let a late commit land
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kCols) : "memory");
    }
}

// Backward of linear_fwd. dZ = dY * act'(A); dX1 += dZ W1, dX2 += dZ W2 (when
// given); per-CTA partial sums of dW (M x K) and db (M) go to `part` at
// blockIdx * (M*K + M).
template <int M, int K1, int K2>
__global__ void __launch_bounds__(256)
    linear_bwd(const float* __restrict__ X1, const float* __restrict__ X2, const float* __restrict__ W,
               const float* __restrict__ A, const float* __restrict__ dY, float* __restrict__ dX1,
               float* __restrict__ dX2, float* __restrict__ part, size_t n, int act, int bf16) {
    constexpr int K = K1 + K2;
    constexpr int ROWS = 16;
    __shared__ float sw[M * K];
    __shared__ float sx[ROWS][K + 1];
    __shared__ float sdz[ROWS][M + 1];
    for (int i = threadIdx.x; i < M * K; i += 256) sw[i] = bf16 ? bfr(W[i]) : W[i];
    const size_t r0 = static_cast<size_t>(blockIdx.x) * ROWS;
    for (int i = threadIdx.x; i < ROWS * K; i += 256) {
        const int rr = i / K, kk = i % K;
        const size_t row = r0 + rr;
        float v = 0.f;
        if (row < n) v = kk < K1 ? X1[row * K1 + kk] : X2[row * K2 + (kk - K1)];
        sx[rr][kk] = v;
    }
    for (int i = threadIdx.x; i < ROWS * M; i += 256) {
        const int rr = i / M, m = i % M;
        const size_t row = r0 + rr;
        float dz = 0.f;
        if (row < n) {
            dz = dY[row * M + m];
            if (act && !(A[row * M + m] > 0.f)) dz = 0.f;
        }
        sdz[rr][m] = dz;
    }
    __syncthreads();
    // input gradients
    for (int i = threadIdx.x; i < ROWS * K; i += 256) {
        const int rr = i / K, kk = i % K;
        const size_t row = r0 + rr;
        if (row >= n) continue;
        float g = 0.f;
#pragma unroll 8
        for (int m = 0; m < M; ++m) g = fmaf(sdz[rr][m], sw[m * K + kk], g);
        if (kk < K1) {
            if (dX1) dX1[row * K1 + kk] += g;
        } else {
            if (dX2) dX2[row * K2 + (kk - K1)] += g;
        }
    }
    // weight gradients of this tile
    float* pw = part + static_cast<size_t>(blockIdx.x) * (M * K + M);
    for (int i = threadIdx.x; i < M * K; i += 256) {
        const int m = i / K, kk = i % K;
        float g = 0.f;
        for (int rr = 0; rr < ROWS; ++rr) g = fmaf(sdz[rr][m], sx[rr][kk], g);
        pw[i] = g;
    }
    for (int m = threadIdx.x; m < M; m += 256) {
        float g = 0.f;
        for (int rr = 0; rr < ROWS; ++rr) g += sdz[rr][m];
        pw[M * K + m] = g;
    }
}

// grad[off + i] += sum over `ntiles` partial records (fixed order).
__global__ void reduce_parts(const float* __restrict__ part, int rec, int ntiles, float* __restrict__ grad,
                             int off_w, int off_b, int nw) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= rec) return;
    double s = 0.0;
    for (int k = 0; k < ntiles; ++k) s += part[static_cast<size_t>(k) * rec + i];
    if (i < nw)
        grad[off_w + i] += static_cast<float>(s);
    else if (off_b >= 0)
        grad[off_b + (i - nw)] += static_cast<float>(s);
}

// One warp per receiving node i: S_i = sum_{j in row i, j != i} relu(Hu_j + e_ij w + c).
__global__ void message_fwd(const uint32_t* __restrict__ rp, const uint32_t* __restrict__ cols,
                            const float* __restrict__ ehat, const float* __restrict__ Hu,
                            const float* __restrict__ w, const float* __restrict__ c, float* __restrict__ S,
                            uint32_t n, int bf16) {
    const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (warp >= n) return;
    const int f0 = lane, f1 = lane + 32;
    const float w0 = bf16 ? bfr(w[f0]) : w[f0], w1 = bf16 ? bfr(w[f1]) : w[f1];
    const float c0 = bf16 ? bfr(c[f0]) : c[f0], c1 = bf16 ? bfr(c[f1]) : c[f1];
    float s0 = 0.f, s1 = 0.f;
    for (uint32_t k = rp[warp]; k < rp[warp + 1]; ++k) {
        const uint32_t j = cols[k];
        if (j == warp) continue;
        const float e = ehat[k];
        s0 += fmaxf(Hu[static_cast<size_t>(j) * H + f0] + e * w0 + c0, 0.f);
        s1 += fmaxf(Hu[static_cast<size_t>(j) * H + f1] + e * w1 + c1, 0.f);
    }
    S[static_cast<size_t>(warp) * H + f0] = s0;
    S[static_cast<size_t>(warp) * H + f1] = s1;
}

// Backward of message_fwd, one warp per sending node j (the pattern is
// symmetric, so row j lists the receivers i and e_ji = e_ij):
// dHu_j = sum_i dS_i * [Hu_j + e_ij w + c > 0]; partial dw, dc per warp into
// part[warp * 2H].
__global__ void message_bwd(const uint32_t* __restrict__ rp, const uint32_t* __restrict__ cols,
                            const float* __restrict__ ehat, const float* __restrict__ Hu,
                            const float* __restrict__ w, const float* __restrict__ c,
                            const float* __restrict__ dS, float* __restrict__ dHu, float* __restrict__ part,
                            uint32_t n, int bf16) {
    const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (warp >= n) return;
    const int f0 = lane, f1 = lane + 32;
    const float w0 = bf16 ? bfr(w[f0]) : w[f0], w1 = bf16 ? bfr(w[f1]) : w[f1];
    const float c0 = bf16 ? bfr(c[f0]) : c[f0], c1 = bf16 ? bfr(c[f1]) : c[f1];
    const float u0 = Hu[static_cast<size_t>(warp) * H + f0], u1 = Hu[static_cast<size_t>(warp) * H + f1];
    float g0 = 0.f, g1 = 0.f, dw0 = 0.f, dw1 = 0.f, dc0 = 0.f, dc1 = 0.f;
    for (uint32_t k = rp[warp]; k < rp[warp + 1]; ++k) {
        const uint32_t i = cols[k];
        if (i == warp) continue;
        const float e = ehat[k];
        const float d0 = (u0 + e * w0 + c0 > 0.f) ? dS[static_cast<size_t>(i) * H + f0] : 0.f;
        const float d1 = (u1 + e * w1 + c1 > 0.f) ? dS[static_cast<size_t>(i) * H + f1] : 0.f;
        g0 += d0;
        g1 += d1;
        dw0 += d0 * e;
        dw1 += d1 * e;
        dc0 += d0;
        dc1 += d1;
    }
    dHu[static_cast<size_t>(warp) * H + f0] = g0;
    dHu[static_cast<size_t>(warp) * H + f1] = g1;
    float* p = part + static_cast<size_t>(warp) * 2 * H;
    p[f0] = dw0;
    p[f1] = dw1;
    p[H + f0] = dc0;
    p[H + f1] = dc1;
}

__device__ __forceinline__ float softplus(float z) { return z > 20.f ? z : log1pf(expf(z)); }
__device__ __forceinline__ float sigmoid(float z) { return 1.f / (1.f + expf(-z)); }

// Output layer, one warp per row i of L = tril(A) (lane = output unit o < 32):
// g_ii = softplus(w_d . h_i + b_d); g_ij = w_o . relu(Hp_i + Hq_j + e r + t) + b_o.
__global__ void output_fwd(const uint32_t* __restrict__ Lrp, const uint32_t* __restrict__ Lcol,
                           const float* __restrict__ Le, const float* __restrict__ Hh,
                           const float* __restrict__ Hp, const float* __restrict__ Hq,
                           const float* __restrict__ prm, Offsets o, float* __restrict__ g, uint32_t n,
                           int bf16) {
    const uint32_t i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (i >= n) return;
    auto W = [&](int k) { return bf16 ? bfr(prm[k]) : prm[k]; };
    const float rr = W(o.r + lane), tt = W(o.t + lane), wo = W(o.w_o + lane), bo = W(o.b_o);
    const float hp = Hp[static_cast<size_t>(i) * HO + lane];
    for (uint32_t k = Lrp[i]; k < Lrp[i + 1]; ++k) {
        const uint32_t j = Lcol[k];
        float val;
        if (j == i) {
            float z = W(o.w_d + lane) * Hh[static_cast<size_t>(i) * H + lane] +
                      W(o.w_d + lane + 32) * Hh[static_cast<size_t>(i) * H + lane + 32];
            z = dev::warp_sum(z) + W(o.b_d);
            val = softplus(z);
        } else {
            const float pre = hp + Hq[static_cast<size_t>(j) * HO + lane] + Le[k] * rr + tt;
            val = dev::warp_sum(wo * fmaxf(pre, 0.f)) + bo;
        }
        if (lane == 0) g[k] = val;
    }
}

// Backward of output_fwd over rows i: dh_i (diagonal part), dHp_i, and the
// per-warp partial parameter gradients [r, t, w_o, b_o, w_d(64), b_d].
constexpr int kOutPart = HO * 3 + 1 + H + 1;
__global__ void output_bwd_rows(const uint32_t* __restrict__ Lrp, const uint32_t* __restrict__ Lcol,
                                const float* __restrict__ Le, const float* __restrict__ Hh,
                                const float* __restrict__ Hp, const float* __restrict__ Hq,
                                const float* __restrict__ prm, Offsets o, const float* __restrict__ dg,
                                float* __restrict__ dH, float* __restrict__ dHp, float* __restrict__ part,
                                uint32_t n, int bf16) {
    const uint32_t i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (i >= n) return;
    auto W = [&](int k) { return bf16 ? bfr(prm[k]) : prm[k]; };
    const float rr = W(o.r + lane), tt = W(o.t + lane), wo = W(o.w_o + lane);
    const float hp = Hp[static_cast<size_t>(i) * HO + lane];
    float dhp = 0.f, dr = 0.f, dt = 0.f, dwo = 0.f, dbo = 0.f, dwd0 = 0.f, dwd1 = 0.f, dbd = 0.f, dh0 = 0.f,
          dh1 = 0.f;
    const float h0 = Hh[static_cast<size_t>(i) * H + lane], h1 = Hh[static_cast<size_t>(i) * H + lane + 32];
    for (uint32_t k = Lrp[i]; k < Lrp[i + 1]; ++k) {
        const uint32_t j = Lcol[k];
        const float d = dg[k];
        if (j == i) {
            const float wd0 = W(o.w_d + lane), wd1 = W(o.w_d + lane + 32);
            const float z = dev::warp_sum(wd0 * h0 + wd1 * h1) + W(o.b_d);
            const float dz = d * sigmoid(z);
            dh0 += dz * wd0;
            dh1 += dz * wd1;
            dwd0 += dz * h0;
            dwd1 += dz * h1;
            dbd += dz;
        } else {
            const float pre = hp + Hq[static_cast<size_t>(j) * HO + lane] + Le[k] * rr + tt;
            const float a = fmaxf(pre, 0.f);
            dwo += d * a;
            dbo += d;
            const float dp = pre > 0.f ? d * wo : 0.f;
            dhp += dp;
            dr += dp * Le[k];
            dt += dp;
        }
    }
    dHp[static_cast<size_t>(i) * HO + lane] = dhp;
    dH[static_cast<size_t>(i) * H + lane] += dh0;
    dH[static_cast<size_t>(i) * H + lane + 32] += dh1;
    float* p = part + static_cast<size_t>(i) * kOutPart;
    p[lane] = dr;
    p[HO + lane] = dt;
    p[2 * HO + lane] = dwo;
    if (lane == 0) p[3 * HO] = dbo;  // lanes agree on dbo
    p[3 * HO + 1 + lane] = dwd0;
    p[3 * HO + 1 + lane + 32] = dwd1;
    if (lane == 0) p[3 * HO + 1 + H] = dbd;
}

// dHq_j = sum over rows i > j of L holding (i, j): dg_ij w_o [pre_ij > 0],
// gathered through the transposed pattern (LTrp, LTrow, LTidx -> entry of L).
__global__ void output_bwd_cols(const uint32_t* __restrict__ LTrp, const uint32_t* __restrict__ LTrow,
                                const uint32_t* __restrict__ LTidx, const float* __restrict__ Le,
                                const float* __restrict__ Hp, const float* __restrict__ Hq,
                                const float* __restrict__ prm, Offsets o, const float* __restrict__ dg,
                                float* __restrict__ dHq, uint32_t n, int bf16) {
    const uint32_t j = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (j >= n) return;
    auto W = [&](int k) { return bf16 ? bfr(prm[k]) : prm[k]; };
    const float rr = W(o.r + lane), tt = W(o.t + lane), wo = W(o.w_o + lane);
    const float hq = Hq[static_cast<size_t>(j) * HO + lane];
    float acc = 0.f;
    for (uint32_t k = LTrp[j]; k < LTrp[j + 1]; ++k) {
        const uint32_t i = LTrow[k];
        if (i == j) continue;
        const uint32_t e = LTidx[k];
        const float pre = Hp[static_cast<size_t>(i) * HO + lane] + hq + Le[e] * rr + tt;
        if (pre > 0.f) acc += dg[e] * wo;
    }
    dHq[static_cast<size_t>(j) * HO + lane] = acc;
}

// Kaporin loss, pass 1: per row tr_i = g_i^T B_i g_i and log g_ii; grid sums.
__global__ void kaporin_sum(const uint32_t* __restrict__ Lrp, const uint32_t* __restrict__ Boff,
                            const float* __restrict__ B, const float* __restrict__ g, uint32_t n,
                            double* parts, uint32_t* ticket, double* out) {
    double acc[2] = {0.0, 0.0};
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t k0 = Lrp[i], m = Lrp[i + 1] - k0;
        const float* Bi = B + Boff[i];
        double t = 0.0;
        for (uint32_t a = 0; a < m; ++a) {
            double s = 0.0;
            for (uint32_t c = 0; c < m; ++c) s += static_cast<double>(Bi[a * m + c]) * g[k0 + c];
            t += s * g[k0 + a];
        }
        acc[0] += t;
        acc[1] += log(static_cast<double>(g[k0 + m - 1]));  // diagonal is last (sorted columns)
    }
    double tot[2];
    if (dev::grid_reduce_last<2>(acc, parts, ticket, tot) && threadIdx.x == 0) {
        out[0] = tot[0];
        out[1] = tot[1];
    }
}

// Kaporin loss, pass 2: dL/dg_i = (2/tr) B_i g_i - (2/n)/g_ii on the diagonal.
__global__ void kaporin_grad(const uint32_t* __restrict__ Lrp, const uint32_t* __restrict__ Boff,
                             const float* __restrict__ B, const float* __restrict__ g, uint32_t n,
                             const double* sums, float* __restrict__ dg) {
    const double tr = sums[0];
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t k0 = Lrp[i], m = Lrp[i + 1] - k0;
        const float* Bi = B + Boff[i];
        for (uint32_t a = 0; a < m; ++a) {
            double s = 0.0;
            for (uint32_t c = 0; c < m; ++c) s += static_cast<double>(Bi[a * m + c]) * g[k0 + c];
            double d = 2.0 * s / tr;
            if (a == m - 1) d -= 2.0 / (static_cast<double>(n) * g[k0 + a]);
            dg[k0 + a] = static_cast<float>(d);
        }
    }
}

// y = G v (rows of L) or y = G^T v (rows of L^T); warp per row, FP32.
__global__ void lspmv(const uint32_t* __restrict__ rp, const uint32_t* __restrict__ idx,
                      const uint32_t* __restrict__ vidx, const float* __restrict__ g,
                      const float* __restrict__ v, float* __restrict__ y, uint32_t n) {
    const uint32_t row = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (row >= n) return;
    float s = 0.f;
    for (uint32_t k = rp[row] + lane; k < rp[row + 1]; k += 32) s += g[vidx ? vidx[k] : k] * v[idx[k]];
    s = dev::warp_sum(s);
    if (lane == 0) y[row] = s;
}

// y = A_hat v with the scaled values (ehat) on A's pattern (diagonal = 1).
__global__ void ahat_spmv(const uint32_t* __restrict__ rp, const uint32_t* __restrict__ cols,
                          const float* __restrict__ ehat, const float* __restrict__ v, float* __restrict__ y,
                          uint32_t n) {
    const uint32_t row = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (row >= n) return;
    float s = 0.f;
    for (uint32_t k = rp[row] + lane; k < rp[row + 1]; k += 32) s += ehat[k] * v[cols[k]];
    s = dev::warp_sum(s);
    if (lane == 0) y[row] = s;
}

// Probe loss pieces. res = v - r scaled: dv = coef * (v - r), and the sum of
// (v - r)^2 / ||r||^2 goes to `out` through a grid sum.
// The probe's weights come from its squared norm rr on the device:
// coef = 2 lambda / (K rr), inv_rr = lambda / (K rr) (the same double
// expressions the host evaluated before); a probe with rr not > 0 adds
// nothing (dv = 0, no loss term).
__global__ void probe_residual(const float* __restrict__ v, const float* __restrict__ r, const double* rr_p,
                               double lambda, int K, float* __restrict__ dv, uint32_t n, double* parts,
                               uint32_t* ticket, double* out) {
    const double rr = *rr_p;
    const bool on = rr > 0.0;
    const float coef = on ? static_cast<float>(2.0 * lambda / (K * rr)) : 0.f;
    const float inv_rr = on ? static_cast<float>(lambda / (K * rr)) : 0.f;
    double acc[1] = {0.0};
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float d = v[i] - r[i];
        dv[i] = on ? coef * d : 0.f;
        if (on) acc[0] += static_cast<double>(d) * d * inv_rr;
    }
    double tot[1];
    if (dev::grid_reduce_last<1>(acc, parts, ticket, tot) && threadIdx.x == 0) out[0] += tot[0];
}

// dg_ij += dv_j u_i + du_i w_j over the entries of L.
__global__ void probe_grad(const uint32_t* __restrict__ Lrp, const uint32_t* __restrict__ Lcol,
                           const float* __restrict__ dv, const float* __restrict__ u,
                           const float* __restrict__ du, const float* __restrict__ w, float* __restrict__ dg,
                           uint32_t n, const double* rr_p) {
    if (!(*rr_p > 0.0)) return;  // a probe without a positive norm contributes nothing
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        for (uint32_t k = Lrp[i]; k < Lrp[i + 1]; ++k) {
            const uint32_t j = Lcol[k];
            dg[k] += dv[j] * u[i] + du[i] * w[j];
        }
}

// g *= scale (the data-parallel mean of summed gradients).
__global__ void scale_kernel(float* g, uint32_t n, float scale) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) g[i] *= scale;
}

__global__ void adam_step(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m,
                          float* __restrict__ v, int n, float lr, float b1, float b2, float eps, float c1,
                          float c2) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

// G values for the solver: g_ij = g_hat_ij / sqrt(a_jj) in L order, as FP32,
// BF16 and FP64.
__global__ void export_factor(const uint32_t* __restrict__ Lrp, const uint32_t* __restrict__ Lcol,
                              const float* __restrict__ ghat, const double* __restrict__ dinvs,
                              float* __restrict__ G32, __nv_bfloat16* __restrict__ G16,
                              double* __restrict__ G64, uint32_t n) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        for (uint32_t k = Lrp[i]; k < Lrp[i + 1]; ++k) {
            const double v = static_cast<double>(ghat[k]) * dinvs[Lcol[k]];
            G32[k] = static_cast<float>(v);
            G16[k] = __double2bfloat16(v);
            G64[k] = v;
        }
}

// The same values in L^T order (rows of G^T).
__global__ void gather_transpose(const uint32_t* __restrict__ LTidx, const float* __restrict__ G32,
                                 const __nv_bfloat16* __restrict__ G16, const double* __restrict__ G64,
                                 float* __restrict__ GT32, __nv_bfloat16* __restrict__ GT16,
                                 double* __restrict__ GT64, uint32_t nnzL) {
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < nnzL; k += gridDim.x * blockDim.x) {
        const uint32_t s = LTidx[k];
        GT32[k] = G32[s];
        GT16[k] = G16[s];
        GT64[k] = G64[s];
    }
}

// node features f = [1, sum_{j != i} |a_hat_ij|, deg_i / 8, 0]
__global__ void node_features(const uint32_t* __restrict__ rp, const uint32_t* __restrict__ cols,
                              const float* __restrict__ ehat, float* __restrict__ F, uint32_t n) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        float s = 0.f;
        uint32_t deg = 0;
        for (uint32_t k = rp[i]; k < rp[i + 1]; ++k)
            if (cols[k] != i) {
                s += fabsf(ehat[k]);
                ++deg;
            }
        F[static_cast<size_t>(i) * NF + 0] = 1.f;
        F[static_cast<size_t>(i) * NF + 1] = s;
        F[static_cast<size_t>(i) * NF + 2] = deg * 0.125f;
        F[static_cast<size_t>(i) * NF + 3] = 0.f;
    }
}

// ---- graph of a matrix, built on the device

// Status bits of the graph build.
enum : uint32_t {
    kGraphNotSpd = 1,     // a row without a positive diagonal entry
    kGraphBadRows = 2,    // columns unsorted, repeated or out of range, or row_pointer[0] != 0
    kGraphAsymmetric = 4  // the pattern is not symmetric (an entry (i, j) without (j, i))
};

// Per row i of A: 1 / sqrt(a_ii), the number of entries with column <= i (a
// row of L = tril(A)) into Lc[i] and with column >= i (a row of L^T, on the
// symmetric pattern) into Uc[i]; checks sortedness and the diagonal.
__global__ void graph_rows(const uint32_t* __restrict__ rp, const uint32_t* __restrict__ cols,
                           const double* __restrict__ vals, uint32_t n, double* __restrict__ dinvs,
                           uint32_t* __restrict__ Lc, uint32_t* __restrict__ Uc, uint32_t* __restrict__ info) {
    uint32_t bad = 0, maxl = 0;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t b = rp[i], e = rp[i + 1];
        if (i == 0 && b != 0) bad |= kGraphBadRows;
        if (e < b) {
            bad |= kGraphBadRows;
            Lc[i] = Uc[i] = 0;
            dinvs[i] = 0.0;
            continue;
        }
        double diag = 0.0;
        uint32_t lc = 0, uc = 0, prev = 0;
        for (uint32_t k = b; k < e; ++k) {
            const uint32_t j = cols[k];
            if (j >= n || (k > b && j <= prev)) bad |= kGraphBadRows;
            prev = j;
            if (j < i) {
                ++lc;
            } else if (j == i) {
                ++lc;
                ++uc;
                diag = vals[k];
            } else {
                ++uc;
            }
        }
        if (!(diag > 0.0)) bad |= kGraphNotSpd;
        dinvs[i] = diag > 0.0 ? 1.0 / sqrt(diag) : 0.0;
        Lc[i] = lc;
        Uc[i] = uc;
        maxl = lc > maxl ? lc : maxl;
    }
    if (bad) atomicOr(info, bad);
    if (maxl) atomicMax(info + 1, maxl);
}

// Scaled values a_hat_ij = a_ij / sqrt(a_ii a_jj) on A's pattern; the rows of
// L (the first Lrp[i+1] - Lrp[i] entries of A's sorted row i) with their
// scaled values; the rows of L^T (the entries of A's row i with column >= i:
// by symmetry, the rows of L holding column i, in increasing order) with the
// position in L of each (the rank of column i in A's row j, a binary search).
__global__ void graph_fill(const uint32_t* __restrict__ rp, const uint32_t* __restrict__ cols,
                           const double* __restrict__ vals, uint32_t n, const double* __restrict__ dinvs,
                           const uint32_t* __restrict__ Lrp, const uint32_t* __restrict__ LTrp,
                           float* __restrict__ ehat, uint32_t* __restrict__ Lcol, float* __restrict__ Le,
                           uint32_t* __restrict__ LTrow, uint32_t* __restrict__ LTidx, uint32_t* __restrict__ info) {
    uint32_t bad = 0;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t b = rp[i], e = rp[i + 1];
        const double di = dinvs[i];
        uint32_t l = Lrp[i], u = LTrp[i];
        const uint32_t lend = Lrp[i + 1], uend = LTrp[i + 1];
        for (uint32_t k = b; k < e; ++k) {
            const uint32_t j = cols[k];
            const float eh = static_cast<float>(vals[k] * di * dinvs[j]);
            ehat[k] = eh;
            if (j <= i && l < lend) {
                Lcol[l] = j;
                Le[l] = eh;
                ++l;
            }
            if (j >= i && u < uend) {
                // entry (j, i) of L: column i in A's row j, lower entries first
                const uint32_t jb = rp[j], je = rp[j + 1];
                uint32_t lo = jb, hi = je;
                while (lo < hi) {
                    const uint32_t mid = lo + (hi - lo) / 2;
                    if (cols[mid] < i)
                        lo = mid + 1;
                    else
                        hi = mid;
                }
                if (lo == je || cols[lo] != i) {
                    bad |= kGraphAsymmetric;
                    LTidx[u] = Lrp[j];
                } else {
                    LTidx[u] = Lrp[j] + (lo - jb);
                }
                LTrow[u] = j;
                ++u;
            }
        }
    }
    if (bad) atomicOr(info, bad);
}

// Squared norm of one probe vector (a grid sum into out).
__global__ void probe_norm(const float* __restrict__ v, uint32_t n, double* parts, uint32_t* ticket,
                           double* out) {
    double acc[1] = {0.0};
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        acc[0] += static_cast<double>(v[i]) * v[i];
    double tot[1];
    if (dev::grid_reduce_last<1>(acc, parts, ticket, tot) && threadIdx.x == 0) out[0] = tot[0];
}

// m_i^2 per row (the size of the local block B_i), for the block offsets.
__global__ void block_sizes(const uint32_t* __restrict__ Lrp, uint32_t n, uint32_t* __restrict__ out) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t m = Lrp[i + 1] - Lrp[i];
        out[i] = m * m;
    }
}

// Local blocks of the Kaporin loss: B_i = A_hat[P_i, P_i] with P_i the
// columns of row i of L (a binary search in A's row P_a for column P_b).
__global__ void block_fill(const uint32_t* __restrict__ rp, const uint32_t* __restrict__ cols,
                           const float* __restrict__ ehat, const uint32_t* __restrict__ Lrp,
                           const uint32_t* __restrict__ Lcol, const uint32_t* __restrict__ Boff, uint32_t n,
                           float* __restrict__ B) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t k0 = Lrp[i], m = Lrp[i + 1] - k0;
        float* Bi = B + Boff[i];
        for (uint32_t a = 0; a < m; ++a) {
            const uint32_t r = Lcol[k0 + a];
            const uint32_t rb = rp[r], re = rp[r + 1];
            for (uint32_t c = 0; c < m; ++c) {
                const uint32_t col = Lcol[k0 + c];
                uint32_t lo = rb, hi = re;
                while (lo < hi) {
                    const uint32_t mid = lo + (hi - lo) / 2;
                    if (cols[mid] < col)
                        lo = mid + 1;
                    else
                        hi = mid;
                }
                Bi[a * m + c] = (lo < re && cols[lo] == col) ? ehat[lo] : 0.f;
            }
        }
    }
}

// ------------------------------------------------------------- host side

constexpr int kRows = 16;  // rows per CTA of linear_fwd / linear_bwd

uint32_t nblk(size_t n, int per) { return static_cast<uint32_t>((n + per - 1) / per); }
uint32_t warps_grid(size_t n) { return static_cast<uint32_t>((n * 32 + 255) / 256); }

template <typename P>
cudaError_t dalloc(P*& p, size_t count) {
    return cudaMalloc(reinterpret_cast<void**>(&p), count * sizeof(P) + 16);
}

uint64_t fnv1a(const void* data, size_t bytes, uint64_t h = 1469598103934665603ull) {
    const unsigned char* c = static_cast<const unsigned char*>(data);
    for (size_t i = 0; i < bytes; ++i) {
        h ^= c[i];
        h *= 1099511628211ull;
    }
    return h;
}

// Graph of one matrix: A's pattern with scaled values, L = tril(A), L^T,
// the local blocks of the loss, and the exported factor.
struct Graph {
    uint32_t n = 0, nnz = 0, nnzL = 0;
    uint32_t cap_n = 0, cap_nnz = 0;  // sizes the buffers were allocated for (rows, entries of A)
    uint32_t maxL = 0;                // longest row of L
    size_t nB = 0, cap_B = 0;         // local blocks (training only, built on first use)
    bool blocks_built = false;
    uint32_t* scan_part = nullptr;    // block totals of the device scans
    uint32_t* info = nullptr;         // [0] status bits, [1] longest row of L, [2..3] sizes read back
    const uint32_t* rp = nullptr;   // A's arrays (user memory)
    const uint32_t* cols = nullptr;
    float* ehat = nullptr;          // a_hat on A's pattern
    double* dinvs = nullptr;        // 1 / sqrt(a_ii)
    uint32_t *Lrp = nullptr, *Lcol = nullptr;
    float* Le = nullptr;
    uint32_t *LTrp = nullptr, *LTrow = nullptr, *LTidx = nullptr;
    uint32_t* Boff = nullptr;
    float* B = nullptr;
    float* F = nullptr;
    // activations
    float* Hs[NL + 1] = {};
    float *Hu[NL] = {}, *S[NL] = {}, *Au[NL] = {};
    float *Hp = nullptr, *Hq = nullptr, *g = nullptr, *dg = nullptr;
    float *dH = nullptr, *dHn = nullptr, *dS = nullptr, *dHu = nullptr, *dHp = nullptr, *dHq = nullptr;
    float* part = nullptr;
    size_t part_floats = 0;
    float *pw = nullptr, *pu = nullptr, *pv = nullptr, *pdv = nullptr, *pdu = nullptr;
    double* red = nullptr;  // [0..3] results, [8..] partials
    uint32_t* ticket = nullptr;
    // exported factor (L order) and its transpose (L^T order)
    float *G32 = nullptr, *GT32 = nullptr;
    __nv_bfloat16 *G16 = nullptr, *GT16 = nullptr;
    double *G64 = nullptr, *GT64 = nullptr;
    bool built = false;
    int device = 0;
    // CSR-Adaptive metas of the patterns of G (L) and G^T (L^T), so the
    // solvers apply the factor with the row-block kernels
    matrix_meta* metaL = nullptr;
    matrix_meta* metaLT = nullptr;
    // The buffers above live in two allocations: `arena` holds what the graph
    // and the factor build need (patterns, features, the factor copies and
    // four activation buffers the layers share: Hs[l] alternates between two,
    // every layer's Hu and S are one each); `train_arena`, made on the first
    // training call for the graph, gives every layer its own activations and
    // adds Au and the gradient buffers. B (Kaporin blocks) is separate.
    void* arena = nullptr;
    void* train_arena = nullptr;

    void release() {
        delete metaL;
        delete metaLT;
        if (arena) cudaFree(arena);
        if (train_arena) cudaFree(train_arena);
        if (B) cudaFree(B);
        *this = Graph();
    }
};

}  // namespace gnn
}  // namespace clsp

using namespace clsp;
using namespace clsp::gnn;

// Host copy of a matrix the network was set to, with the device addresses it
// came from: the key of the graph cache (contents compared bit for bit, so a
// matrix changed in place is never taken for the cached one).
struct HostCsr {
    const void* ptrs[3] = {};
    uint32_t n = 0, nnz = 0;
    std::vector<uint32_t> rp, cols;
    std::vector<double> vals;
    bool same(const HostCsr& o) const {
        return ptrs[0] == o.ptrs[0] && ptrs[1] == o.ptrs[1] && ptrs[2] == o.ptrs[2] && n == o.n && nnz == o.nnz &&
               rp == o.rp && cols == o.cols &&
               std::memcmp(vals.data(), o.vals.data(), vals.size() * sizeof(double)) == 0;
    }
};

struct CachedGraph {
    HostCsr key;
    Graph gr;
};

// The learned preconditioner object: network parameters, optimiser state, the
// graph of the matrix it is set to, and the graphs of up to kGraphCache
// matrices it was set to before (training cycles through a set of matrices;
// each graph takes tens of allocations and host passes to build).
struct _clsparseB200Spai {
    Offsets o;
    float* prm = nullptr;   // FP32 master weights
    float* grad = nullptr;
    float* m = nullptr;
    float* v = nullptr;
    int step = 0;
    int device = 0;
    Graph gr;
    HostCsr cur;                       // the matrix gr was built from
    std::vector<CachedGraph> cache;    // least recently used first
    ~_clsparseB200Spai() {
        gr.release();
        for (CachedGraph& e : cache) e.gr.release();
        if (prm) cudaFree(prm);
        if (grad) cudaFree(grad);
        if (m) cudaFree(m);
        if (v) cudaFree(v);
    }
};

namespace {

// Graphs of matrices up to kGraphCacheRows rows are kept for reuse, at most
// kGraphCache of them (CLSPARSE_B200_SPAI_CACHE=0: none).
constexpr size_t kGraphCache = 8;
constexpr uint32_t kGraphCacheRows = 65536;

bool graph_cache_enabled() {
    const char* e = std::getenv("CLSPARSE_B200_SPAI_CACHE");
    return !(e && e[0] == '0' && e[1] == '\0');
}

// Copies A's arrays to the host (the graph is built there).
clsparseStatus read_host_csr(const clsparseCsrMatrix* A, clsparseControl c, HostCsr& h) {
    h.n = A->num_rows;
    h.nnz = A->num_nonzeros;
    h.ptrs[0] = dev_ptr<const uint32_t>(A->row_pointer, A->off_row_pointer);
    h.ptrs[1] = dev_ptr<const uint32_t>(A->col_indices, A->off_col_indices);
    h.ptrs[2] = dev_ptr<const double>(A->values, A->off_values);
    h.rp.resize(size_t(h.n) + 1);
    h.cols.resize(h.nnz);
    h.vals.resize(h.nnz);
    cudaStream_t s = c->stream;
    cudaMemcpyAsync(h.rp.data(), h.ptrs[0], (size_t(h.n) + 1) * 4, cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(h.cols.data(), h.ptrs[1], size_t(h.nnz) * 4, cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(h.vals.data(), h.ptrs[2], size_t(h.nnz) * 8, cudaMemcpyDeviceToHost, s);
    return cudaStreamSynchronize(s) == cudaSuccess ? clsparseSuccess : clsparseInvalidMemObject;
}

// Allocates the graph's buffers for n rows and nnz entries of A (L and L^T
// hold at most nnz entries), or keeps the present ones when they are large
// enough: a network set to one matrix after another of the same size
// allocates once. The local blocks of the loss are allocated on first use.
// Lays buffers out from `base` (nullptr: only sizes them), 256-byte aligned.
struct Carver {
    char* base;
    size_t off = 0;
    template <typename T>
    void take(T*& p, size_t count) {
        off = (off + 255) & ~size_t(255);
        p = base ? reinterpret_cast<T*>(base + off) : nullptr;
        off += count * sizeof(T);
    }
};

// One allocation for the layout `lay` describes: sized by a dry run, then
// laid out from the new block.
template <typename F>
bool allocate_laid_out(void*& block, F lay) {
    Carver dry{nullptr};
    lay(dry);
    if (cudaMalloc(&block, dry.off) != cudaSuccess) {
        cudaGetLastError();
        block = nullptr;
        return false;
    }
    Carver c{static_cast<char*>(block)};
    lay(c);
    return true;
}

bool ensure_graph_buffers(Graph& gr, uint32_t n, uint32_t nnz) {
    if (gr.arena != nullptr && gr.cap_n >= n && gr.cap_nnz >= nnz) return true;
    gr.release();
    const size_t nl = nnz, nh = size_t(n) * H, nho = size_t(n) * HO;
    float *act0 = nullptr, *act1 = nullptr, *hu = nullptr, *sb = nullptr;
    const bool ok = allocate_laid_out(gr.arena, [&](Carver& c) {
        c.take(gr.ehat, nnz);
        c.take(gr.dinvs, n);
        c.take(gr.Lrp, size_t(n) + 1);
        c.take(gr.Lcol, nl);
        c.take(gr.Le, nl);
        c.take(gr.LTrp, size_t(n) + 1);
        c.take(gr.LTrow, nl);
        c.take(gr.LTidx, nl);
        c.take(gr.Boff, size_t(n) + 1);
        c.take(gr.F, size_t(n) * NF);
        c.take(gr.scan_part, scan::parts_for(n) + 1);
        c.take(gr.info, 4);
        c.take(act0, nh);
        c.take(act1, nh);
        c.take(hu, nh);
        c.take(sb, nh);
        c.take(gr.Hp, nho);
        c.take(gr.Hq, nho);
        c.take(gr.g, nl);
        c.take(gr.red, 8 + 2 * kMaxReduceCtas);
        c.take(gr.ticket, 4);
        c.take(gr.G32, nl);
        c.take(gr.GT32, nl);
        c.take(gr.G16, nl);
        c.take(gr.GT16, nl);
        c.take(gr.G64, nl);
        c.take(gr.GT64, nl);
    });
    if (!ok) {
        gr.release();
        return false;
    }
    for (int l = 0; l <= NL; ++l) gr.Hs[l] = (l & 1) ? act1 : act0;
    for (int l = 0; l < NL; ++l) {
        gr.Hu[l] = hu;
        gr.S[l] = sb;
    }
    gr.cap_n = n;
    gr.cap_nnz = nnz;
    return true;
}

// The training layout of the current graph: every layer's activations kept
// for the backward pass, the pre-activations Au and the gradient buffers.
bool ensure_training_buffers(Graph& gr) {
    if (gr.train_arena != nullptr) return true;
    const size_t n = gr.cap_n, nl = gr.cap_nnz, nh = n * H, nho = n * HO;
    const size_t tiles = nblk(n, kRows);
    const size_t part_floats = std::max({tiles * size_t(H * 2 * H + H), n * 2 * H, n * kOutPart});
    Graph t = gr;  // laid out on a copy, adopted only when the allocation succeeded
    const bool ok = allocate_laid_out(t.train_arena, [&](Carver& c) {
        for (int l = 0; l <= NL; ++l) c.take(t.Hs[l], nh);
        for (int l = 0; l < NL; ++l) {
            c.take(t.Hu[l], nh);
            c.take(t.S[l], nh);
            c.take(t.Au[l], nh);
        }
        c.take(t.dg, nl);
        c.take(t.dH, nh);
        c.take(t.dHn, nh);
        c.take(t.dS, nh);
        c.take(t.dHu, nh);
        c.take(t.dHp, nho);
        c.take(t.dHq, nho);
        c.take(t.part, part_floats);
        c.take(t.pw, n);
        c.take(t.pu, n);
        c.take(t.pv, n);
        c.take(t.pdv, n);
        c.take(t.pdu, n);
    });
    if (!ok) return false;
    t.part_floats = part_floats;
    gr = t;
    return true;
}

// Reads the graph build's status words (and the two sizes copied next to
// them) back to the host.
bool read_info(Graph& gr, cudaStream_t s, uint32_t (&h)[4]) {
    return cudaMemcpyAsync(h, gr.info, sizeof(h), cudaMemcpyDeviceToHost, s) == cudaSuccess &&
           cudaStreamSynchronize(s) == cudaSuccess;
}

// Builds the graph structures of an SPD matrix A (FP64 values, sorted
// columns, every diagonal present, symmetric pattern, row_pointer[0] == 0) on
// the device: the scaled values, L = tril(A) and L^T with the positions of
// L^T's entries in L, the node features, and the CSR-Adaptive metas of L and
// L^T. The work is a row pass, two scans, a second row pass (no host copy of
// A); the host reads back a few words to size and check the result.
clsparseStatus build_graph(_clsparseB200Spai* net, const clsparseCsrMatrix* A, clsparseControl c) {
    Graph& gr = net->gr;
    const uint32_t n = A->num_rows, nnz = A->num_nonzeros;
    cudaStream_t s = c->stream;
    delete gr.metaL;
    delete gr.metaLT;
    gr.metaL = gr.metaLT = nullptr;
    gr.built = false;
    gr.blocks_built = false;
    if (!ensure_graph_buffers(gr, n, nnz)) return clsparseOutOfResources;
    gr.n = n;
    gr.nnz = nnz;
    gr.rp = dev_ptr<const uint32_t>(A->row_pointer, A->off_row_pointer);
    gr.cols = dev_ptr<const uint32_t>(A->col_indices, A->off_col_indices);
    const double* vals = dev_ptr<const double>(A->values, A->off_values);
    gr.device = c->device;
    const uint32_t grid = std::min<uint32_t>(nblk(n, 256), static_cast<uint32_t>(std::max(c->sm_count, 1)) * 8);
    cudaMemsetAsync(gr.info, 0, 16, s);
    cudaMemsetAsync(gr.Lrp, 0, 4, s);
    cudaMemsetAsync(gr.LTrp, 0, 4, s);
    graph_rows<<<grid, 256, 0, s>>>(gr.rp, gr.cols, vals, n, gr.dinvs, gr.Lrp + 1, gr.LTrp + 1, gr.info);
    scan::inclusive_u32(gr.Lrp + 1, n, gr.scan_part, s);
    scan::inclusive_u32(gr.LTrp + 1, n, gr.scan_part, s);
    cudaMemcpyAsync(gr.info + 2, gr.Lrp + n, 4, cudaMemcpyDeviceToDevice, s);
    cudaMemcpyAsync(gr.info + 3, gr.LTrp + n, 4, cudaMemcpyDeviceToDevice, s);
    uint32_t h[4];
    if (cudaGetLastError() != cudaSuccess || !read_info(gr, s, h)) return clsparseInvalidKernelExecution;
    // not SPD, unsorted or out-of-range columns, or an asymmetric pattern
    if (h[0] != 0 || h[2] != h[3] || h[2] > nnz) return clsparseInvalidValue;
    gr.nnzL = h[2];
    gr.maxL = h[1];
    graph_fill<<<grid, 256, 0, s>>>(gr.rp, gr.cols, vals, n, gr.dinvs, gr.Lrp, gr.LTrp, gr.ehat, gr.Lcol, gr.Le,
                                    gr.LTrow, gr.LTidx, gr.info);
    cudaMemsetAsync(gr.ticket, 0, 16, s);
    node_features<<<nblk(n, 256), 256, 0, s>>>(gr.rp, gr.cols, gr.ehat, gr.F, n);
    if (cudaGetLastError() != cudaSuccess || !read_info(gr, s, h)) return clsparseInvalidKernelExecution;
    if (h[0] != 0) return clsparseInvalidValue;
    // The CSR-Adaptive metas of the patterns of G and G^T are made when a
    // CSR solve first needs them (spai_ensure_metas): their row blocks are
    // computed on the host, and the banded inner solves do without them.
    gr.built = true;
    return clsparseSuccess;
}

// The local blocks B_i of the Kaporin loss, built on the first training use
// of a graph (the factor build does not need them). Rows of L longer than
// kMaxTrainP entries are refused (the blocks grow as the square).
clsparseStatus ensure_blocks(Graph& gr, cudaStream_t s) {
    if (gr.blocks_built) return clsparseSuccess;
    if (gr.maxL > static_cast<uint32_t>(kMaxTrainP)) return clsparseInvalidValue;
    if (static_cast<uint64_t>(gr.n) * gr.maxL * gr.maxL >= (1ull << 32)) return clsparseInvalidSize;
    const uint32_t n = gr.n;
    cudaMemsetAsync(gr.Boff, 0, 4, s);
    block_sizes<<<nblk(n, 256), 256, 0, s>>>(gr.Lrp, n, gr.Boff + 1);
    scan::inclusive_u32(gr.Boff + 1, n, gr.scan_part, s);
    cudaMemcpyAsync(gr.info + 2, gr.Boff + n, 4, cudaMemcpyDeviceToDevice, s);
    uint32_t h[4];
    if (cudaGetLastError() != cudaSuccess || !read_info(gr, s, h)) return clsparseInvalidKernelExecution;
    const size_t nB = h[2];
    if (nB > gr.cap_B) {
        if (gr.B) cudaFree(gr.B);
        gr.B = nullptr;
        gr.cap_B = 0;
        if (dalloc(gr.B, nB) != cudaSuccess) {
            cudaGetLastError();
            return clsparseOutOfResources;
        }
        gr.cap_B = nB;
    }
    gr.nB = nB;
    block_fill<<<nblk(n, 128), 128, 0, s>>>(gr.rp, gr.cols, gr.ehat, gr.Lrp, gr.Lcol, gr.Boff, n, gr.B);
    if (cudaGetLastError() != cudaSuccess) return clsparseInvalidKernelExecution;
    gr.blocks_built = true;
    return clsparseSuccess;
}

// Launches the tcgen05 dense layer: a persistent grid of four CTAs per SM
// (shared memory and TMEM columns allow four on every layer), one 128-row
// tile at a time.
template <int M, int K1, int K2>
void launch_umma(const float* X1, const float* X2, const float* W, const float* b, const float* R, float* Y,
                 float* A, size_t n, int act, int device, cudaStream_t s) {
    constexpr size_t bytes = umma::smem_bytes<M, K1 + K2>();
    static_assert(4 * (M < 32 ? 32 : M) <= 512 && 4 * bytes <= 227 * 1024, "four CTAs per SM");
    static bool configured = false;
    if (!configured) {
        cudaFuncSetAttribute(linear_fwd_umma<M, K1, K2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             static_cast<int>(bytes));
        configured = true;
    }
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    const size_t tiles = (n + 127) / 128;
    const uint32_t grid = static_cast<uint32_t>(std::max<size_t>(1, std::min<size_t>(tiles, size_t(sms) * 4)));
    linear_fwd_umma<M, K1, K2><<<grid, 128, bytes, s>>>(X1, X2, W, b, R, Y, A, n, act);
}

// Whether a tcgen05 layer's commit wait ran out since the last check (clears
// the flag).
bool umma_failed() {
    int h = 0;
    cudaMemcpyFromSymbol(&h, g_umma_error, sizeof(int));
    if (h) {
        const int zero = 0;
        cudaMemcpyToSymbol(g_umma_error, &zero, sizeof(int));
    }
    return h != 0;
}

// keep_act: store the pre-activations Au the backward pass reads (training);
// the factor build skips those writes.
void forward(_clsparseB200Spai* net, int bf16, cudaStream_t s, bool keep_act = true) {
    Graph& gr = net->gr;
    const Offsets& o = net->o;
    const float* P = net->prm;
    const size_t n = gr.n;
    const uint32_t tiles = nblk(n, kRows);
    linear_fwd<H, NF, 0><<<tiles, 256, 0, s>>>(gr.F, nullptr, P + o.w_in, P + o.b_in, nullptr, gr.Hs[0],
                                                nullptr, n, 1, bf16);
    // BF16 forward: the dense layers on the tcgen05 tensor cores; FP32 weights
    // (gradient checks): CUDA-core FMAs.
    const int dev = net->device;
    for (int l = 0; l < NL; ++l) {
        if (bf16)
            launch_umma<H, H, 0>(gr.Hs[l], nullptr, P + o.U[l], nullptr, nullptr, gr.Hu[l], nullptr, n, 0, dev, s);
        else
            linear_fwd<H, H, 0><<<tiles, 256, 0, s>>>(gr.Hs[l], nullptr, P + o.U[l], nullptr, nullptr, gr.Hu[l],
                                                      nullptr, n, 0, bf16);
        message_fwd<<<warps_grid(n), 256, 0, s>>>(gr.rp, gr.cols, gr.ehat, gr.Hu[l], P + o.w[l], P + o.c[l],
                                                  gr.S[l], gr.n, bf16);
        if (bf16)
            launch_umma<H, H, H>(gr.Hs[l], gr.S[l], P + o.V[l], P + o.d[l], gr.Hs[l], gr.Hs[l + 1],
                                 keep_act ? gr.Au[l] : nullptr, n, 1, dev, s);
        else
            linear_fwd<H, H, H><<<tiles, 256, 0, s>>>(gr.Hs[l], gr.S[l], P + o.V[l], P + o.d[l], gr.Hs[l],
                                                      gr.Hs[l + 1], gr.Au[l], n, 1, bf16);
    }
    if (bf16) {
        launch_umma<HO, H, 0>(gr.Hs[NL], nullptr, P + o.P, nullptr, nullptr, gr.Hp, nullptr, n, 0, dev, s);
        launch_umma<HO, H, 0>(gr.Hs[NL], nullptr, P + o.Q, nullptr, nullptr, gr.Hq, nullptr, n, 0, dev, s);
    } else {
        linear_fwd<HO, H, 0><<<tiles, 256, 0, s>>>(gr.Hs[NL], nullptr, P + o.P, nullptr, nullptr, gr.Hp,
                                                   nullptr, n, 0, bf16);
        linear_fwd<HO, H, 0><<<tiles, 256, 0, s>>>(gr.Hs[NL], nullptr, P + o.Q, nullptr, nullptr, gr.Hq,
                                                   nullptr, n, 0, bf16);
    }
    output_fwd<<<warps_grid(n), 256, 0, s>>>(gr.Lrp, gr.Lcol, gr.Le, gr.Hs[NL], gr.Hp, gr.Hq, P, o, gr.g,
                                             gr.n, bf16);
}

// Loss and dL/dg; the loss is read back (a host sync) only when want_loss.
double loss_and_dg(_clsparseB200Spai* net, const float* probes, int K, double lambda, cudaStream_t s,
                   bool want_loss) {
    Graph& gr = net->gr;
    const uint32_t n = gr.n;
    double* parts = gr.red + 8;
    const uint32_t rg = std::min<uint32_t>(nblk(n, 256), 1024);
    kaporin_sum<<<rg, 256, 0, s>>>(gr.Lrp, gr.Boff, gr.B, gr.g, n, parts, gr.ticket, gr.red);
    kaporin_grad<<<rg, 256, 0, s>>>(gr.Lrp, gr.Boff, gr.B, gr.g, n, gr.red, gr.dg);
    cudaMemsetAsync(gr.red + 2, 0, sizeof(double), s);
    if (K > 0 && lambda > 0.0) {
        // squared norms of the probes on the device, four at a time; the
        // probe kernels read them there (nothing comes back to the host)
        double* dnorm = gr.red + 4;  // [4..7]; red[0..3] hold the loss sums
        for (int k0 = 0; k0 < K; k0 += 4) {
            const int kk = std::min(4, K - k0);
            for (int k = 0; k < kk; ++k)
                probe_norm<<<rg, 256, 0, s>>>(probes + size_t(k0 + k) * n, n, parts, gr.ticket, dnorm + k);
            for (int k = 0; k < kk; ++k) {
                const float* r = probes + size_t(k0 + k) * n;
                ahat_spmv<<<warps_grid(n), 256, 0, s>>>(gr.rp, gr.cols, gr.ehat, r, gr.pw, n);
                lspmv<<<warps_grid(n), 256, 0, s>>>(gr.Lrp, gr.Lcol, nullptr, gr.g, gr.pw, gr.pu, n);
                lspmv<<<warps_grid(n), 256, 0, s>>>(gr.LTrp, gr.LTrow, gr.LTidx, gr.g, gr.pu, gr.pv, n);
                probe_residual<<<rg, 256, 0, s>>>(gr.pv, r, dnorm + k, lambda, K, gr.pdv, n, parts, gr.ticket,
                                                  gr.red + 2);
                lspmv<<<warps_grid(n), 256, 0, s>>>(gr.Lrp, gr.Lcol, nullptr, gr.g, gr.pdv, gr.pdu, n);
                probe_grad<<<rg, 256, 0, s>>>(gr.Lrp, gr.Lcol, gr.pdv, gr.pu, gr.pdu, gr.pw, gr.dg, n, dnorm + k);
            }
        }
    }
    if (!want_loss) return 0.0;
    double h[3];
    cudaMemcpyAsync(h, gr.red, 3 * sizeof(double), cudaMemcpyDeviceToHost, s);
    cudaStreamSynchronize(s);
    return std::log(h[0] / n) - 2.0 * h[1] / n + h[2];
}

void reduce_into(_clsparseB200Spai* net, int rec, int ntiles, int off_w, int off_b, int nw, cudaStream_t s) {
    reduce_parts<<<nblk(rec, 256), 256, 0, s>>>(net->gr.part, rec, ntiles, net->grad, off_w, off_b, nw);
}

void backward(_clsparseB200Spai* net, int bf16, cudaStream_t s) {
    Graph& gr = net->gr;
    const Offsets& o = net->o;
    const float* P = net->prm;
    const size_t n = gr.n;
    const size_t nh = n * H;
    const uint32_t tiles = nblk(n, kRows);
    cudaMemsetAsync(net->grad, 0, size_t(o.total) * 4, s);
    cudaMemsetAsync(gr.dH, 0, nh * 4, s);
    output_bwd_rows<<<warps_grid(n), 256, 0, s>>>(gr.Lrp, gr.Lcol, gr.Le, gr.Hs[NL], gr.Hp, gr.Hq, P, o, gr.dg,
                                                  gr.dH, gr.dHp, gr.part, gr.n, bf16);
    reduce_into(net, kOutPart, static_cast<int>(n), o.r, -1, kOutPart, s);
    output_bwd_cols<<<warps_grid(n), 256, 0, s>>>(gr.LTrp, gr.LTrow, gr.LTidx, gr.Le, gr.Hp, gr.Hq, P, o, gr.dg,
                                                  gr.dHq, gr.n, bf16);
    linear_bwd<HO, H, 0><<<tiles, 256, 0, s>>>(gr.Hs[NL], nullptr, P + o.P, nullptr, gr.dHp, gr.dH, nullptr,
                                               gr.part, n, 0, bf16);
    reduce_into(net, HO * H + HO, tiles, o.P, -1, HO * H, s);
    linear_bwd<HO, H, 0><<<tiles, 256, 0, s>>>(gr.Hs[NL], nullptr, P + o.Q, nullptr, gr.dHq, gr.dH, nullptr,
                                               gr.part, n, 0, bf16);
    reduce_into(net, HO * H + HO, tiles, o.Q, -1, HO * H, s);
    // gr.dH holds dL/dH_NL; walk the layers back
    for (int l = NL - 1; l >= 0; --l) {
        // H_{l+1} = H_l + relu(V [H_l; S_l] + d): dH_l = dH_{l+1} + ..., dS_l = ...
        cudaMemcpyAsync(gr.dHn, gr.dH, nh * 4, cudaMemcpyDeviceToDevice, s);
        cudaMemsetAsync(gr.dS, 0, nh * 4, s);
        linear_bwd<H, H, H><<<tiles, 256, 0, s>>>(gr.Hs[l], gr.S[l], P + o.V[l], gr.Au[l], gr.dH, gr.dHn, gr.dS,
                                                  gr.part, n, 1, bf16);
        reduce_into(net, H * 2 * H + H, tiles, o.V[l], o.d[l], H * 2 * H, s);
        message_bwd<<<warps_grid(n), 256, 0, s>>>(gr.rp, gr.cols, gr.ehat, gr.Hu[l], P + o.w[l], P + o.c[l],
                                                  gr.dS, gr.dHu, gr.part, gr.n, bf16);
        reduce_into(net, 2 * H, static_cast<int>(n), o.w[l], o.c[l], H, s);
        linear_bwd<H, H, 0><<<tiles, 256, 0, s>>>(gr.Hs[l], nullptr, P + o.U[l], nullptr, gr.dHu, gr.dHn,
                                                  nullptr, gr.part, n, 0, bf16);
        reduce_into(net, H * H + H, tiles, o.U[l], -1, H * H, s);
        std::swap(gr.dH, gr.dHn);
    }
    linear_bwd<H, NF, 0><<<tiles, 256, 0, s>>>(gr.F, nullptr, P + o.w_in, gr.Hs[0], gr.dH, nullptr, nullptr,
                                               gr.part, n, 1, bf16);
    reduce_into(net, H * NF + H, tiles, o.w_in, o.b_in, H * NF, s);
}

void export_g(_clsparseB200Spai* net, cudaStream_t s) {
    Graph& gr = net->gr;
    const uint32_t g = std::min<uint32_t>(nblk(gr.n, 256), 4096);
    export_factor<<<g, 256, 0, s>>>(gr.Lrp, gr.Lcol, gr.g, gr.dinvs, gr.G32, gr.G16, gr.G64, gr.n);
    gather_transpose<<<g, 256, 0, s>>>(gr.LTidx, gr.G32, gr.G16, gr.G64, gr.GT32, gr.GT16, gr.GT64, gr.nnzL);
}

clsparseStatus check_net(clsparseB200Spai net, clsparseControl c, bool need_graph) {
    if (net == nullptr) return clsparseInvalidValue;
    clsparseStatus st = check_entry(c);
    if (st != clsparseSuccess) return st;
    if (need_graph && !net->gr.built) return clsparseStructInvalid;
    return clsparseSuccess;
}

}  // namespace

extern "C" {

clsparseStatus clsparseB200SpaiCreate(clsparseB200Spai* out, cl_ulong seed) {
    if (out == nullptr) return clsparseInvalidValue;
    auto* net = new (std::nothrow) _clsparseB200Spai();
    if (!net) return clsparseOutOfHostMemory;
    net->o = layout();
    const int P = net->o.total;
    cudaGetDevice(&net->device);
    if (dalloc(net->prm, P) != cudaSuccess || dalloc(net->grad, P) != cudaSuccess ||
        dalloc(net->m, P) != cudaSuccess || dalloc(net->v, P) != cudaSuccess) {
        cudaGetLastError();
        delete net;
        return clsparseOutOfResources;
    }
    // He-style initialisation from a fixed-seed generator
    std::vector<float> h(P, 0.f);
    std::mt19937_64 rng(seed);
    auto fill = [&](int off, int rows, int cols, float gain) {
        std::normal_distribution<float> nd(0.f, gain / std::sqrt(static_cast<float>(cols)));
        for (int i = 0; i < rows * cols; ++i) h[off + i] = nd(rng);
    };
    const Offsets& o = net->o;
    fill(o.w_in, H, NF, 1.4f);
    for (int l = 0; l < NL; ++l) {
        fill(o.U[l], H, H, 1.0f);
        fill(o.w[l], 1, H, 1.0f);
        fill(o.V[l], H, 2 * H, 0.5f);
    }
    fill(o.P, HO, H, 1.0f);
    fill(o.Q, HO, H, 1.0f);
    fill(o.r, 1, HO, 1.0f);
    fill(o.w_o, 1, HO, 0.05f);
    fill(o.w_d, 1, H, 0.05f);
    h[o.b_d] = 0.5413f;  // softplus(0.5413) = 1: starts near the Jacobi factor
    cudaMemcpy(net->prm, h.data(), size_t(P) * 4, cudaMemcpyHostToDevice);
    cudaMemset(net->m, 0, size_t(P) * 4);
    cudaMemset(net->v, 0, size_t(P) * 4);
    *out = net;
    return clsparseSuccess;
}

clsparseStatus clsparseB200SpaiRelease(clsparseB200Spai net) {
    if (net == nullptr) return clsparseInvalidValue;
    delete net;
    return clsparseSuccess;
}

clsparseStatus clsparseB200SpaiSetMatrix(clsparseB200Spai net, const clsparseCsrMatrix* A,
                                         clsparseControl control) {
    clsp::TraceRange trace_("clsparseB200SpaiSetMatrix");
    clsparseStatus st = check_net(net, control, false);
    if (st != clsparseSuccess) return st;
    if (!A || A->num_rows != A->num_cols || A->num_rows == 0) return clsparseInvalidSystemSize;
    DeviceGuard g(control->device);
    if (A->num_rows > kGraphCacheRows || !graph_cache_enabled()) {
        // Large matrices are built straight from the device arrays, every
        // time (a rebuild reuses the buffers), with no host copy of A.
        net->cur = HostCsr();
        return build_graph(net, A, control);
    }
    HostCsr h;
    st = read_host_csr(A, control, h);
    if (st != clsparseSuccess) return st;
    if (net->gr.built && net->cur.same(h)) return clsparseSuccess;
    if (graph_cache_enabled()) {
        // keep the current graph (most recent last), take a cached one if it matches
        size_t hit = net->cache.size();
        for (size_t i = 0; i < net->cache.size(); ++i)
            if (net->cache[i].key.same(h)) {
                hit = i;
                break;
            }
        CachedGraph found;
        if (hit < net->cache.size()) {
            found = std::move(net->cache[hit]);
            net->cache.erase(net->cache.begin() + static_cast<std::ptrdiff_t>(hit));
        }
        if (net->gr.built && net->gr.n <= kGraphCacheRows) {
            net->cache.push_back(CachedGraph{std::move(net->cur), net->gr});
            net->gr = Graph();  // now owned by the cache entry
            while (net->cache.size() > kGraphCache) {
                net->cache.front().gr.release();
                net->cache.erase(net->cache.begin());
            }
        }
        if (found.gr.built) {
            net->gr.release();
            net->gr = found.gr;
            net->cur = std::move(found.key);
            return clsparseSuccess;
        }
    }
    net->cur = std::move(h);
    st = build_graph(net, A, control);
    if (st != clsparseSuccess) net->cur = HostCsr();
    return st;
}

clsparseStatus clsparseB200SpaiParams(clsparseB200Spai net, cl_float* host, size_t capacity, size_t* count,
                                      cl_int toDevice) {
    if (net == nullptr || count == nullptr) return clsparseInvalidValue;
    *count = static_cast<size_t>(net->o.total);
    if (host == nullptr) return clsparseSuccess;
    if (capacity < *count) return clsparseInsufficientMemory;
    DeviceGuard g(net->device);
    const cudaError_t e = toDevice ? cudaMemcpy(net->prm, host, *count * 4, cudaMemcpyHostToDevice)
                                   : cudaMemcpy(host, net->prm, *count * 4, cudaMemcpyDeviceToHost);
    return e == cudaSuccess ? clsparseSuccess : clsparseInvalidKernelExecution;
}

clsparseStatus clsparseB200SpaiLossGrad(clsparseB200Spai net, const cldenseVector* probes, cl_int K,
                                        cl_double lambda, cl_int fp32Weights, cl_double* loss, cl_float* grad,
                                        size_t capacity, clsparseControl control) {
    clsp::TraceRange trace_("clsparseB200SpaiLossGrad");
    clsparseStatus st = check_net(net, control, true);
    if (st != clsparseSuccess) return st;
    if (K > 0 && (!probes || probes->num_values < size_t(K) * net->gr.n)) return clsparseInvalidSize;
    DeviceGuard g(control->device);
    if (!ensure_training_buffers(net->gr)) return clsparseOutOfResources;
    st = ensure_blocks(net->gr, control->stream);
    if (st != clsparseSuccess) return st;
    const int bf16 = fp32Weights ? 0 : 1;
    forward(net, bf16, control->stream);
    const double L = loss_and_dg(net, K > 0 ? dev_ptr<const float>(probes->values, probes->off_values) : nullptr,
                                 K, lambda, control->stream, loss != nullptr);
    backward(net, bf16, control->stream);
    if (loss) *loss = L;
    if (grad) {
        if (capacity < size_t(net->o.total)) return clsparseInsufficientMemory;
        cudaMemcpyAsync(grad, net->grad, size_t(net->o.total) * 4, cudaMemcpyDeviceToHost, control->stream);
    }
    if (cudaStreamSynchronize(control->stream) != cudaSuccess || umma_failed())
        return clsparseInvalidKernelExecution;
    return clsparseSuccess;
}

clsparseStatus clsparseB200SpaiTrainStep(clsparseB200Spai net, const cldenseVector* probes, cl_int K,
                                         cl_double lambda, cl_double lr, cl_double* loss,
                                         clsparseControl control) {
    clsp::TraceRange trace_("clsparseB200SpaiTrainStep");
    clsparseStatus st = clsparseB200SpaiLossGrad(net, probes, K, lambda, 0, loss, nullptr, 0, control);
    if (st != clsparseSuccess) return st;
    DeviceGuard g(control->device);
    net->step += 1;
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.f - std::pow(b1, float(net->step)), c2 = 1.f - std::pow(b2, float(net->step));
    adam_step<<<nblk(net->o.total, 256), 256, 0, control->stream>>>(net->prm, net->grad, net->m, net->v,
                                                                    net->o.total, float(lr), b1, b2, 1e-8f, c1,
                                                                    c2);
    return finish_call(control);
}

clsparseStatus clsparseB200SpaiGradient(clsparseB200Spai net, cl_float** deviceGrad, size_t* count) {
    if (net == nullptr || deviceGrad == nullptr) return clsparseInvalidValue;
    *deviceGrad = net->grad;
    if (count) *count = static_cast<size_t>(net->o.total);
    return clsparseSuccess;
}

clsparseStatus clsparseB200SpaiAdamStep(clsparseB200Spai net, cl_double lr, cl_double gradScale,
                                        clsparseControl control) {
    clsp::TraceRange trace_("clsparseB200SpaiAdamStep");
    if (net == nullptr) return clsparseInvalidValue;
    if (control == nullptr) return clsparseInvalidControlObject;
    if (!(lr >= 0.0) || !std::isfinite(gradScale)) return clsparseInvalidValue;
    DeviceGuard g(control->device);
    const uint32_t P = static_cast<uint32_t>(net->o.total);
    if (gradScale != 1.0) scale_kernel<<<nblk(P, 256), 256, 0, control->stream>>>(net->grad, P, float(gradScale));
    net->step += 1;
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.f - std::pow(b1, float(net->step)), c2 = 1.f - std::pow(b2, float(net->step));
    adam_step<<<nblk(P, 256), 256, 0, control->stream>>>(net->prm, net->grad, net->m, net->v, P, float(lr), b1, b2,
                                                         1e-8f, c1, c2);
    return finish_call(control);
}

clsparseStatus clsparseB200SpaiBuild(clsparseB200Spai net, clsparseControl control) {
    clsp::TraceRange trace_("clsparseB200SpaiBuild");
    clsparseStatus st = check_net(net, control, true);
    if (st != clsparseSuccess) return st;
    DeviceGuard g(control->device);
    forward(net, 1, control->stream, false);
    export_g(net, control->stream);
    if (cudaStreamSynchronize(control->stream) != cudaSuccess || umma_failed())
        return clsparseInvalidKernelExecution;
    return finish_call(control);
}

// Copies the exported factor (FP64, L = tril(A) order) and its pattern to the host.
clsparseStatus clsparseB200SpaiGetFactor(clsparseB200Spai net, clsparseIdx_t* rowPtr, clsparseIdx_t* cols,
                                         cl_double* vals, size_t capacity, size_t* nnz) {
    if (net == nullptr || nnz == nullptr || !net->gr.built) return clsparseInvalidValue;
    *nnz = net->gr.nnzL;
    if (!rowPtr && !cols && !vals) return clsparseSuccess;
    if (capacity < net->gr.nnzL) return clsparseInsufficientMemory;
    DeviceGuard g(net->device);
    if (rowPtr) cudaMemcpy(rowPtr, net->gr.Lrp, (net->gr.n + 1) * 4, cudaMemcpyDeviceToHost);
    if (cols) cudaMemcpy(cols, net->gr.Lcol, size_t(net->gr.nnzL) * 4, cudaMemcpyDeviceToHost);
    if (vals) cudaMemcpy(vals, net->gr.G64, size_t(net->gr.nnzL) * 8, cudaMemcpyDeviceToHost);
    return cudaGetLastError() == cudaSuccess ? clsparseSuccess : clsparseInvalidKernelExecution;
}

// Checkpoint: "CLSPSPAI", version, parameter count, step, FP32 weights, Adam
// moments, FNV-1a 64 checksum of everything before it.
clsparseStatus clsparseB200SpaiSave(clsparseB200Spai net, const char* path) {
    if (net == nullptr || path == nullptr) return clsparseInvalidValue;
    DeviceGuard g(net->device);
    const size_t P = size_t(net->o.total);
    std::vector<float> buf(3 * P);
    cudaMemcpy(buf.data(), net->prm, P * 4, cudaMemcpyDeviceToHost);
    cudaMemcpy(buf.data() + P, net->m, P * 4, cudaMemcpyDeviceToHost);
    cudaMemcpy(buf.data() + 2 * P, net->v, P * 4, cudaMemcpyDeviceToHost);
    const char magic[8] = {'C', 'L', 'S', 'P', 'S', 'P', 'A', 'I'};
    const uint32_t hdr[3] = {1u, static_cast<uint32_t>(P), static_cast<uint32_t>(net->step)};
    uint64_t h = fnv1a(magic, 8);
    h = fnv1a(hdr, sizeof(hdr), h);
    h = fnv1a(buf.data(), buf.size() * 4, h);
    FILE* f = std::fopen(path, "wb");
    if (!f) return clsparseInvalidFile;
    bool ok = std::fwrite(magic, 1, 8, f) == 8 && std::fwrite(hdr, 4, 3, f) == 3 &&
              std::fwrite(buf.data(), 4, buf.size(), f) == buf.size() && std::fwrite(&h, 8, 1, f) == 1;
    ok = (std::fclose(f) == 0) && ok;
    return ok ? clsparseSuccess : clsparseInvalidFile;
}

clsparseStatus clsparseB200SpaiLoad(clsparseB200Spai net, const char* path) {
    if (net == nullptr || path == nullptr) return clsparseInvalidValue;
    FILE* f = std::fopen(path, "rb");
    if (!f) return clsparseInvalidFile;
    char magic[8];
    uint32_t hdr[3];
    const size_t P = size_t(net->o.total);
    std::vector<float> buf(3 * P);
    uint64_t h_file = 0;
    bool ok = std::fread(magic, 1, 8, f) == 8 && std::memcmp(magic, "CLSPSPAI", 8) == 0 &&
              std::fread(hdr, 4, 3, f) == 3 && hdr[0] == 1u && hdr[1] == P &&
              std::fread(buf.data(), 4, buf.size(), f) == buf.size() && std::fread(&h_file, 8, 1, f) == 1;
    std::fclose(f);
    if (!ok) return clsparseInvalidFileFormat;
    uint64_t h = fnv1a(magic, 8);
    h = fnv1a(hdr, sizeof(hdr), h);
    h = fnv1a(buf.data(), buf.size() * 4, h);
    if (h != h_file) return clsparseInvalidFileFormat;
    DeviceGuard g(net->device);
    cudaMemcpy(net->prm, buf.data(), P * 4, cudaMemcpyHostToDevice);
    cudaMemcpy(net->m, buf.data() + P, P * 4, cudaMemcpyHostToDevice);
    cudaMemcpy(net->v, buf.data() + 2 * P, P * 4, cudaMemcpyHostToDevice);
    net->step = static_cast<int>(hdr[2]);
    return cudaGetLastError() == cudaSuccess ? clsparseSuccess : clsparseInvalidKernelExecution;
}

}  // extern "C"

namespace clsp {

// The CSR-Adaptive metas of the patterns of G (tril(A)) and G^T, made on
// first use after a graph build.
clsparseStatus spai_ensure_metas(clsparseB200Spai net, clsparseControl c) {
    if (net == nullptr || !net->gr.built) return clsparseStructInvalid;
    Graph& gr = net->gr;
    if (gr.metaL != nullptr && gr.metaLT != nullptr) return clsparseSuccess;
    delete gr.metaL;
    delete gr.metaLT;
    gr.metaL = gr.metaLT = nullptr;
    clsparseCsrMatrix pat;
    std::memset(&pat, 0, sizeof(pat));
    pat.num_rows = gr.n;
    pat.num_cols = gr.n;
    pat.num_nonzeros = gr.nnzL;
    pat.row_pointer = gr.Lrp;
    pat.col_indices = gr.Lcol;
    if (clsparseCsrMetaCreate(&pat, c) != clsparseSuccess) return clsparseOutOfResources;
    gr.metaL = static_cast<matrix_meta*>(pat.meta);
    pat.meta = nullptr;
    pat.row_pointer = gr.LTrp;
    pat.col_indices = gr.LTrow;
    if (clsparseCsrMetaCreate(&pat, c) != clsparseSuccess) return clsparseOutOfResources;
    gr.metaLT = static_cast<matrix_meta*>(pat.meta);
    return clsparseSuccess;
}

// Views of the exported factor for the solvers (mixed.cu); the metas are null
// until spai_ensure_metas.
bool spai_factor_views(clsparseB200Spai net, CsrView<__nv_bfloat16>& G16, CsrView<__nv_bfloat16>& GT16,
                       CsrView<float>& G32, CsrView<float>& GT32, CsrView<double>& G64, CsrView<double>& GT64) {
    if (net == nullptr || !net->gr.built) return false;
    const Graph& gr = net->gr;
    G16 = CsrView<__nv_bfloat16>{gr.G16, gr.Lcol, gr.Lrp, gr.n, gr.n, gr.nnzL, gr.metaL};
    GT16 = CsrView<__nv_bfloat16>{gr.GT16, gr.LTrow, gr.LTrp, gr.n, gr.n, gr.nnzL, gr.metaLT};
    G32 = CsrView<float>{gr.G32, gr.Lcol, gr.Lrp, gr.n, gr.n, gr.nnzL, gr.metaL};
    GT32 = CsrView<float>{gr.GT32, gr.LTrow, gr.LTrp, gr.n, gr.n, gr.nnzL, gr.metaLT};
    G64 = CsrView<double>{gr.G64, gr.Lcol, gr.Lrp, gr.n, gr.n, gr.nnzL, gr.metaL};
    GT64 = CsrView<double>{gr.GT64, gr.LTrow, gr.LTrp, gr.n, gr.n, gr.nnzL, gr.metaLT};
    return true;
}

}  // namespace clsp
