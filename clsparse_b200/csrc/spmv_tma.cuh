// TMA-staged, warp-specialised CSR-Adaptive SpMV for sm_100a (included by
// spmv.cu after the shared helpers).
//
// One persistent CTA per resident slot walks the row-block words assigned to
// it (word w goes to CTA w mod gridDim). A producer warp reads the words ahead
// of time and, for every STREAM block, issues three 1-D bulk copies
// (cp.async.bulk, completing on a full-barrier) that bring the block's column
// indices, values and row pointers into one of kStages shared-memory stages.
// Eight consumer warps wait on the stage's full-barrier, gather x for all of
// the block's nonzeros in parallel (4 independent gathers per thread), write
// the products linearly into a product buffer, reduce every row out of it
// with 1..32 lanes per row (the reference's per-block width, capped at a
// warp) and release the stage on its empty-barrier. Streaming the matrix
// through the bulk-copy engine keeps the load/store pipe free for the x
// gathers, and kStages blocks per CTA stay in flight without holding
// registers.
//
// VECTOR rows and LONG-row chunks (>= 1024 nonzeros each) are read by the
// consumers straight from global memory; LONG chunks finish with the same
// arrival-ticket merge as the plain kernel. Blocks whose copies would reach
// outside the arrays (ragged ends) or that hold more rows than a stage keeps
// are processed from global memory as well. Every barrier wait is bounded
// (pipe::kSpinLimit polls); a timeout records an error in *err and ends the
// kernel instead of waiting forever.

namespace tma {

constexpr int kConsumerWarps = 8;
constexpr int kConsumers = kConsumerWarps * 32;
constexpr int kThreads = kConsumers + 32;  // + one producer warp
constexpr int kStages = 3;
constexpr uint32_t kStageCols = kBlkSize + 16;  // u32 slots (block + alignment slack)
constexpr uint32_t kStageVals = kBlkSize + 16;  // value slots
constexpr uint32_t kStageRp = kBlkSize + 16;    // u32 slots

enum : uint32_t { kStream = 0, kStreamGlobal = 1, kVector = 2, kLong = 3, kSkip = 4 };

struct TaskDesc {
    uint32_t row, stop, nb, ne;
    uint32_t low, kind, col_off, val_off;
    uint32_t rp_off, pad0, pad1, pad2;
};

template <typename V, typename T>
struct Layout {
    static constexpr size_t cols_bytes = kStageCols * 4;
    static constexpr size_t vals_bytes = ((kStageVals * sizeof(V) + 127) / 128) * 128;
    static constexpr size_t rp_bytes = kStageRp * 4;
    static constexpr size_t stage_bytes = cols_bytes + vals_bytes + rp_bytes;
    static constexpr size_t head_bytes = 1024;  // barriers, descriptors, reduction scratch
    static constexpr size_t pbuf_bytes = ((kBlkSize * sizeof(T) + 127) / 128) * 128;
    static constexpr size_t total = head_bytes + pbuf_bytes + kStages * stage_bytes;
};

// Block-wide sum over the consumer warps only (named barrier 1).
template <typename T, bool EXT>
__device__ __forceinline__ dev::Acc<T, EXT> consumer_reduce(dev::Acc<T, EXT> a, T* ss, T* sc) {
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    dev::group_reduce<32>(a);
    pipe::named_sync(1, kConsumers);
    if (lane == 0) {
        ss[warp] = a.s;
        sc[warp] = a.c;
    }
    pipe::named_sync(1, kConsumers);
    dev::Acc<T, EXT> b;
    if (lane < kConsumerWarps) {
        b.s = ss[lane];
        b.c = sc[lane];
    }
    dev::group_reduce<32>(b);
    return b;
}

template <typename V, typename T, bool EXT, int K>
__global__ void __launch_bounds__(kThreads, EXT ? 1 : 2)
    csr_adaptive_tma_kernel(const V* __restrict__ vals, const uint32_t* __restrict__ cols,
                            const uint32_t* __restrict__ rp, const T* __restrict__ x,
                            T* __restrict__ y, const T* __restrict__ alpha_p,
                            const T* __restrict__ beta_p, const uint64_t* __restrict__ words,
                            const uint32_t* __restrict__ word_nnz, uint32_t nblocks,
                            uint32_t nrows_total, uint32_t hi, int aligned,
                            double* __restrict__ lr_partial, uint32_t* __restrict__ lr_ticket,
                            int* __restrict__ err, EpiDev<T> epi) {
    using L = Layout<V, T>;
    extern __shared__ __align__(128) unsigned char smem[];
    uint64_t* full = reinterpret_cast<uint64_t*>(smem);
    uint64_t* empty = full + kStages;
    TaskDesc* desc = reinterpret_cast<TaskDesc*>(smem + 64);
    T* red_s = reinterpret_cast<T*>(smem + 64 + kStages * sizeof(TaskDesc));
    T* red_c = red_s + 32;
    // [0] written only by consumers (a consumer's full-barrier wait timed
    // out), [1] written only by the producer (it stopped early)
    volatile int* flags = reinterpret_cast<volatile int*>(red_c + 32);
    T* pbuf = reinterpret_cast<T*>(smem + L::head_bytes);
    unsigned char* stages = smem + L::head_bytes + L::pbuf_bytes;
    auto scols = [&](uint32_t s) { return reinterpret_cast<uint32_t*>(stages + s * L::stage_bytes); };
    auto svals = [&](uint32_t s) {
        return reinterpret_cast<V*>(stages + s * L::stage_bytes + L::cols_bytes);
    };
    auto srp = [&](uint32_t s) {
        return reinterpret_cast<uint32_t*>(stages + s * L::stage_bytes + L::cols_bytes + L::vals_bytes);
    };

    if (epi.done != nullptr && *epi.done) return;

    const int tid = threadIdx.x;
    const int warp = tid >> 5;
    const int lane = tid & 31;
    if (tid == 0) {
        for (int s = 0; s < kStages; ++s) {
            pipe::mbar_init(&full[s], 1);
            pipe::mbar_init(&empty[s], kConsumerWarps);
        }
        flags[0] = 0;
        flags[1] = 0;
        pipe::fence_barrier_init();
    }
    __syncthreads();

    const T alpha = *alpha_p;
    RowSink<T, K> sink;
    sink.init(y, epi, *beta_p);
    const uint32_t G = gridDim.x;

    if (warp == kConsumerWarps) {
        // ------------------------------------------------------ producer
        constexpr uint32_t VA = 16 / sizeof(V);  // values per 16 bytes
        uint32_t k = 0;
        bool abort = false;
        // per stage: bit s of `issued` = a bulk copy was issued into it, bit s
        // of `parity` = parity of the full-barrier phase of the last one
        uint32_t issued = 0, parity = 0;
        for (uint64_t t0 = blockIdx.x; t0 < nblocks && !abort; t0 += 32ull * G) {
            const uint64_t tl = t0 + static_cast<uint64_t>(lane) * G;
            uint64_t a0 = 0, a1 = 0;
            uint32_t b0 = 0, b1 = 0;
            if (tl < nblocks) {
                a0 = words[tl];
                a1 = words[tl + 1];
                b0 = word_nnz[tl];
                b1 = word_nnz[tl + 1];
            }
            const uint64_t left = (nblocks - t0 + G - 1) / G;
            const uint32_t navail = left < 32 ? static_cast<uint32_t>(left) : 32u;
            for (uint32_t i = 0; i < navail; ++i, ++k) {
                const uint64_t w0 = __shfl_sync(0xffffffffu, a0, i);
                const uint64_t w1 = __shfl_sync(0xffffffffu, a1, i);
                const uint32_t nb = __shfl_sync(0xffffffffu, b0, i);
                const uint32_t ne = __shfl_sync(0xffffffffu, b1, i);
                const uint32_t s = k % kStages;
                int ok = 1;
                if (lane == 0) {
                    if (k >= static_cast<uint32_t>(kStages))
                        ok = pipe::mbar_wait(&empty[s], ((k / kStages) - 1) & 1, err) ? 1 : 0;
                    if (ok) {
                        TaskDesc d;
                        d.row = static_cast<uint32_t>(w0 >> 32);
                        d.stop = static_cast<uint32_t>(w1 >> 32);
                        d.nb = nb;
                        d.ne = ne;
                        d.low = static_cast<uint32_t>(w0 & ((1u << kWgBits) - 1u));
                        d.col_off = d.val_off = d.rp_off = 0;
                        const uint32_t nr = d.stop - d.row;
                        uint32_t bytes = 0;
                        if (nr > kRowsForVector) {
                            d.kind = kStreamGlobal;
                            const uint32_t c0 = nb & ~3u, c1 = (ne + 3u) & ~3u;
                            const uint32_t v0 = nb & ~(VA - 1u), v1 = (ne + VA - 1u) & ~(VA - 1u);
                            const uint32_t r0 = d.row & ~3u, r1 = (d.stop + 4u) & ~3u;
                            if (aligned && ne > nb && ne - nb <= kBlkSize && c1 <= hi && v1 <= hi &&
                                r1 <= nrows_total + 1 && r1 - r0 <= kStageRp) {
                                d.kind = kStream;
                                d.col_off = nb - c0;
                                d.val_off = nb - v0;
                                d.rp_off = d.row - r0;
                                bytes = (c1 - c0) * 4u + (v1 - v0) * static_cast<uint32_t>(sizeof(V)) +
                                        (r1 - r0) * 4u;
                                desc[s] = d;
                                pipe::mbar_arrive_expect_tx(&full[s], bytes);
                                pipe::bulk_g2s(scols(s), cols + c0, (c1 - c0) * 4u, &full[s]);
                                pipe::bulk_g2s(svals(s), vals + v0,
                                               (v1 - v0) * static_cast<uint32_t>(sizeof(V)), &full[s]);
                                pipe::bulk_g2s(srp(s), rp + r0, (r1 - r0) * 4u, &full[s]);
                                issued |= 1u << s;
                                parity = (parity & ~(1u << s)) | (((k / kStages) & 1u) << s);
                            }
                        } else if (nr == 1 && d.low == 0) {
                            d.kind = kVector;
                        } else {
                            d.kind = kLong;
                        }
                        if (bytes == 0) {
                            desc[s] = d;
                            pipe::mbar_arrive(&full[s]);
                        }
                    }
                }
                ok = __shfl_sync(0xffffffffu, ok, 0);
                if (!ok) {
                    abort = true;
                    break;
                }
            }
        }
        if (abort && lane == 0) {
            flags[1] = 1;
            // let the copies already issued land before the CTA can exit
            for (int s = 0; s < kStages; ++s)
                if (issued & (1u << s)) pipe::mbar_wait(&full[s], (parity >> s) & 1u, nullptr);
        }
    } else {
        // ----------------------------------------------------- consumers
        uint32_t k = 0;
        for (uint64_t t = blockIdx.x; t < nblocks; t += G, ++k) {
            const uint32_t s = k % kStages;
            const bool got = pipe::mbar_wait(&full[s], (k / kStages) & 1, err);
            if (!got) flags[0] = 1;
            pipe::named_sync(1, kConsumers);
            if (flags[0]) break;
            const TaskDesc d = desc[s];
            const uint32_t nr = d.stop - d.row;
            if (d.kind == kStream || d.kind == kStreamGlobal) {
                const bool staged_in = d.kind == kStream;
                const uint32_t cnt = d.ne - d.nb;
                const bool use_pbuf = cnt <= kBlkSize;
                if (use_pbuf) {
                    const uint32_t* sc = scols(s) + d.col_off;
                    const V* sv = svals(s) + d.val_off;
                    uint32_t cc[4];
                    T vv[4], xv[4];
#pragma unroll
                    for (int u = 0; u < 4; ++u) {
                        const uint32_t i = tid + u * kConsumers;
                        if (i < cnt) {
                            if (staged_in) {
                                cc[u] = sc[i];
                                vv[u] = dev::to_t<T>(sv[i]);
                            } else {
                                cc[u] = dev::ld_stream(cols + d.nb + i);
                                vv[u] = dev::ld_val<T>(vals + d.nb + i);
                            }
                        }
                    }
#pragma unroll
                    for (int u = 0; u < 4; ++u)
                        if (tid + u * kConsumers < cnt) xv[u] = dev::ld_gather(x + cc[u]);
#pragma unroll
                    for (int u = 0; u < 4; ++u) {
                        const uint32_t i = tid + u * kConsumers;
                        if (i < cnt) pbuf[i] = dev::mul_rn(alpha * vv[u], xv[u]);
                    }
                }
                pipe::named_sync(1, kConsumers);
                const uint32_t* rps = srp(s) + d.rp_off;
                const uint32_t gw = d.low == 0 ? 1u : (d.low > 32u ? 32u : d.low);
                auto reduce_rows = [&](auto gc) {
                    constexpr int GW = decltype(gc)::value;
                    const uint32_t groups = kConsumers / GW;
                    const uint32_t grp = tid / GW;
                    const uint32_t ln = tid & (GW - 1);
                    for (uint32_t rb = 0; rb < nr; rb += groups) {
                        const uint32_t r = rb + grp;
                        dev::Acc<T, EXT> a;
                        if (r < nr) {
                            const uint32_t f = (staged_in ? rps[r] : dev::ld_ro(rp + d.row + r)) - d.nb;
                            const uint32_t l = (staged_in ? rps[r + 1] : dev::ld_ro(rp + d.row + r + 1)) - d.nb;
                            if (use_pbuf) {
                                for (uint32_t j = f + ln; j < l; j += GW) a.add(pbuf[j]);
                            } else {
                                for (uint32_t j = d.nb + f + ln; j < d.nb + l; j += GW)
                                    a.add(dev::mul_rn(alpha * dev::ld_val<T>(vals + j), dev::ld_ro(x + cols[j])));
                            }
                        }
                        dev::group_reduce<GW>(a);
                        if (r < nr && ln == 0) sink.template put<EXT>(d.row + r, a);
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
            } else if (d.kind == kVector) {
                dev::Acc<T, EXT> a =
                    range_sum<V, T, EXT, kConsumers>(vals, cols, DenseX<T>{x}, alpha, d.nb, d.ne, 0u, hi, aligned != 0);
                a = consumer_reduce(a, red_s, red_c);
                if (tid == 0) sink.template put<EXT>(d.row, a);
            } else if (d.kind == kLong) {
                const uint32_t re = dev::ld_ro(rp + d.row + 1);
                const uint32_t len = re - d.nb;
                const uint32_t nchunks = (len + kLongChunk - 1) / kLongChunk;
                if (nchunks >= 2 && d.low < nchunks) {
                    const uint32_t gid = static_cast<uint32_t>(t);
                    const uint32_t first = gid - d.low;
                    const uint32_t cb = d.nb + d.low * kLongChunk;
                    const uint32_t ce = min(re, cb + kLongChunk);
                    dev::Acc<T, EXT> a =
                        range_sum<V, T, EXT, kConsumers>(vals, cols, DenseX<T>{x}, alpha, cb, ce, 0u, hi, aligned != 0);
                    a = consumer_reduce(a, red_s, red_c);
                    if (tid == 0) {
                        lr_partial[gid] = static_cast<double>(a.value());
                        __threadfence();
                        const uint32_t tk = atomicAdd(lr_ticket + first, 1u);
                        if (tk == nchunks - 1) {
                            __threadfence();
                            dev::Acc<T, EXT> tot;
                            for (uint32_t w = 0; w < nchunks; ++w)
                                tot.add(static_cast<T>(__ldcg(lr_partial + first + w)));
                            lr_ticket[first] = 0u;
                            sink.template put<EXT>(d.row, tot);
                        }
                    }
                }
            }
            pipe::named_sync(1, kConsumers);  // pbuf and the stage are free again
            __syncwarp();
            if (lane == 0) pipe::mbar_arrive(&empty[s]);
        }
    }
    run_epilogue<T, K>(sink, epi);
}

}  // namespace tma
