// Interface of the persistent (single cooperative launch) solvers in
// fused_cg.cu, used by the solver entry points in solvers.cu.
#pragma once

#include <vector>

#include "internal.h"
#include "solver_state.cuh"

namespace clsp {

constexpr int kFusedThreads = 128;

// A CSR matrix with its row-block words and the static word range of every
// CTA (cta_words[c] .. cta_words[c+1]).
template <typename V>
struct WordMat {
    const V* vals;
    const uint32_t* cols;
    const uint32_t* rp;
    const uint64_t* words;
    const uint32_t* word_nnz;
    const uint32_t* cta_words;
    double* lr_partial;
    uint32_t* lr_ticket;
    uint32_t lo, hi;
    int vec;
};

// Grid exchange area: arrival counter, release flag and error flag (zero at
// launch) and two buffers of four partial sums per CTA; the limit of one
// barrier wait, and a test switch under which the last CTA to arrive does not
// release the first barrier, so that every wait runs out (the failure path's
// test: the kernel must end with the barrier-timeout status, every CTA gone).
struct FusedSync {
    unsigned long long* arrive;
    unsigned long long* release;
    int* err;
    double* partials;
    unsigned long long wait_ns;
    int never_release;
};

constexpr unsigned long long kFusedWaitNs = 4000000000ull;  // one barrier wait gives up after 4 s

constexpr size_t kFusedSyncHead = 256;  // bytes zeroed before each launch
inline size_t fused_sync_bytes(uint32_t G) { return kFusedSyncHead + 2 * 4 * static_cast<size_t>(G) * sizeof(double); }

inline FusedSync fused_sync_at(void* base) {
    char* b = static_cast<char*>(base);
    FusedSync s;
    s.arrive = reinterpret_cast<unsigned long long*>(b);
    s.release = reinterpret_cast<unsigned long long*>(b + 128);
    s.err = reinterpret_cast<int*>(b + 192);
    s.partials = reinterpret_cast<double*>(b + kFusedSyncHead);
    s.wait_ns = kFusedWaitNs;
    s.never_release = 0;
    return s;
}

template <typename V, typename T, typename VG>
struct FusedCgArgs {
    WordMat<V> A;
    WordMat<VG> G, Gt;  // factor and its transpose (factor PCG only)
    T* x;
    const T* b;
    T* q;
    T* r;
    T* p;
    T* t;
    T* z;
    T* invD;  // Jacobi (CG only); nullptr: no preconditioner
    SolverState<T>* st;
    FusedSync sync;
    uint32_t n;
};

// cta_words for a grid of G CTAs, balanced by nonzeros.
void word_partition(const matrix_meta* m, uint32_t G, std::vector<uint32_t>& out);

template <typename V>
WordMat<V> word_mat(const CsrView<V>& A, const uint32_t* cta_words);

// Grid size of the persistent kernel (all CTAs resident): SMs x CTAs per SM.
template <typename V, typename T, typename VG>
uint32_t fused_grid(int sm_count, bool ext, int pk);

// pk = 0: CG (Jacobi or none), pk = 1: PCG with M^-1 = G^T G.
template <typename V, typename T, typename VG>
cudaError_t launch_pcg_fused(const FusedCgArgs<V, T, VG>& a, uint32_t grid, bool ext, int pk, cudaStream_t s);

}  // namespace clsp
