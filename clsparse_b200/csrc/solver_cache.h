// Per-control cache of the last solve's work vectors and CUDA graph, so that
// repeated solves on the same operands re-launch one instantiated graph
// instead of allocating and capturing again.
#pragma once

#include <cstring>

#include "internal.h"

namespace clsp {

struct SolverKey {
    int kind = 0;       // 1 CG, 2 BiCGStab
    int dtype = 0;      // sizeof(T)
    int precond = 0;
    int ext = 0;
    int loop_mode = 0;
    int warm = 0;       // continues the previous solve's search direction
    const void* ptrs[8] = {};  // vals, cols, rowptr, x, b, meta, preconditioner factors
    uint32_t n = 0, nnz = 0;
    size_t meta_words = 0;
    cudaStream_t stream = nullptr;
    bool operator==(const SolverKey& o) const { return std::memcmp(this, &o, sizeof(*this)) == 0; }
};

struct SolverCache {
    SolverKey key;
    bool valid = false;
    DeviceBuffer vecs;
    DeviceBuffer parts;
    DeviceBuffer state;
    DeviceBuffer fused;      // persistent solver: barrier area + per-CTA word ranges
    uint32_t fused_grid = 0; // grid the word ranges in `fused` were made for (0: none)
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    void drop_graph() {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        exec = nullptr;
        graph = nullptr;
    }
    ~SolverCache() { drop_graph(); }
};

}  // namespace clsp
