// refine.cuh -- state of the FP32 triangular solve refined with FP64
// residuals (refine.cu).
#pragma once

#include "common.cuh"

namespace smax {

struct RefineState {
    uint64_t vals_version = ~0ull;  // value upload the float copies were made from
    DevBuf val32, D32;              // float copies of the (diagonal-last) values and the diagonal
    DevBuf b32, x32, r32;           // float work vectors
    DevBuf stats;                   // max|d|, max|x| as ordered bit patterns (2 x u64)
    AuxStream aux;                  // capture stream when the caller's cannot be captured
    cudaGraphExec_t graph = nullptr;
    const void *gkey[2] = {nullptr, nullptr};
    int g_steps = -1, g_merge = -1;
    uint64_t g_serial = ~0ull, g_aver = ~0ull;  // level plan and A upload the graph was captured for
    const void *g_pack = nullptr;                // level pack the graph reads
    int steps_done = 0;
    double last_rel = 0.0;          // max|d| / max|x| of the last correction
    void release_graph() {
        if (graph) cudaGraphExecDestroy(graph);
        graph = nullptr;
    }
    RefineState() = default;
    RefineState(const RefineState &) = delete;
    RefineState &operator=(const RefineState &) = delete;
    ~RefineState() { release_graph(); }
};

}  // namespace smax
