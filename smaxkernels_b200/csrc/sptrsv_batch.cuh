// sptrsv_batch.cuh -- persistent triangular solves (sptrsv_batch.cu).
#pragma once

#include <cstring>
#include <vector>

#include "kernel_obj.cuh"
#include "sptrsv.cuh"

namespace smax {

// A batch of independent lower-triangular matrices packed as one
// block-diagonal CRS (global row numbers), with per-matrix level sets.
struct TriBatch {
    int vbytes = 8;
    int n_mats = 0;
    int64_t n_rows = 0, nnz = 0;
    int total_levels = 0;
    std::vector<int> mat_levels;          // levels per matrix
    std::vector<int64_t> row_off;         // first packed row of each matrix
    std::vector<int> h_lvl_rows, h_mat_lvl_off;
    DevCRS A;
    DevBuf D, order, mat_lvl_off, lvl_rows, queue_order, queue;
    LevelPack pack;          // level-ordered pack, one single-CTA run per matrix
    bool pack_ok = false;    // false: the plain batch kernel (the pack would be too sparse)
    cudaGraphExec_t graph = nullptr;
    const void *graph_b = nullptr, *graph_x = nullptr;
    AuxStream aux;  // capture stream when the caller's stream cannot be captured

    void build(int vbytes, const std::vector<RegCRS> &mats, cudaStream_t st);
    template <typename VT> void solve_persistent(const VT *B, VT *X, cudaStream_t st);
    template <typename VT> void solve_graph(const VT *B, VT *X, cudaStream_t st);
    template <typename VT> void solve_per_level(const VT *B, VT *X, cudaStream_t st);
    ~TriBatch();
};

// One matrix, all levels in one cooperative launch with a bounded grid
// barrier; a barrier that does not complete within spin_limit polls records
// SMAX_ERR_TIMEOUT in st and ends the kernel.  force_timeout makes the barrier
// wait for one arrival more than the grid has (test knob).
template <typename VT>
void tri_solve_persistent(const TriPlan &p, const DevCRS &a, const VT *D, const VT *B, VT *X, DevStatus *st,
                          DevBuf &scratch, bool force_timeout, long long spin_limit, cudaStream_t s);

}  // namespace smax
