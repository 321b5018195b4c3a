// spmv_formats.cuh -- device-resident SELL-C-sigma and BCRS matrices, their
// SpMV launchers and the GPU conversions from CRS; SpMM launchers.
#pragma once

#include "common.cuh"

namespace smax {

// Device copy of a CRS matrix (int32 indices); col/val may be padded.
struct DevCRS {
    int64_t n_rows = 0, n_cols = 0, nnz = 0;
    DevBuf row_ptr, col, val;
    const int *rp() const { return row_ptr.as<int>(); }
    const int *ci() const { return col.as<int>(); }
};

// SELL-C-sigma (src/common.hpp:62-88)
struct DevSCS {
    int64_t C = 0, sigma = 0, n_rows = 0, n_rows_padded = 0, n_cols = 0, n_chunks = 0, n_elements = 0, nnz = 0;
    DevBuf chunk_ptr, chunk_len, col, val;
    // warp tasks of at most kScsTaskCols chunk columns (scs_plan): a chunk
    // longer than that is split, its tasks write partial sums to slots that a
    // fix-up pass adds in task order
    int64_t n_tasks = 0, n_multi = 0, n_slots = 0;
    DevBuf task_chunk, task_j0, task_slot, multi_chunk, multi_first, multi_count, partial;
    // per padded row: its entries up to the last one that is not padding
    // (column 0, value 0); the task kernel skips the rest when x[0] is finite
    DevBuf row_len;
    int plan_vbytes = 0;
};

constexpr int kScsTaskCols = 64;
// Builds the task plan of a SELL-C-sigma matrix (after upload or conversion).
void scs_plan(DevSCS &m, int vbytes, cudaStream_t st);

// BCRS (src/common.hpp:90-111): n_rows/n_cols count blocks
struct DevBCRS {
    int64_t n_rows = 0, n_cols = 0, n_blocks = 0, bh = 0, bw = 0, hpad = 0, wpad = 0;
    bool col_major = false;
    DevBuf row_ptr, col, val;
    // block rows longest first (bcrs_plan): the warp-per-block-row kernel
    // starts the long rows first, so none is left running alone at the end
    DevBuf order;
};
void bcrs_plan(DevBCRS &m, cudaStream_t st);

void validate_scs(const DevSCS &m, DevStatus *st, cudaStream_t s);
void validate_bcrs(const DevBCRS &m, DevStatus *st, cudaStream_t s);

template <typename VT> void scs_spmv(const DevSCS &m, const VT *x, VT *y, cudaStream_t st);
bool scs_vector_path(int64_t C, int vbytes);
// perm (device, n_rows ints) receives perm[old] = new
void crs_to_scs(const DevCRS &a, int vbytes, int64_t C, int64_t sigma, DevSCS &out, DevBuf &perm, cudaStream_t st);

template <typename VT> void bcrs_spmv(const DevBCRS &m, const VT *x, VT *y, cudaStream_t st);
// max_blocks >= 0: when the matrix needs more blocks, only out.n_blocks is set
// (out.val stays empty)
void crs_to_bcrs(const DevCRS &a, int vbytes, int64_t bh, int64_t bw, int64_t hpad, int64_t wpad, bool col_major,
                 DevBCRS &out, cudaStream_t st, int64_t max_blocks = -1);

// Y = A X with k right-hand sides.  Row-major: X[col*k+v], Y[row*k+v].
// Column-major: X[ldx*v+col], Y[row+ldy*v] (the reference uses A's n_rows as
// the leading dimension of X and Y, src/kernels/spmm/spmm_cpu/spmm_cpu_crs_impl.hpp:29,44).
// Row-major SpMM launch plan.  variant 1: one thread group per row over a
// grid of all rows.  variant 2 ("walk"): one CTA per SM, each walking a
// contiguous, nonzero-balanced range of rows in order, so the X rows that
// neighbouring rows share can stay in that SM's L1 (an autotuner candidate:
// on the 27-point stencil it loses to the grid's occupancy).  variant 0: the
// grid.
struct SpmmPlan {
    DevBuf ranges;  // int64 row bounds of the walk CTAs, grid + 1 entries
    int grid = 0;
    const void *key = nullptr;
    int64_t n = -1, nnz = -1;
};
template <typename VT>
void crs_spmm_row_major(const DevCRS &a, int64_t k, const VT *X, VT *Y, cudaStream_t st, SpmmPlan *plan = nullptr,
                        int variant = 0);

}  // namespace smax
