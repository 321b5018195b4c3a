// spmv_crs.cuh -- CRS SpMV plan and launcher (see spmv_crs.cu).
#pragma once

#include "common.cuh"

namespace smax {

// Row tiles of one CRS matrix: tiles[t] .. tiles[t+1] are the rows of tile t.
struct CrsTilePlan {
    DevBuf tiles;
    int n_tiles = 0;
    int cap = 0;
    int64_t n_rows = 0;
    void build(const int *d_row_ptr, int64_t n_rows, int cap, cudaStream_t st);
};

int crs_default_cap(int vbits);

// Warp-stream plan (spmv_crs_stream.cu): fixed 512-entry slices, row-end bit
// mask, per-slice rank of the open row, carries for rows crossing slices.
struct CrsStreamPlan {
    int64_t n_rows = 0, nnz = 0, n_tasks = 0, n_empty = 0, n_nonempty = 0;
    const int *row_ptr = nullptr;  // the matrix's device row pointer given to build (not owned)
    bool short_rows = true;        // no row has more than 32 entries: slices need no carries
    DevBuf endbits, task_rank, carry_val, carry_rank, row_list, empty_rows;
    void build(const int *d_row_ptr, int64_t n_rows, int64_t nnz, int vbytes, cudaStream_t st);
};

// col/val of a matrix used with the warp-stream kernel must be allocated (and
// zero-filled) up to a multiple of this many entries.
int crs_stream_pad();

template <typename VT>
void crs_spmv_stream(const CrsStreamPlan &plan, const int *col, const VT *val, const VT *x, VT *y,
                     cudaStream_t st);

template <typename VT>
void crs_spmv(const CrsTilePlan &plan, const int *row_ptr, const int *col, const VT *val, const VT *x, VT *y,
              cudaStream_t st);

}  // namespace smax
