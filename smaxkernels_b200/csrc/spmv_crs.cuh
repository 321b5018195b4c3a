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

template <typename VT>
void crs_spmv(const CrsTilePlan &plan, const int *row_ptr, const int *col, const VT *val, const VT *x, VT *y,
              cudaStream_t st);

}  // namespace smax
