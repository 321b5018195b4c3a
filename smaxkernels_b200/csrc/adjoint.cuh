// adjoint.cuh -- reverse-mode derivatives of SpMV and SpTRSV (adjoint.cu).
#pragma once

#include "spmv_crs.cuh"
#include "spmv_formats.cuh"

namespace smax {

// Transposed copy of a CRS matrix A (n x m): row c of At lists the entries of
// A's column c, ordered by ascending row of A (descending when asked), so the
// transposed products sum in a fixed order.  map[e] is the index in A of At's
// entry e; row_of[k] is the row of A's entry k.  At's col/val are padded for
// the warp-stream SpMV.
struct DevTranspose {
    DevCRS at;
    DevBuf map, row_of;
    CrsStreamPlan plan;
    bool built = false;
    bool descending = false;
    bool has_plan = false;
};

// row_of[k] = the row of entry k (warp per row).
void crs_row_of(const DevCRS &a, DevBuf &row_of, cudaStream_t st);

void build_transpose(const DevCRS &a, int vbytes, bool descending_rows, bool with_plan, DevTranspose &t,
                     cudaStream_t st);
// At.val[e] = A.val[map[e]] (after A's values changed)
void refresh_transpose_values(const DevCRS &a, int vbytes, DevTranspose &t, cudaStream_t st);

// dval[k] = s * g[row(k)] * x[col(k)] over A's pattern (a sampled outer product)
template <typename VT>
void sddmm_outer(const DevCRS &a, const int *row_of, VT s, const VT *g, const VT *x, VT *dval, cudaStream_t st);

// Checks that the last entry of every row of a square matrix is its
// diagonal (the layout the triangular kernels need); reports NO_DIAG.
void check_diag_last(const DevCRS &a, DevStatus *status, cudaStream_t st);

}  // namespace smax
