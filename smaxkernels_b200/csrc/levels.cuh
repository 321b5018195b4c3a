// levels.cuh -- level sets, permutations and A+A^T on the GPU (levels.cu).
#pragma once

#include <vector>

#include "spmv_formats.cuh"

namespace smax {

// A + A^T pattern (src/utils/permutations.hpp:236-392, one-thread order)
void build_symmetric(const DevCRS &a, DevBuf &sym_row_ptr, DevBuf &sym_col, int64_t &sym_nnz, cudaStream_t st);
// RS levels of a symmetric pattern; returns n_levels (lvl[] per row).  With
// rev the roles of lower and higher rows swap (levels of an upper triangle);
// with prio a node's earlier neighbours are those of smaller prio (a
// permutation of 0..n-1) instead of smaller index.
int rs_levels(const int *srp, const int *scol, int64_t n, DevBuf &lvl, cudaStream_t st, bool rev = false,
              const int *prio = nullptr);
// rows sorted by (level, row) and the level pointer (host) of n_levels levels
void level_order(const int *lvl, int64_t n, int n_levels, DevBuf &order, std::vector<int> &lvl_ptr, cudaStream_t st);
// the one-thread BFS queue order of generate_perm_BFS, from the level order;
// with first_discoverer, the queue order of a FIFO breadth-first search whose
// level sets (hop distances from the level-0 roots) are given instead
// (generate_color_perm's queue)
void bfs_order(const int *srp, const int *scol, int64_t n, const std::vector<int> &lvl_ptr, const int *order,
               DevBuf &perm, cudaStream_t st, bool first_discoverer = false);
void inverse_perm(const int *perm, int64_t n, int *inv, cudaStream_t st);

// Colourings of a symmetric pattern (colour.cu); each returns the number of
// colours and leaves colour[n]: generate_color_perm ("SC"),
// generate_color_perm_par ("PC") and generate_color_perm_bal ("PC_BAL",
// applied to a PC colouring in place) with one-thread semantics.
int colour_sc(const int *srp, const int *scol, int64_t n, DevBuf &colour, cudaStream_t st);
int colour_pc(const int *srp, const int *scol, int64_t n, DevBuf &colour, cudaStream_t st);
int colour_balance(const int *srp, const int *scol, int64_t n, DevBuf &colour, int n_colours, cudaStream_t st);
// sanity_check_perm: no row shares a non-zero colour with a lower neighbour
bool colours_valid(const int *rp, const int *col, int64_t n, const int *colour, int64_t *first_bad_row,
                   cudaStream_t st);
void apply_mat_perm(const DevCRS &a, const int *perm, const int *inv, int vbytes, DevCRS &out, cudaStream_t st);
void apply_vec_perm(const void *vec, const int *perm, int64_t n, int vbytes, void *out, cudaStream_t st);

}  // namespace smax
