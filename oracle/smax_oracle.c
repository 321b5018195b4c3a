/*
 * smax_oracle.c -- plain-C restatement of the SmaxKernels CPU algorithms on the
 * sparse hot path.  TEST INFRASTRUCTURE ONLY: tests/, __graft_entry__.smoke()
 * and bench.py's CPU-baseline leg load it (oracle/liboracle.so) as the checker;
 * the product never calls it.
 *
 * Each function restates, serially and in the reference's own summation order,
 * the reference routine named in its comment (paths are relative to the
 * SmaxKernels checkout).  Index type is int32, value type float or double.
 *
 * Parity status: pinned.  tests/test_oracle_golden.py checks every function
 * against the known-answer vectors of the reference's unit tests
 * (examples/tests/*.hpp, extracted to tests/golden/ by tests/golden/make_golden.py)
 * and, where the reference is built (oracle/_ref), against the reference itself
 * on seeded random inputs.
 *
 * Tie order.  convert_crs_to_scs sorts each sigma-window with std::sort by
 * descending row length (src/utils/convert_formats.hpp:46-55).  std::sort is
 * only guaranteed to be stable for windows of at most 16 rows (libstdc++ then
 * runs a pure insertion sort); this restatement always breaks ties by ascending
 * original row, which equals the reference whenever sigma <= 16 or no two rows
 * of a window have the same length.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <math.h>

typedef int32_t I;

#define ORC_OK 0
#define ORC_ERR_ZERO_DIAG (-4)
#define ORC_ERR_NO_DIAG (-5)
#define ORC_ERR_ARG (-1)

/* ------------------------------------------------------------------------ *
 * Value-typed kernels, instantiated for double (f64) and float (f32).
 * ------------------------------------------------------------------------ */
#define ORC_VALUE_KERNELS(VT, SFX)                                              \
                                                                                \
/* src/kernels/spmv/spmv_cpu/spmv_cpu_crs_impl.hpp:9-38 */                      \
void orc_spmv_crs_##SFX(int64_t n_rows, const I *col, const I *row_ptr,         \
                        const VT *val, const VT *x, VT *y) {                    \
    for (int64_t r = 0; r < n_rows; ++r) {                                      \
        VT sum = (VT)0;                                                         \
        for (I j = row_ptr[r]; j < row_ptr[r + 1]; ++j)                         \
            sum += val[j] * x[col[j]];                                          \
        y[r] = sum;                                                             \
    }                                                                           \
}                                                                               \
                                                                                \
/* src/kernels/spmv/spmv_cpu/spmv_cpu_scs_impl.hpp:9-49: chunk c covers rows   \
 * c*C..c*C+C-1 of the permuted order; element (row i, slot j) of chunk c is   \
 * at chunk_ptr[c] + j*C + i. */                                                \
void orc_spmv_scs_##SFX(int64_t C, int64_t n_chunks, const I *chunk_ptr,        \
                        const I *chunk_lengths, const I *col, const VT *val,    \
                        const VT *x, VT *y) {                                   \
    for (int64_t c = 0; c < n_chunks; ++c) {                                    \
        for (int64_t i = 0; i < C; ++i) {                                       \
            VT sum = (VT)0;                                                     \
            for (I j = 0; j < chunk_lengths[c]; ++j) {                          \
                int64_t idx = (int64_t)chunk_ptr[c] + (int64_t)j * C + i;       \
                sum += val[idx] * x[col[idx]];                                  \
            }                                                                   \
            y[c * C + i] = sum;                                                 \
        }                                                                       \
    }                                                                           \
}                                                                               \
                                                                                \
/* src/kernels/spmv/spmv_cpu/spmv_cpu_bcrs_impl.hpp:19-85: block j of block   \
 * row r starts at val[j*hpad*wpad]; in-block element (ix, jx) is at          \
 * jx*hpad+ix (column-major) or ix*wpad+jx (row-major); x is indexed by        \
 * col[j]*wpad+jx and y by r*hpad+ix. */                                        \
void orc_spmv_bcrs_##SFX(int64_t n_rows, int64_t bh, int64_t bw, int64_t hpad,  \
                         int64_t wpad, const I *col, const I *row_ptr,          \
                         const VT *val, int col_major, const VT *x, VT *y) {    \
    int64_t bs = hpad * wpad;                                                   \
    VT *acc = (VT *)malloc(sizeof(VT) * (size_t)(bh > 0 ? bh : 1));             \
    for (int64_t r = 0; r < n_rows; ++r) {                                      \
        for (int64_t ix = 0; ix < bh; ++ix)                                     \
            acc[ix] = (VT)0;                                                    \
        for (I j = row_ptr[r]; j < row_ptr[r + 1]; ++j) {                       \
            const VT *blk = val + (int64_t)j * bs;                              \
            const VT *xb = x + (int64_t)col[j] * wpad;                          \
            if (col_major) {                                                    \
                for (int64_t jx = 0; jx < bw; ++jx)                             \
                    for (int64_t ix = 0; ix < bh; ++ix)                         \
                        acc[ix] += blk[jx * hpad + ix] * xb[jx];                \
            } else {                                                            \
                for (int64_t ix = 0; ix < bh; ++ix)                             \
                    for (int64_t jx = 0; jx < bw; ++jx)                         \
                        acc[ix] += blk[ix * wpad + jx] * xb[jx];                \
            }                                                                   \
        }                                                                       \
        for (int64_t ix = 0; ix < bh; ++ix)                                     \
            y[r * hpad + ix] = acc[ix];                                         \
    }                                                                           \
    free(acc);                                                                  \
}                                                                               \
                                                                                \
/* src/kernels/spmm/spmm_cpu/spmm_cpu_crs_impl.hpp:9-89.  Row-major:          \
 * X[col*k+v], Y[row*k+v].  Column-major: X[n_rows*v+col] and                  \
 * Y[row+v*n_rows] -- the reference uses A's n_rows as the leading dimension   \
 * of X as well (:29,44). */                                                    \
void orc_spmm_##SFX(int row_major, int64_t n_rows, const I *col,                \
                    const I *row_ptr, const VT *val, int64_t k, const VT *X,    \
                    VT *Y) {                                                    \
    for (int64_t r = 0; r < n_rows; ++r) {                                      \
        for (int64_t v = 0; v < k; ++v) {                                       \
            VT sum = (VT)0;                                                     \
            for (I j = row_ptr[r]; j < row_ptr[r + 1]; ++j) {                   \
                VT xv = row_major ? X[(int64_t)col[j] * k + v]                  \
                                  : X[n_rows * v + col[j]];                     \
                sum += val[j] * xv;                                             \
            }                                                                   \
            if (row_major)                                                      \
                Y[r * k + v] = sum;                                             \
            else                                                                \
                Y[r + v * n_rows] = sum;                                        \
        }                                                                       \
    }                                                                           \
}                                                                               \
                                                                                \
/* src/kernels/spgemm/spgemm_cpu/numerical_phase_impl.hpp:9-91: products are  \
 * accumulated in (j over A's row, k over B's row) order into a dense row      \
 * accumulator, then gathered in C's column order. */                          \
void orc_spgemm_numeric_##SFX(int64_t a_n_rows, const I *a_col,                 \
                              const I *a_row_ptr, const VT *a_val,              \
                              const I *b_col, const I *b_row_ptr,               \
                              const VT *b_val, int64_t c_n_cols,                \
                              const I *c_col, const I *c_row_ptr, VT *c_val) {  \
    VT *acc = (VT *)calloc((size_t)(c_n_cols > 0 ? c_n_cols : 1), sizeof(VT));  \
    for (int64_t i = 0; i < a_n_rows; ++i) {                                    \
        for (I j = a_row_ptr[i]; j < a_row_ptr[i + 1]; ++j) {                   \
            I lc = a_col[j];                                                    \
            for (I k = b_row_ptr[lc]; k < b_row_ptr[lc + 1]; ++k)               \
                acc[b_col[k]] += a_val[j] * b_val[k];                           \
        }                                                                       \
        for (I j = c_row_ptr[i]; j < c_row_ptr[i + 1]; ++j) {                   \
            c_val[j] = acc[c_col[j]];                                           \
            acc[c_col[j]] = (VT)0;                                              \
        }                                                                       \
    }                                                                           \
    free(acc);                                                                  \
}                                                                               \
                                                                                \
/* src/kernels/sptrsv/sptrsv_cpu/sptrsv_cpu_crs_helpers_impl.hpp:9-38: copies \
 * the diagonal to D and swaps the diagonal entry to the last slot of its row  \
 * (mutating col/val).  A diagonal with |d| < 1e-16 or no diagonal at all is   \
 * fatal in the reference; here it returns an error code and *bad_row. */      \
int orc_peel_diag_##SFX(int64_t n_rows, I *col, const I *row_ptr, VT *val,     \
                        VT *D, int64_t *bad_row) {                              \
    for (int64_t r = 0; r < n_rows; ++r) {                                      \
        I rs = row_ptr[r], re = row_ptr[r + 1] - 1;                             \
        int64_t dj = -1;                                                        \
        for (I j = rs; j <= re; ++j) {                                          \
            if (col[j] == (I)r) {                                               \
                dj = j;                                                         \
                D[r] = val[j];                                                  \
                if (fabs((double)D[r]) < 1e-16) {                               \
                    if (bad_row) *bad_row = r;                                  \
                    return ORC_ERR_ZERO_DIAG;                                   \
                }                                                               \
            }                                                                   \
        }                                                                       \
        if (dj < 0) {                                                           \
            if (bad_row) *bad_row = r;                                          \
            return ORC_ERR_NO_DIAG;                                             \
        }                                                                       \
        if ((I)dj != re) {                                                      \
            I tc = col[dj]; col[dj] = col[re]; col[re] = tc;                    \
            VT tv = val[dj]; val[dj] = val[re]; val[re] = tv;                   \
        }                                                                       \
    }                                                                           \
    return ORC_OK;                                                              \
}                                                                               \
                                                                                \
/* src/kernels/sptrsv/sptrsv_cpu/sptrsv_cpu_crs_impl.hpp:9-55 (diagonal       \
 * already peeled to the row end): x[r] = (b[r] - sum_{j<end-1} val*x[col])    \
 * / D[r], rows forward (lower) or backward (upper). */                         \
void orc_sptrsv_##SFX(int lower, int64_t n_rows, const I *col,                  \
                      const I *row_ptr, const VT *val, const VT *D, VT *x,      \
                      const VT *b) {                                            \
    for (int64_t t = 0; t < n_rows; ++t) {                                      \
        int64_t r = lower ? t : n_rows - 1 - t;                                 \
        VT sum = (VT)0;                                                         \
        for (I j = row_ptr[r]; j < row_ptr[r + 1] - 1; ++j)                     \
            sum += val[j] * x[col[j]];                                          \
        x[r] = (b[r] - sum) / D[r];                                             \
    }                                                                           \
}                                                                               \
                                                                                \
/* src/kernels/sptrsv/sptrsv_cpu/sptrsv_lvl_cpu_crs_impl.hpp:11-82: the same  \
 * row recurrence, rows of level l are [lvl_ptr[l], lvl_ptr[l+1]); levels run  \
 * in ascending (lower) or descending (upper) order. */                         \
void orc_sptrsv_lvl_##SFX(int lower, int n_levels, const int *lvl_ptr,          \
                          const I *col, const I *row_ptr, const VT *val,        \
                          const VT *D, VT *x, const VT *b) {                    \
    for (int t = 0; t < n_levels; ++t) {                                        \
        int l = lower ? t : n_levels - 1 - t;                                   \
        for (int r = lvl_ptr[l]; r < lvl_ptr[l + 1]; ++r) {                     \
            VT sum = (VT)0;                                                     \
            for (I j = row_ptr[r]; j < row_ptr[r + 1] - 1; ++j)                 \
                sum += val[j] * x[col[j]];                                      \
            x[r] = (b[r] - sum) / D[r];                                         \
        }                                                                       \
    }                                                                           \
}                                                                               \
                                                                                \
/* src/kernels/sptrsm/sptrsm_cpu/sptrsm_cpu_crs_impl.hpp:9-102: SpTRSV per    \
 * right-hand side; row-major X[row*k+v], column-major X[row+n_rows*v]. */      \
void orc_sptrsm_##SFX(int row_major, int lower, int64_t n_rows, const I *col,   \
                      const I *row_ptr, const VT *val, const VT *D, int64_t k,  \
                      VT *X, const VT *B) {                                     \
    for (int64_t t = 0; t < n_rows; ++t) {                                      \
        int64_t r = lower ? t : n_rows - 1 - t;                                 \
        for (int64_t v = 0; v < k; ++v) {                                       \
            VT sum = (VT)0;                                                     \
            for (I j = row_ptr[r]; j < row_ptr[r + 1] - 1; ++j) {               \
                VT xv = row_major ? X[(int64_t)col[j] * k + v]                  \
                                  : X[n_rows * v + col[j]];                     \
                sum += val[j] * xv;                                             \
            }                                                                   \
            if (row_major)                                                      \
                X[r * k + v] = (B[r * k + v] - sum) / D[r];                     \
            else                                                                \
                X[r + n_rows * v] = (B[r + n_rows * v] - sum) / D[r];           \
        }                                                                       \
    }                                                                           \
}                                                                               \
                                                                                \
/* src/utils/convert_formats.hpp:93-128: zero-filled chunk-column-major      \
 * scatter of the CRS rows into SELL-C-sigma, given perm[old] = new. */         \
void orc_scs_fill_##SFX(int64_t n_rows, int64_t C, const I *row_ptr,            \
                        const I *col, const VT *val, const I *chunk_ptr,        \
                        const I *perm, int64_t n_elements, I *o_col,            \
                        VT *o_val) {                                            \
    memset(o_col, 0, sizeof(I) * (size_t)n_elements);                           \
    memset(o_val, 0, sizeof(VT) * (size_t)n_elements);                          \
    for (int64_t r = 0; r < n_rows; ++r) {                                      \
        int64_t nr = perm[r];                                                   \
        int64_t base = (int64_t)chunk_ptr[nr / C] + nr % C;                     \
        int64_t k = 0;                                                          \
        for (I j = row_ptr[r]; j < row_ptr[r + 1]; ++j, ++k) {                  \
            o_col[base + k * C] = col[j];                                       \
            o_val[base + k * C] = val[j];                                       \
        }                                                                       \
    }                                                                           \
}                                                                               \
                                                                                \
/* src/utils/convert_formats.hpp:223-243: zero-filled blocks, each CRS entry   \
 * written to block (row/bh, col/bw) at in-block index                        \
 * col_major ? hpad*(col%bw)+lrow : wpad*lrow+col%bw. */                        \
void orc_bcrs_fill_##SFX(int64_t n_brows, int64_t bh, int64_t bw,               \
                         int64_t hpad, int64_t wpad, int col_major,             \
                         const I *row_ptr, const I *col, const VT *val,         \
                         const I *b_row_ptr, const I *b_col, VT *b_val) {       \
    int64_t bs = hpad * wpad;                                                   \
    memset(b_val, 0, sizeof(VT) * (size_t)(b_row_ptr[n_brows] * bs));           \
    for (int64_t br = 0; br < n_brows; ++br) {                                  \
        for (int64_t lr = 0; lr < bh; ++lr) {                                   \
            int64_t r = br * bh + lr;                                           \
            for (I j = row_ptr[r]; j < row_ptr[r + 1]; ++j) {                   \
                I bc = col[j] / (I)bw;                                          \
                /* sorted unique block columns of this block row */             \
                I lo = b_row_ptr[br], hi = b_row_ptr[br + 1];                   \
                while (lo < hi) {                                               \
                    I mid = lo + (hi - lo) / 2;                                 \
                    if (b_col[mid] < bc) lo = mid + 1; else hi = mid;           \
                }                                                               \
                int64_t in = col_major ? hpad * (col[j] % bw) + lr              \
                                       : wpad * lr + col[j] % bw;               \
                b_val[(int64_t)lo * bs + in] = val[j];                          \
            }                                                                   \
        }                                                                       \
    }                                                                           \
}                                                                               \
                                                                                \
/* src/utils/permutations.hpp:820-861: row r of the permuted matrix is old    \
 * row perm[r]; its columns are mapped through inv_perm, in-row order kept. */  \
void orc_apply_mat_perm_##SFX(int64_t n_rows, const I *row_ptr, const I *col,   \
                              const VT *val, I *p_row_ptr, I *p_col,            \
                              VT *p_val, const int *perm,                       \
                              const int *inv_perm) {                            \
    p_row_ptr[0] = 0;                                                           \
    for (int64_t r = 0; r < n_rows; ++r)                                        \
        p_row_ptr[r + 1] = p_row_ptr[r] + (row_ptr[perm[r] + 1] -               \
                                           row_ptr[perm[r]]);                   \
    for (int64_t r = 0; r < n_rows; ++r) {                                      \
        I o = row_ptr[perm[r]];                                                 \
        for (I p = p_row_ptr[r]; p < p_row_ptr[r + 1]; ++p, ++o) {              \
            p_col[p] = inv_perm[col[o]];                                        \
            p_val[p] = val[o];                                                  \
        }                                                                       \
    }                                                                           \
}                                                                               \
                                                                                \
/* src/utils/permutations.hpp:863-874: vec_perm[i] = vec[perm[i]]. */           \
void orc_apply_vec_perm_##SFX(int64_t n, const VT *vec, VT *vec_perm,           \
                              const int *perm) {                                \
    for (int64_t i = 0; i < n; ++i)                                             \
        vec_perm[i] = vec[perm[i]];                                             \
}

ORC_VALUE_KERNELS(double, f64)
ORC_VALUE_KERNELS(float, f32)

/* ------------------------------------------------------------------------ *
 * Integer / pattern routines.
 * ------------------------------------------------------------------------ */

/* src/kernels/spgemm/spgemm_cpu/symbolic_phase_impl.hpp:86-127: per row of C,
 * the distinct columns of B reached through A's row, counted.  */
void orc_spgemm_row_counts(int64_t a_n_rows, const I *a_col, const I *a_row_ptr,
                           int64_t b_n_cols, const I *b_col, const I *b_row_ptr,
                           I *c_row_nnz) {
    unsigned char *used = (unsigned char *)calloc((size_t)(b_n_cols > 0 ? b_n_cols : 1), 1);
    I *touched = (I *)malloc(sizeof(I) * (size_t)(b_n_cols > 0 ? b_n_cols : 1));
    for (int64_t i = 0; i < a_n_rows; ++i) {
        I cnt = 0;
        for (I j = a_row_ptr[i]; j < a_row_ptr[i + 1]; ++j) {
            I lc = a_col[j];
            for (I k = b_row_ptr[lc]; k < b_row_ptr[lc + 1]; ++k) {
                I rc = b_col[k];
                if (!used[rc]) {
                    used[rc] = 1;
                    touched[cnt++] = rc;
                }
            }
        }
        for (I t = 0; t < cnt; ++t)
            used[touched[t]] = 0;
        c_row_nnz[i] = cnt;
    }
    free(used);
    free(touched);
}

/* Same traversal, writing each row's distinct columns in FIRST-TOUCH order
 * (the order the reference stores them, :102-113 then :155-163) at
 * c_row_ptr[i]. */
void orc_spgemm_fill_cols(int64_t a_n_rows, const I *a_col, const I *a_row_ptr,
                          int64_t b_n_cols, const I *b_col, const I *b_row_ptr,
                          const I *c_row_ptr, I *c_col) {
    unsigned char *used = (unsigned char *)calloc((size_t)(b_n_cols > 0 ? b_n_cols : 1), 1);
    for (int64_t i = 0; i < a_n_rows; ++i) {
        I p = c_row_ptr[i];
        for (I j = a_row_ptr[i]; j < a_row_ptr[i + 1]; ++j) {
            I lc = a_col[j];
            for (I k = b_row_ptr[lc]; k < b_row_ptr[lc + 1]; ++k) {
                I rc = b_col[k];
                if (!used[rc]) {
                    used[rc] = 1;
                    c_col[p++] = rc;
                }
            }
        }
        for (I t = c_row_ptr[i]; t < p; ++t)
            used[c_col[t]] = 0;
    }
    free(used);
}

/* src/utils/convert_formats.hpp:27-30,57-78: n_chunks = ceil(n/C),
 * n_rows_padded = n_chunks*C, chunk length = longest row of the chunk after
 * the sigma-window sort.  Returns the permutation perm[old] = new (:81-86),
 * chunk_lengths and chunk_ptr; *n_elements = chunk_ptr[n_chunks].
 *
 * The window sort (:46-55) is std::sort over (index, count) pairs with the
 * comparator a.count > b.count.  That sort is not stable: rows of equal
 * length end up in whatever order the library's algorithm leaves them.  The
 * reference is built with GCC 13.3, whose libstdc++ std::sort is the
 * published introsort restated below (and in the GPU conversion,
 * smaxkernels_b200/csrc/scs_window_sort.cuh), so the permutation is
 * reproduced exactly:
 *   sort(a, n):  if n > 0: introsort_loop(a, 0, n, 2*floor(log2 n));
 *                          final_insertion_sort(a, 0, n)
 *   introsort_loop(lo, hi, depth): while hi - lo > 16:
 *       depth == 0 -> heapsort [lo, hi) (make_heap + sort_heap), return;
 *       --depth; cut = partition around the median of a[lo+1], a[mid],
 *       a[hi-1] moved to a[lo]; introsort_loop(cut, hi, depth); hi = cut
 *   final_insertion_sort: insertion sort of the first 16, then unguarded
 *       insertion of the rest (plain insertion sort when n <= 16). */
typedef struct { int idx; int cnt; } orc_pair;

/* the reference's comparator: longer rows first */
static int orc_before(orc_pair x, orc_pair y) { return x.cnt > y.cnt; }

static void orc_swap(orc_pair *a, int64_t i, int64_t j) {
    orc_pair t = a[i];
    a[i] = a[j];
    a[j] = t;
}

static void orc_median_to_first(orc_pair *a, int64_t r, int64_t x, int64_t y, int64_t z) {
    if (orc_before(a[x], a[y])) {
        if (orc_before(a[y], a[z])) orc_swap(a, r, y);
        else if (orc_before(a[x], a[z])) orc_swap(a, r, z);
        else orc_swap(a, r, x);
    } else if (orc_before(a[x], a[z])) {
        orc_swap(a, r, x);
    } else if (orc_before(a[y], a[z])) {
        orc_swap(a, r, z);
    } else {
        orc_swap(a, r, y);
    }
}

/* Hoare partition of [lo, hi) around a[pivot]; no bounds checks needed
 * because the median-of-three leaves sentinels on both sides */
static int64_t orc_partition(orc_pair *a, int64_t lo, int64_t hi, int64_t pivot) {
    for (;;) {
        while (orc_before(a[lo], a[pivot])) ++lo;
        --hi;
        while (orc_before(a[pivot], a[hi])) --hi;
        if (!(lo < hi)) return lo;
        orc_swap(a, lo, hi);
        ++lo;
    }
}

/* sift `v` down from `hole` in the heap a[base .. base+len), then up to `top` */
static void orc_adjust_heap(orc_pair *a, int64_t base, int64_t hole, int64_t len, orc_pair v) {
    const int64_t top = hole;
    int64_t child = hole;
    while (child < (len - 1) / 2) {
        child = 2 * (child + 1);
        if (orc_before(a[base + child], a[base + child - 1])) --child;
        a[base + hole] = a[base + child];
        hole = child;
    }
    if ((len & 1) == 0 && child == (len - 2) / 2) {
        child = 2 * (child + 1);
        a[base + hole] = a[base + child - 1];
        hole = child - 1;
    }
    int64_t parent = (hole - 1) / 2;
    while (hole > top && orc_before(a[base + parent], v)) {
        a[base + hole] = a[base + parent];
        hole = parent;
        parent = (hole - 1) / 2;
    }
    a[base + hole] = v;
}

static void orc_heapsort(orc_pair *a, int64_t lo, int64_t hi) {
    const int64_t len = hi - lo;
    if (len >= 2)
        for (int64_t parent = (len - 2) / 2;; --parent) {
            orc_adjust_heap(a, lo, parent, len, a[lo + parent]);
            if (parent == 0) break;
        }
    for (int64_t last = hi; last - lo > 1;) {
        --last;
        orc_pair v = a[last];
        a[last] = a[lo];
        orc_adjust_heap(a, lo, 0, last - lo, v);
    }
}

static void orc_linear_insert(orc_pair *a, int64_t i) {
    orc_pair v = a[i];
    int64_t j = i - 1;
    while (orc_before(v, a[j])) {
        a[i] = a[j];
        i = j;
        --j;
    }
    a[i] = v;
}

static void orc_insertion_sort(orc_pair *a, int64_t lo, int64_t hi) {
    if (lo == hi) return;
    for (int64_t i = lo + 1; i < hi; ++i) {
        if (orc_before(a[i], a[lo])) {
            orc_pair v = a[i];
            for (int64_t j = i; j > lo; --j) a[j] = a[j - 1];
            a[lo] = v;
        } else {
            orc_linear_insert(a, i);
        }
    }
}

static void orc_introsort_loop(orc_pair *a, int64_t lo, int64_t hi, int depth) {
    while (hi - lo > 16) {
        if (depth == 0) {
            orc_heapsort(a, lo, hi);
            return;
        }
        --depth;
        const int64_t mid = lo + (hi - lo) / 2;
        orc_median_to_first(a, lo, lo + 1, mid, hi - 1);
        const int64_t cut = orc_partition(a, lo + 1, hi, lo);
        orc_introsort_loop(a, cut, hi, depth);
        hi = cut;
    }
}

static void orc_std_sort_window(orc_pair *a, int64_t n) {
    if (n <= 0) return;
    int lg = 0;
    while (((int64_t)1 << (lg + 1)) <= n) ++lg;
    orc_introsort_loop(a, 0, n, 2 * lg);
    if (n > 16) {
        orc_insertion_sort(a, 0, 16);
        for (int64_t i = 16; i < n; ++i) orc_linear_insert(a, i);
    } else {
        orc_insertion_sort(a, 0, n);
    }
}

int orc_scs_layout(int64_t n_rows, const I *row_ptr, int64_t C, int64_t sigma,
                   I *chunk_ptr, I *chunk_lengths, I *perm,
                   int64_t *n_elements) {
    if (C <= 0 || sigma <= 0) return ORC_ERR_ARG;
    int64_t n_chunks = (n_rows + C - 1) / C;
    int64_t npad = n_chunks * C;
    orc_pair *e = (orc_pair *)malloc(sizeof(orc_pair) * (size_t)(npad > 0 ? npad : 1));
    for (int64_t i = 0; i < npad; ++i) {
        e[i].idx = (int)i;
        e[i].cnt = i < n_rows ? (int)(row_ptr[i + 1] - row_ptr[i]) : 0;
    }
    for (int64_t w = 0; w < npad; w += sigma) {
        int64_t len = (w + sigma < npad) ? sigma : npad - w;
        orc_std_sort_window(e + w, len);
    }
    I cur = 0;
    for (int64_t c = 0; c < n_chunks; ++c) {
        int mx = 0;
        for (int64_t i = 0; i < C; ++i)
            if (e[c * C + i].cnt > mx) mx = e[c * C + i].cnt;
        chunk_lengths[c] = mx;
        chunk_ptr[c] = cur;
        cur += (I)(mx * C);
    }
    chunk_ptr[n_chunks] = cur;
    for (int64_t i = 0; i < npad; ++i)
        if (e[i].idx < n_rows) perm[e[i].idx] = (I)i;
    *n_elements = cur;
    free(e);
    return ORC_OK;
}

/* src/utils/convert_formats.hpp:175-206: per block row, the sorted set of
 * block columns col/bw over its bh rows; b_row_ptr by prefix sum.  Pass
 * b_col = NULL to only count (b_row_ptr is always filled). */
static int orc_cmp_int(const void *a, const void *b) {
    I x = *(const I *)a, y = *(const I *)b;
    return (x > y) - (x < y);
}

int orc_bcrs_pattern(int64_t n_rows, int64_t n_cols, const I *row_ptr,
                     const I *col, int64_t bh, int64_t bw, I *b_row_ptr,
                     I *b_col) {
    if (bh <= 0 || bw <= 0 || n_rows % bh || n_cols % bw) return ORC_ERR_ARG;
    int64_t nb = n_rows / bh;
    b_row_ptr[0] = 0;
    I *tmp = NULL;
    size_t cap = 0;
    for (int64_t br = 0; br < nb; ++br) {
        I s = row_ptr[br * bh], e = row_ptr[(br + 1) * bh];
        size_t m = (size_t)(e - s);
        if (m > cap) {
            cap = m * 2;
            tmp = (I *)realloc(tmp, sizeof(I) * cap);
        }
        for (I j = s; j < e; ++j) tmp[j - s] = col[j] / (I)bw;
        qsort(tmp, m, sizeof(I), orc_cmp_int);
        I u = 0;
        for (size_t t = 0; t < m; ++t)
            if (t == 0 || tmp[t] != tmp[t - 1]) {
                if (b_col) b_col[b_row_ptr[br] + u] = tmp[t];
                ++u;
            }
        b_row_ptr[br + 1] = b_row_ptr[br] + u;
    }
    free(tmp);
    return ORC_OK;
}

/* src/utils/permutations.hpp:236-392 (build_symmetric_crs_parallel_adapted)
 * run with ONE OpenMP thread: row c of A+A^T is A's row c as stored, followed
 * by every r (ascending) whose row holds c != r while row c does not hold r.
 * Pass sym_col = NULL to only compute sym_row_ptr. */
void orc_build_symmetric(int64_t n, const I *row_ptr, const I *col,
                         I *sym_row_ptr, I *sym_col) {
    I *extra = (I *)calloc((size_t)(n > 0 ? n : 1), sizeof(I));
    for (int64_t r = 0; r < n; ++r)
        for (I j = row_ptr[r]; j < row_ptr[r + 1]; ++j) {
            I c = col[j];
            if (c != r && c >= 0 && c < n) {
                int has = 0;
                for (I k = row_ptr[c]; k < row_ptr[c + 1]; ++k)
                    if (col[k] == r) { has = 1; break; }
                if (!has) extra[c]++;
            }
        }
    sym_row_ptr[0] = 0;
    for (int64_t r = 0; r < n; ++r)
        sym_row_ptr[r + 1] = sym_row_ptr[r] + (row_ptr[r + 1] - row_ptr[r]) + extra[r];
    if (sym_col) {
        I *fill = (I *)malloc(sizeof(I) * (size_t)(n > 0 ? n : 1));
        for (int64_t r = 0; r < n; ++r) {
            I p = sym_row_ptr[r];
            for (I j = row_ptr[r]; j < row_ptr[r + 1]; ++j) sym_col[p++] = col[j];
            fill[r] = p;
        }
        for (int64_t r = 0; r < n; ++r)
            for (I j = row_ptr[r]; j < row_ptr[r + 1]; ++j) {
                I c = col[j];
                if (c != r && c >= 0 && c < n) {
                    int has = 0;
                    for (I k = row_ptr[c]; k < row_ptr[c + 1]; ++k)
                        if (col[k] == r) { has = 1; break; }
                    if (!has) sym_col[fill[c]++] = (I)r;
                }
            }
        free(fill);
    }
    free(extra);
}

/* src/utils/permutations.hpp:394-414: lvl[r] = 1 + max lvl over neighbours
 * c < r of the symmetric pattern (0 if none).  Returns n_levels. */
int orc_levels_rs(int64_t n, const I *sym_row_ptr, const I *sym_col, int *lvl) {
    int mx = 0;
    for (int64_t r = 0; r < n; ++r) {
        int l = 0;
        for (I j = sym_row_ptr[r]; j < sym_row_ptr[r + 1]; ++j) {
            I c = sym_col[j];
            if (c < r && lvl[c] + 1 > l) l = lvl[c] + 1;
        }
        lvl[r] = l;
        if (l > mx) mx = l;
    }
    return n > 0 ? mx + 1 : 1;
}

/* src/utils/permutations.hpp:416-483 with ONE OpenMP thread: roots (no
 * neighbour below) queued in ascending order; a node's level is set when it
 * leaves the queue; while visiting u, each neighbour v (in u's symmetric row
 * order) is queued if unvisited and none of v's lower neighbours is still
 * unlevelled.  perm = dequeue order.  Returns n_levels. */
int orc_perm_bfs(int64_t n, const I *sym_row_ptr, const I *sym_col, int *perm,
                 int *lvl) {
    unsigned char *vis = (unsigned char *)calloc((size_t)(n > 0 ? n : 1), 1);
    int *q = (int *)malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
    int64_t head = 0, tail = 0;
    for (int64_t i = 0; i < n; ++i) lvl[i] = -1;
    for (int64_t s = 0; s < n; ++s) {
        int root = 1;
        for (I j = sym_row_ptr[s]; j < sym_row_ptr[s + 1]; ++j)
            if (sym_col[j] < s) { root = 0; break; }
        if (root) { q[tail++] = (int)s; vis[s] = 1; }
    }
    int cur = 0, mx = 0;
    int64_t pi = 0;
    while (head < tail) {
        int64_t lsz = tail - head;
        for (int64_t t = 0; t < lsz; ++t) {
            int u = q[head++];
            perm[pi++] = u;
            lvl[u] = cur;
            if (cur > mx) mx = cur;
            for (I jj = sym_row_ptr[u]; jj < sym_row_ptr[u + 1]; ++jj) {
                I v = sym_col[jj];
                int dep = 0;
                for (I k = sym_row_ptr[v]; k < sym_row_ptr[v + 1]; ++k)
                    if (sym_col[k] < v && lvl[sym_col[k]] == -1) { dep = 1; break; }
                if (!vis[v] && !dep) { vis[v] = 1; q[tail++] = v; }
            }
        }
        ++cur;
    }
    free(vis);
    free(q);
    return mx + 1;
}

/* src/utils/permutations.hpp:485-584 for type RS (1), BFS (0) or NONE (2):
 * builds A+A^T, computes levels, perm (BFS: queue order; otherwise stable
 * sort of the identity by level), inv_perm, and lvl_ptr (capacity n+1).
 * Returns n_levels or a negative error. */
int orc_generate_perm(int64_t n, const I *row_ptr, const I *col, int type,
                      int *perm, int *inv_perm, int *lvl_ptr) {
    I *srp = (I *)malloc(sizeof(I) * (size_t)(n + 1));
    orc_build_symmetric(n, row_ptr, col, srp, NULL);
    I *scol = (I *)malloc(sizeof(I) * (size_t)(srp[n] > 0 ? srp[n] : 1));
    orc_build_symmetric(n, row_ptr, col, srp, scol);
    int *lvl = (int *)malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
    for (int64_t i = 0; i < n; ++i) lvl[i] = -1;
    int nl;
    if (type == 0) {
        nl = orc_perm_bfs(n, srp, scol, perm, lvl);
    } else if (type == 1) {
        nl = orc_levels_rs(n, srp, scol, lvl);
    } else if (type == 2) {
        for (int64_t i = 0; i < n; ++i) lvl[i] = (int)i;
        nl = (int)n;
    } else {
        free(srp); free(scol); free(lvl);
        return ORC_ERR_ARG;
    }
    int *cnt = (int *)calloc((size_t)nl + 1, sizeof(int));
    for (int64_t i = 0; i < n; ++i) cnt[lvl[i]]++;
    lvl_ptr[0] = 0;
    for (int l = 0; l < nl; ++l) lvl_ptr[l + 1] = lvl_ptr[l] + cnt[l];
    if (type != 0) {
        /* stable counting sort by level == std::stable_sort of the identity */
        int *pos = (int *)malloc(sizeof(int) * ((size_t)nl + 1));
        for (int l = 0; l <= nl; ++l) pos[l] = lvl_ptr[l];
        for (int64_t i = 0; i < n; ++i) perm[pos[lvl[i]]++] = (int)i;
        free(pos);
    }
    for (int64_t i = 0; i < n; ++i) inv_perm[perm[i]] = (int)i;
    free(cnt);
    free(srp);
    free(scol);
    free(lvl);
    return nl;
}
