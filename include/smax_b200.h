/*
 * smax_b200.h -- C ABI of the SmaxKernels sm_100a (B200) CUDA platform.
 *
 * This is the boundary a SmaxKernels build binds to run its
 * PlatformType::CUDA kernels on a B200.  It replaces, one for one, the
 * reference's per-platform entry points
 *
 *   SPMV::initialize_cuda / apply_cuda / finalize_cuda
 *       (src/kernels/spmv/spmv_cuda.hpp:137-184, bodies in
 *        src/kernels/spmv/spmv_cuda/spmv_cuda_core.cuh:11-205)
 *
 * and adds the CUDA arms the reference lacks for SpMM, SpGEMM, SpTRSV and
 * SpTRSM (src/kernels/spmm.hpp:68-100, spgemm.hpp:91-130, sptrsv.hpp:74-113,
 * sptrsm.hpp:67-106 only dispatch to the CPU).  The objects mirror the
 * reference's own:
 *
 *   smax_ctx     <-> SMAX::Interface's UtilitiesContainer (level pointers
 *                    written by Utils::generate_perm, src/common.hpp:187-195)
 *   smax_kernel  <-> one registered SMAX::Kernel: KernelContext + Args + Flags
 *                    (src/kernel.hpp:7-127, src/kernels/<k>/<k>_common.hpp)
 *
 * Conventions
 *   - Every function returns smax_status: 0 on success, a negative SMAX_ERR_*
 *     code otherwise; smax_last_error() then holds a message for the calling
 *     thread.  Nothing here exits, aborts or traps.
 *   - Pointers given to register_* are HOST pointers owned by the caller, as in
 *     the reference (src/kernels/spmv.hpp:89-91), unless the kernel has the
 *     SMAX_FLAG_DEVICE_POINTERS flag, in which case B and C are device pointers.
 *     A CRS matrix may also be registered as device arrays: initialize copies
 *     it in the direction its addresses give.
 *   - Index type int32 and value types float32/float64 are supported; other
 *     combinations return SMAX_ERR_UNSUPPORTED_TYPE.
 *   - Streams are passed as void* (a cudaStream_t).
 */
#ifndef SMAX_B200_H
#define SMAX_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SMAX_B200_ABI_VERSION 1

typedef int smax_status;

/* status codes */
#define SMAX_OK 0
#define SMAX_ERR_BAD_ARG (-1)
#define SMAX_ERR_UNSUPPORTED_TYPE (-2)
#define SMAX_ERR_OOM (-3)
#define SMAX_ERR_ZERO_DIAG (-4)
#define SMAX_ERR_NO_DIAG (-5)
#define SMAX_ERR_TIMEOUT (-6)
#define SMAX_ERR_CUDA (-7)
#define SMAX_ERR_COL_OOB (-8)
#define SMAX_ERR_STATE (-9)
#define SMAX_ERR_UNSUPPORTED (-10)

/* kernel types, in the order of SMAX::KernelType (src/common.hpp:12) */
#define SMAX_KERNEL_SPMV 0
#define SMAX_KERNEL_SPMM 1
#define SMAX_KERNEL_SPGEMM 2
#define SMAX_KERNEL_SPTRSV 3
#define SMAX_KERNEL_SPTRSM 4

/* index / value types, in the order of SMAX::IntType / SMAX::FloatType
 * (src/common.hpp:25-28) */
#define SMAX_INT16 0
#define SMAX_INT32 1
#define SMAX_INT64 2
#define SMAX_UINT16 3
#define SMAX_UINT32 4
#define SMAX_UINT64 5
#define SMAX_FLOAT32 0
#define SMAX_FLOAT64 1

/* kernel flags: the reference's Kernel::set_* setters (src/kernel.hpp:58-90)
 * plus platform options */
#define SMAX_FLAG_MAT_PERM 0           /* set_mat_perm: level-scheduled solve */
#define SMAX_FLAG_MAT_UPPER_TRIANG 1   /* set_mat_upper_triang */
#define SMAX_FLAG_MAT_LOWER_TRIANG 2   /* set_mat_lower_triang */
#define SMAX_FLAG_VEC_ROW_MAJOR 3      /* set_vec_row_major */
#define SMAX_FLAG_MAT_SCS 4            /* set_mat_scs */
#define SMAX_FLAG_MAT_BCRS 5           /* set_mat_bcrs */
#define SMAX_FLAG_BLOCK_COLUMN_MAJOR 6 /* set_block_column_major */
#define SMAX_FLAG_KERNEL_IMPL 7        /* set_kernel_implementation(SpMVType) */
#define SMAX_FLAG_DEVICE_POINTERS 8    /* B and C registered as device pointers */
#define SMAX_FLAG_A_DIRTY 9            /* re-upload A at the next initialize */
#define SMAX_FLAG_SPMV_VARIANT 10      /* CRS SpMV kernel: 0 auto, 1 warp-stream, 2 row-tile; row-major SpMM:
                                          0 auto (= 1), 1 a grid of all rows, 2 one CTA per SM walking a row range */
#define SMAX_FLAG_SOLVE_MODE 11        /* SpTRSV/SpTRSM launch scheme, one of SMAX_SOLVE_* */
#define SMAX_FLAG_LEVEL_MERGE 12       /* levels with <= this many rows*rhs run merged in one CTA (0: never) */
#define SMAX_FLAG_SPIN_LIMIT 13        /* polls (x 1000) before a wait of the persistent or sync-free solve times out */
#define SMAX_FLAG_TEST_FORCE_TIMEOUT 14 /* test only: the persistent solve's barrier waits for a missing arrival */
#define SMAX_FLAG_REFINE 15            /* float64 SpTRSV: solve in FP32, then this many FP64-residual corrections (0: off) */
#define SMAX_FLAG_REFINE_TOL 16        /* stop refining once max|dx| <= 10^-value * max|x| (host check per step; 0: run all) */
#define SMAX_FLAG_SWEEP_CLUSTER 17     /* SpTRSV: runs with levels wider than 1024 rows on a thread-block cluster (0: one CTA) */
#define SMAX_FLAG_SPMV_PIPELINE 18     /* CRS SpMV with host pointers: B row blocks, block b with 2^b/(2^B-1) of the entries, whose y is downloaded while later blocks compute (default 6, at most 16 used; 0/1: off) */
#define SMAX_FLAG_TIMERS 19            /* 1 (default): time every apply with a pair of CUDA events (timer "apply", SpGEMM's phases); 0: no events, those timers stay 0.  A timing event between launches costs about 2.5 us of device time */

/* SpTRSV / SpTRSM launch schemes (SMAX_FLAG_SOLVE_MODE) */
#define SMAX_SOLVE_AUTO 0        /* the default: SMAX_SOLVE_SYNCFREE for one right-hand side and few wide
                                    levels (>= 2^17 rows, >= 32768 rows per level on average) and for
                                    SpTRSM over many narrow levels (>= 2^16 rows, >= 64 levels,
                                    <= 16384 rows per level on average), else SMAX_SOLVE_GRAPH */
#define SMAX_SOLVE_PER_LEVEL 1   /* one kernel launch per level, no merging, no graph */
#define SMAX_SOLVE_MERGED 2      /* narrow levels merged into single-CTA runs, no graph */
#define SMAX_SOLVE_GRAPH 3       /* the merged launch sequence captured into a CUDA graph */
#define SMAX_SOLVE_PERSISTENT 4  /* one cooperative launch, bounded grid barrier per level (SpTRSV, k = 1) */
#define SMAX_SOLVE_SYNCFREE 5    /* one launch, no level barriers: each row waits (bounded) on the rows it reads
                                    (SpTRSV and SpTRSM, both block layouts; falls back to SMAX_SOLVE_MERGED
                                    where it does not apply) */

typedef struct smax_ctx_s *smax_ctx;
typedef struct smax_kernel_s *smax_kernel;

/* ---------------------------------------------------------------- library */
int smax_abi_version(void);
const char *smax_last_error(void);

/* Allocation-failure injection for tests (no counterpart in the reference,
 * whose CUDA path only prints a failed allocation, src/platforms/cuda/
 * cuda.cuh:23-44).  Every device allocation of this library is counted; with
 * n >= 1 the n-th allocation from this call on fails as an out-of-memory
 * cudaMalloc would (the call in progress returns SMAX_ERR_OOM, cudaMalloc is
 * not called) and the injection disarms itself; n = 0 disarms.  Process-wide,
 * host-side only: no GPU is faulted. */
smax_status smax_test_fail_device_alloc(int64_t n);
/* Device allocations attempted since the library was loaded. */
uint64_t smax_test_device_alloc_count(void);

/* ---------------------------------------------------------------- context */
/* Interface-level state; kernels created from one context share its level
 * sets (src/interface.hpp:23-26, src/interface.cpp:53-57). */
smax_status smax_ctx_create(smax_ctx *out);
smax_status smax_ctx_destroy(smax_ctx ctx);
int smax_ctx_get_n_levels(smax_ctx ctx);             /* Interface::get_n_levels */
int smax_ctx_get_level_ptr_at(smax_ctx ctx, int idx); /* Interface::get_level_ptr_at */
/* Stores a level pointer computed elsewhere (e.g. by the reference's own CPU
 * Utils::generate_perm, which fills UtilitiesContainer::lvl_ptr,
 * src/utils/permutations.hpp:485-584): n_levels + 1 non-decreasing entries
 * starting at 0.  Level-scheduled solves read it as they read generate_perm's. */
smax_status smax_ctx_set_levels(smax_ctx ctx, int n_levels, const int *lvl_ptr);

/* ---------------------------------------------------------------- kernels */
/* Interface::register_kernel(name, KernelType, PlatformType::CUDA, IntType,
 * FloatType) (src/interface.cpp:59-123). */
smax_status smax_kernel_create(smax_kernel *out, smax_ctx ctx, int kernel_type, int int_type,
                               int float_type);
smax_status smax_kernel_destroy(smax_kernel k);
smax_status smax_kernel_set_flag(smax_kernel k, int flag, int value);

/* register_A for a CRS matrix, argument order of src/kernels/spmv.hpp:77-91
 * (also SpMM, SpGEMM A, SpTRSV and SpTRSM: spmm.hpp:24-38, spgemm.hpp:34-48,
 * sptrsv.hpp:23-37, sptrsm.hpp:23-37). */
smax_status smax_kernel_register_A_crs(smax_kernel k, uint64_t n_rows, uint64_t n_cols, uint64_t nnz,
                                       void *col, void *row_ptr, void *val);

/* register_A for a SELL-C-sigma matrix (with SMAX_FLAG_MAT_SCS), the 13
 * arguments of src/kernels/spmv.hpp:25-53: C, sigma, n_rows, n_rows_padded,
 * n_cols, n_chunks, n_elements, nnz, chunk_ptr, chunk_lengths, col, val, perm.
 * y is produced in the permuted row order, of length n_rows_padded. */
smax_status smax_kernel_register_A_scs(smax_kernel k, uint64_t C, uint64_t sigma, uint64_t n_rows,
                                       uint64_t n_rows_padded, uint64_t n_cols, uint64_t n_chunks,
                                       uint64_t n_elements, uint64_t nnz, void *chunk_ptr, void *chunk_lengths,
                                       void *col, void *val, void *perm);

/* register_A for a BCRS matrix (with SMAX_FLAG_MAT_BCRS), the 10 arguments of
 * src/kernels/spmv.hpp:54-76: block rows, block columns, blocks, block height
 * and width, height and width padding, col, row_ptr, val.  The in-block order
 * follows SMAX_FLAG_BLOCK_COLUMN_MAJOR. */
smax_status smax_kernel_register_A_bcrs(smax_kernel k, uint64_t n_rows, uint64_t n_cols, uint64_t n_blocks,
                                        uint64_t b_height, uint64_t b_width, uint64_t height_pad,
                                        uint64_t width_pad, void *col, void *row_ptr, void *val);

/* SpGEMM: register_B of the CRS matrix B (src/kernels/spgemm.hpp:51-66) and
 * register_C of the output references (src/kernels/spgemm.hpp:68-83): after
 * finalize, *n_rows/*n_cols/*nnz hold C's sizes and *col/*row_ptr/*val point
 * to new[]-allocated arrays owned by the caller (int32 indices, values of the
 * kernel's float type), columns of each row in first-touch order. */
smax_status smax_kernel_register_B_crs(smax_kernel k, uint64_t n_rows, uint64_t n_cols, uint64_t nnz, void *col,
                                       void *row_ptr, void *val);
smax_status smax_kernel_register_C_crs_ref(smax_kernel k, uint64_t *n_rows, uint64_t *n_cols, uint64_t *nnz,
                                           void **col, void **row_ptr, void **val);

/* register_B / register_C of a dense operand: (n_rows, val) for vectors
 * (spmv.hpp:97-115, sptrsv.hpp:40-58) or (n_rows, n_cols, val) for blocks of
 * vectors (spmm.hpp:40-61, sptrsm.hpp:40-60).  slot 1 = B, slot 2 = C. */
smax_status smax_kernel_register_dense(smax_kernel k, int slot, uint64_t n_rows, uint64_t n_cols, void *val);

/* Kernel::initialize / apply / finalize / run with the reference's offset
 * arguments (src/kernel.hpp:48-52,99-111).  On this platform initialize
 * uploads A (only when registered anew or marked dirty) and B, apply launches
 * the kernel asynchronously on the kernel's stream, finalize downloads C and
 * synchronises. */
smax_status smax_kernel_initialize(smax_kernel k, uint64_t A_offset, uint64_t B_offset, uint64_t C_offset);
smax_status smax_kernel_apply(smax_kernel k, uint64_t A_offset, uint64_t B_offset, uint64_t C_offset);
smax_status smax_kernel_finalize(smax_kernel k, uint64_t A_offset, uint64_t B_offset, uint64_t C_offset);
smax_status smax_kernel_run(smax_kernel k, uint64_t A_offset, uint64_t B_offset, uint64_t C_offset);

/* Waits for the kernel's stream and reports any device-side error. */
smax_status smax_kernel_sync(smax_kernel k);

/* Accumulated seconds of a stopwatch ("initialize", "apply", "finalize", ...;
 * src/kernel.hpp:36-43).  "apply" is measured with CUDA events on the
 * kernel's stream. */
smax_status smax_kernel_get_timer(smax_kernel k, const char *name, double *seconds);

/* The kernel's CUDA stream (a cudaStream_t). */
void *smax_kernel_stream(smax_kernel k);

/* Kernel::swap_operands (src/kernels/spmv.hpp:197-200, spmm.hpp:102-105):
 * B and C exchange roles (x <-> y), for iterations that feed an SpMV's output
 * back as its input.  The device copies are exchanged too, so an
 * apply-swap-apply loop reads the previous result without any copy. */
smax_status smax_kernel_swap_operands(smax_kernel k);

/* Runs the kernel's work on the caller's stream (a cudaStream_t, e.g. the
 * current stream of a framework) instead of its own; NULL restores its own.
 * The caller keeps ownership of the stream. */
smax_status smax_kernel_set_stream(smax_kernel k, void *stream);

/* ------------------------------------------------- reverse-mode derivatives */
/* Adjoint of an initialized kernel (no counterpart in the reference), for a
 * loss gradient g:
 *   SpMV (CRS, y = A x):  d_in = A^T g (n_cols values),
 *                         d_val[k] = g[row(k)] * x[col(k)]   (nnz values)
 *   SpTRSV (L x = b):     L^T lambda = g;  d_in = lambda = dLoss/db (n values),
 *                         d_val[k] = -lambda[row(k)] * x[col(k)]
 * d_val follows the entry order of the device copy of A: the registered order
 * for SpMV; for SpTRSV the order after initialize moved each diagonal to the
 * end of its row (the order the caller's arrays then hold).  x is the SpMV
 * input or the SpTRSV solution; NULL means the registered B.  g, x, d_in and
 * d_val are device pointers when SMAX_FLAG_DEVICE_POINTERS is set, host
 * pointers otherwise (the call then returns when the outputs are written).
 * d_in or d_val may be NULL to skip that output.  A^T (L^T) is built on the
 * first call and kept with the kernel. */
smax_status smax_kernel_adjoint(smax_kernel k, const void *x, const void *g, void *d_in, void *d_val);

/* Replaces the values of the device copy of a CRS A (SpMV, SpMM, SpTRSV,
 * SpTRSM) in place, keeping the pattern and every plan; val holds nnz values
 * in the entry order described for d_val above.  For solves the diagonal is
 * re-read and checked (ZERO_DIAG).  Host or device pointer as above. */
smax_status smax_kernel_update_A_values(smax_kernel k, const void *val);

/* Refinement statistics of the last solve with SMAX_FLAG_REFINE: corrections
 * applied and max|dx| / max|x| of the last one. */
smax_status smax_kernel_get_refine_stats(smax_kernel k, int *steps, double *last_rel_correction);

/* --------------------------------------------------------------- autotuning */
/* Times the launch variants of an initialized kernel on its registered
 * operands and keeps the fastest: the CRS SpMV kernel for SpMV; the solve
 * mode, the level-merge threshold and (SpTRSV) cluster runs for SpTRSV /
 * SpTRSM.  Choices are cached
 * for the life of the process per matrix (kernel type, value type, sizes and
 * a hash of the pattern); a later kernel with the same matrix takes them from
 * the cache.  Overwrites the output operand (C for SpMV, B for solves). */
typedef struct smax_tuning {
    int spmv_variant; /* SMAX_FLAG_SPMV_VARIANT chosen (SpMV, row-major SpMM) */
    int solve_mode;   /* SMAX_SOLVE_* chosen (SpTRSV / SpTRSM) */
    int level_merge;  /* SMAX_FLAG_LEVEL_MERGE chosen (SpTRSV / SpTRSM) */
    int sweep_cluster; /* SMAX_FLAG_SWEEP_CLUSTER chosen (SpTRSV) */
    int from_cache;   /* 1: taken from the process-wide cache */
    int n_candidates; /* configurations timed (0 from the cache) */
    double seconds;   /* one apply with the choice */
} smax_tuning;
smax_status smax_kernel_autotune(smax_kernel k, smax_tuning *out);

/* Chooses the storage format of a CRS matrix for SpMV by converting it on the
 * GPU and timing each candidate: CRS (both kernels), SELL-C-sigma with
 * C in {8, 16, 32, 64} and sigma in {1, C*8, 1024}, and BCRS with square
 * blocks of 2 and 4 where the dimensions divide and the fill stays below
 * twice the nonzeros.  Host arrays. */
typedef struct smax_format_choice {
    int format;             /* 0 CRS, 1 SELL-C-sigma, 2 BCRS */
    int spmv_variant;       /* CRS kernel (format 0) */
    int C, sigma;           /* SELL-C-sigma parameters (format 1) */
    int b_height, b_width;  /* BCRS block (format 2) */
    int n_candidates;       /* configurations timed */
    double seconds;         /* one SpMV with the choice */
    double crs_seconds;     /* one SpMV with the best CRS kernel */
} smax_format_choice;
smax_status smax_utils_tune_spmv_format(int float_type, uint64_t n_rows, uint64_t n_cols, uint64_t nnz,
                                        const void *row_ptr, const void *col, const void *val,
                                        smax_format_choice *out);

/* -------------------------------------------------------- batched SpTRSV */
/* A batch of independent lower-triangular CRS matrices (host arrays, each with
 * its diagonal; no counterpart in the reference, which solves one matrix per
 * kernel) solved together: one persistent kernel whose CTAs take matrices from
 * a device work queue (longest critical path first) and sweep each matrix's
 * dependency levels with the CTA barrier as the level barrier.  The batch owns
 * device copies; the caller's arrays are not modified. */
typedef struct smax_batch_s *smax_batch;
smax_status smax_batch_sptrsv_create(smax_batch *out, int float_type, int n_mats, const uint64_t *n_rows,
                                     const uint64_t *nnz, void *const *row_ptr, void *const *col, void *const *val);
/* rhs and x are DEVICE arrays of the packed rows (matrix m at row offset
 * smax_batch_row_offset(b, m)); mode: SMAX_SOLVE_GRAPH (persistent kernel
 * replayed from a CUDA graph), SMAX_SOLVE_MERGED (persistent kernel, direct
 * launch) or SMAX_SOLVE_PER_LEVEL (one launch per level of every matrix, the
 * plain baseline).  stream: a cudaStream_t (NULL = legacy default stream). */
smax_status smax_batch_sptrsv_solve(smax_batch b, const void *rhs, void *x, int mode, void *stream);
uint64_t smax_batch_row_offset(smax_batch b, int m);
/* total packed rows, sum of the matrices' level counts, largest level count */
smax_status smax_batch_info(smax_batch b, uint64_t *n_rows, int *total_levels, int *max_levels);
smax_status smax_batch_destroy(smax_batch b);

/* ------------------------------------------------------------------ utils */
/* Utils::convert_crs_to_scs (src/utils/convert_formats.hpp:16-132), computed on
 * the GPU.  meta[6] receives n_rows, n_rows_padded, n_cols, n_chunks,
 * n_elements, nnz; the five arrays are allocated with new[] (release with
 * delete[] or smax_free_host).  Rows of equal length inside a sigma window are
 * ordered by ascending row index. */
smax_status smax_utils_convert_crs_to_scs(int int_type, int float_type, uint64_t n_rows, uint64_t n_cols,
                                          uint64_t nnz, const void *col, const void *row_ptr, const void *val,
                                          uint64_t C, uint64_t sigma, uint64_t *meta, void **chunk_ptr,
                                          void **chunk_lengths, void **col_out, void **val_out, void **perm);

/* Utils::convert_crs_to_bcrs (src/utils/convert_formats.hpp:134-247), computed
 * on the GPU.  meta[7] receives n_rows, n_cols, n_blocks, b_height, b_width,
 * height_pad, width_pad (in blocks); arrays as above. */
smax_status smax_utils_convert_crs_to_bcrs(int int_type, int float_type, uint64_t n_rows, uint64_t n_cols,
                                           uint64_t nnz, const void *col, const void *row_ptr, const void *val,
                                           uint64_t b_height, uint64_t b_width, uint64_t height_pad,
                                           uint64_t width_pad, int block_column_major, uint64_t *meta,
                                           void **col_out, void **row_ptr_out, void **val_out);

/* Utils::build_symmetric_crs (src/utils/permutations.hpp:236-392): the
 * pattern of A + A^T; row c is A's row c followed by the missing transposes in
 * ascending row order.  Arrays allocated with new[]. */
smax_status smax_utils_build_symmetric_crs(int int_type, uint64_t n_rows, const void *row_ptr, const void *col,
                                           void **sym_row_ptr, void **sym_col, uint64_t *sym_nnz);

/* Utils::generate_perm (src/utils/permutations.hpp:485-584) for every type
 * of the reference, computed on the GPU: "BFS" (the default; queue order of
 * its one-thread BFS), "RS" (rows stably sorted by level), the colourings
 * "SC", "PC" and "PC_BAL" (rows stably sorted by colour, one level per
 * colour; the results the reference gives with one OpenMP thread, whose
 * colourings otherwise depend on thread timing) and "NONE".  perm and
 * inv_perm are caller arrays of n_rows ints; the level pointer is stored in
 * ctx (smax_ctx_get_n_levels / smax_ctx_get_level_ptr_at). */
smax_status smax_utils_generate_perm(smax_ctx ctx, int int_type, uint64_t n_rows, const void *row_ptr,
                                     const void *col, int *perm, int *inv_perm, const char *type);

/* Utils::sanity_check_perm (src/utils/permutations.hpp:794-818): *valid = 1
 * when no row shares a colour other than 0 with a lower neighbour of the CRS
 * pattern (colors: n_rows ints, host); else 0 and *first_bad_row (may be
 * NULL) = the lowest such row. */
smax_status smax_utils_sanity_check_perm(int int_type, uint64_t n_rows, const void *row_ptr, const void *col,
                                         const int *colors, int *valid, int64_t *first_bad_row);

/* Utils::apply_mat_perm (src/utils/permutations.hpp:820-861): row r of the
 * result is row perm[r], columns mapped through inv_perm; output arrays are the
 * caller's (n_rows+1, nnz, nnz). */
smax_status smax_utils_apply_mat_perm(int int_type, int float_type, uint64_t n_rows, const void *row_ptr,
                                      const void *col, const void *val, void *perm_row_ptr, void *perm_col,
                                      void *perm_val, const int *perm, const int *inv_perm);

/* Utils::apply_vec_perm (src/utils/permutations.hpp:863-874):
 * vec_perm[i] = vec[perm[i]]. */
smax_status smax_utils_apply_vec_perm(int float_type, uint64_t n_rows, const void *vec, void *vec_perm,
                                      const int *perm);

/* Matrix Market ingestion, as the reference's examples read matrices
 * (COOMatrix::read_from_mtx without fast_matrix_market and
 * CRSMatrix::convert_coo_to_crs, examples/matrix_structs.hpp:52-180, 338-387;
 * examples/mmio.cpp): a coordinate file with real, integer or pattern values
 * (pattern entries get 0.01) and general or symmetric storage (every
 * off-diagonal entry of a symmetric file is followed by its mirror); entries
 * stably sorted by row only, so each row keeps the file's order.  The text is
 * parsed on the host (threads over line-aligned slices), the sort and the row
 * pointer run on the GPU.  Outputs are new[] arrays (int32 row_ptr and col,
 * values of float_type).  SMAX_ERR_UNSUPPORTED for other formats, BAD_ARG
 * for malformed text, COL_OOB / BAD_ARG for indices outside the size line's
 * dimensions. */
smax_status smax_utils_read_mtx(const char *path, int float_type, uint64_t *n_rows, uint64_t *n_cols, uint64_t *nnz,
                                void **row_ptr, void **col, void **val);
/* COO (0-based int32 I, J; double values; host or device arrays) to CRS with
 * the same stable by-row order (convert_coo_to_crs after sort_perm). */
smax_status smax_utils_convert_coo_to_crs(int float_type, uint64_t n_rows, uint64_t n_cols, uint64_t nnz,
                                          const int *I, const int *J, const double *val, void **row_ptr,
                                          void **col, void **val_out);

/* Releases an array returned by an smax_utils_* function. */
void smax_free_host(void *p);

/* ------------------------------------------------- allocation-free SpMV */
/* CRS SpMV y = A*x for callers that cannot allocate device memory (an
 * application whose pool already owns the GPU, a plugin whose host forbids
 * device allocations, a loop that must not enter the allocator).  No
 * counterpart exists in the reference.  All arrays are the caller's DEVICE
 * arrays (int32 row_ptr/col, float32 or float64 val/x/y); the call allocates
 * nothing and keeps its working data in one fixed scratch area of
 * SMAX_NOALLOC_SCRATCH_BYTES per GPU, held from library load until exit.
 * Limits: n_rows <= SMAX_NOALLOC_MAX_ROWS and nnz <= SMAX_NOALLOC_MAX_NNZ, else
 * SMAX_ERR_BAD_ARG.  Calls share the scratch area: calls that overlap on the
 * GPU race, so issue them on one stream or serialise them.  The first call on
 * a device does the set-up (it looks up the scratch address); make it before
 * any stream capture.
 * The call validates the matrix (SMAX_ERR_COL_OOB / SMAX_ERR_BAD_ARG) and
 * synchronises `stream` (a cudaStream_t; NULL = legacy default stream). */
#define SMAX_NOALLOC_MAX_ROWS (1 << 20)
#define SMAX_NOALLOC_MAX_NNZ (1 << 24)
#define SMAX_NOALLOC_SCRATCH_BYTES (7u << 20)
smax_status smax_spmv_crs_noalloc(int float_type, uint64_t n_rows, uint64_t n_cols, uint64_t nnz,
                                  const void *d_row_ptr, const void *d_col, const void *d_val, const void *d_x,
                                  void *d_y, void *stream);

/* ---------------------------------------------------------- solver callers */
/* The iterative solvers of the reference's applications on device-resident
 * operators.  The reference runs them as programs that call run() on SpMV and
 * SpTRSV kernels once per iteration and do the vector arithmetic on the host:
 *   Jacobi        examples/applications/jacobi/jacobi.cpp:14-130 with
 *                 jacobi/utils.hpp:7-50 (diagonal moved to the end of each
 *                 row; x_new = (b - (A x_old - D x_old)) / D)
 *   Gauss-Seidel  examples/applications/gauss_seidel/gauss_seidel.cpp:13-111
 *                 on the D+L / U split of examples/examples_common.hpp:283-398
 *                 (x = (D+L)^-1 (b - U x))
 * Both run the applications' loop:
 *   residual = max_i |b_i - (A x)_i|
 *   while (residual > tol && n_iters < max_iters) {
 *       one iteration; ++n_iters;
 *       if (n_iters % check_length == 0) residual = max_i |b_i - (A x)_i|;
 *   }
 * NaN entries never become the maximum (applications_common.hpp:122-133).
 * Jacobi keeps the application's two iterate buffers, swapped after every
 * iteration; its residual kernel stays bound to the first x_new buffer
 * (jacobi.cpp:14-24, 96-100), so the residual after an odd iteration count is
 * that of the latest iterate and after an even count that of the one before.
 *
 * create copies the square CRS matrix (int32 indices, host or device arrays)
 * to the device and validates it: Jacobi needs a diagonal entry with
 * |a_ii| >= 1e-16 in every row (SMAX_ERR_NO_DIAG / SMAX_ERR_ZERO_DIAG), as
 * utils.hpp:7-36 does; Gauss-Seidel's D+L part is solved by this platform's
 * level-scheduled SpTRSV, with the same diagonal checks.  The solver owns its
 * vectors; solve copies b and x in (host or device arrays, n_rows values of
 * the solver's type), runs the loop on `stream` (a cudaStream_t; NULL = the
 * solver's own stream) and copies the solution back into x before it returns.
 * Drivers (smax_solver_opts.mode), all with the same kernel launches:
 *   SMAX_SOLVER_DEVICE_LOOP   one CUDA graph: a conditional while node repeats
 *                             check_length iterations and the residual until a
 *                             device kernel ends the loop; the host waits once
 *   SMAX_SOLVER_GRAPH_BLOCKS  one graph launch per check_length iterations and
 *                             residual; the host reads each residual
 *   SMAX_SOLVER_PLAIN         the same launches one by one, no graphs
 * Systems of at most 4096 rows run the whole loop in one launch of one CTA
 * (x, b and D in shared memory) whatever the driver. */
typedef struct smax_solver_s *smax_solver;
#define SMAX_SOLVER_JACOBI 0
#define SMAX_SOLVER_GAUSS_SEIDEL 1
#define SMAX_SOLVER_DEVICE_LOOP 0
#define SMAX_SOLVER_GRAPH_BLOCKS 1
#define SMAX_SOLVER_PLAIN 2

typedef struct {
    double tol;       /* the loop runs while residual > tol (the applications' TOL: 1e-8) */
    int max_iters;    /* MAX_ITERS: 1000 */
    int check_length; /* CHECK_LENGTH: 5 (>= 1) */
    int mode;         /* SMAX_SOLVER_* driver */
} smax_solver_opts;

typedef struct {
    int n_iters;          /* iterations run */
    int converged;        /* residual_norm < tol, the applications' test */
    double residual_norm; /* the last residual measured */
    int n_checks;         /* residuals measured, the one before the loop included */
    int host_waits;       /* times the host waited for the device inside the loop */
} smax_solver_stats;

smax_status smax_solver_create(smax_solver *out, int kind, int float_type, uint64_t n_rows, uint64_t nnz,
                               const void *row_ptr, const void *col, const void *val);
smax_status smax_solver_solve(smax_solver s, const void *b, void *x, const smax_solver_opts *opts,
                              smax_solver_stats *stats, void *stream);
/* The residuals of the last solve in the order they were measured (the first
 * 2^20 of them): writes min(cap, n_checks, 2^20) values to out (host array)
 * and n_checks to *count. */
smax_status smax_solver_get_history(smax_solver s, double *out, int cap, int *count);
smax_status smax_solver_destroy(smax_solver s);

/* ------------------------------------------------------------ measurement */
/* The memory-traffic floor of the warp-stream CRS SpMV on given arrays: the
 * same 512-entry warp slices and 16-byte streaming loads of col and val, one
 * x gather per entry, products summed per slice into out[] (no row
 * bookkeeping).  No counterpart exists in the reference; the benchmark uses
 * it to measure the gather ceiling the SpMV kernels are judged against.
 *   mode 0: gathers -- lanes [0, tma_lanes) of every warp fetch x through TMA
 *           tile::gather4 loads, the others through ordinary L2 loads;
 *   mode 1: stream only (x is not read).
 * depth (1, 2 or 4) chunks of 128 entries are kept in flight per warp.
 * d_col/d_val: n_slices*512 entries (16-byte aligned, columns in
 * [0, n_cols)); d_out: n_slices values; d_err: one int, set to 1 when a TMA
 * wait gave up (never expected).  Asynchronous on `stream`. */
smax_status smax_measure_gather(int float_type, int mode, int tma_lanes, int depth, uint64_t n_slices,
                                const void *d_col, const void *d_val, const void *d_x, uint64_t n_cols, void *d_out,
                                void *d_err, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* SMAX_B200_H */
