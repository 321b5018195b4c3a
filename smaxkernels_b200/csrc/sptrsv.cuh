// sptrsv.cuh -- level-scheduled triangular solves (sptrsv.cu).
#pragma once

#include <vector>

#include "levelpack.cuh"
#include "levels.cuh"
#include "spmv_formats.cuh"

namespace smax {

// Copies the diagonal into D and swaps it to the last slot of each row (in
// place on the device copy); missing / |d| < 1e-16 diagonals are reported.
void peel_diag(DevCRS &a, int vbytes, DevBuf &D, DevStatus *st, cudaStream_t s);
// Re-reads D from a matrix whose diagonals already sit last in their rows
// (after a value update); a row whose last entry is not its diagonal reports
// NO_DIAG, |d| < 1e-16 ZERO_DIAG.
void refresh_diag(const DevCRS &a, int vbytes, DevBuf &D, DevStatus *st, cudaStream_t s);

// The level schedule of one triangular matrix and its launch plan.
struct TriPlan {
    int64_t n_rows = 0;
    std::vector<int> lvl_ptr;  // host copy, n_levels + 1 entries
    DevBuf order;              // rows sorted by level (own levels) or unused
    bool has_order = false;
    bool descending = false;   // sweep levels last to first

    // launch plan: steps of single wide levels (kind 0) or merged runs (kind 1)
    struct Step {
        int kind = 0;
        int row0 = 0, m = 0;
        int seg_first = 0, seg_count = 0;
        int sweep_first = 0, sweep_count = 0;  // levels of the step, in sweep order
    };
    std::vector<Step> steps;
    std::vector<int2> seg_ranges;
    DevBuf d_ranges;
    bool ranges_uploaded = false;
    int64_t scheduled_k = -1;
    int scheduled_merge = -1;

    // CUDA graph of the launch sequence (bound to the operand addresses)
    cudaGraphExec_t graph = nullptr;
    bool graph_valid = false;
    const void *graph_key[4] = {nullptr, nullptr, nullptr, nullptr};
    bool graph_row_major = false;
    int64_t graph_ld = 0;
    AuxStream aux;  // capture stream when the caller's stream cannot be captured

    // level-ordered pack for one right-hand side (levelpack.cu), built for the
    // value arrays, their version tag and the merge threshold below
    LevelPack pack;
    std::vector<PackStep> pack_steps;
    bool pack_ok = false, pack_unfit = false;
    bool allow_cluster = false;  // runs wider than one CTA covers may use a cluster
    // sets allow_cluster; a change drops the pack and the graph
    void set_allow_cluster(bool v) {
        if (v != allow_cluster) {
            allow_cluster = v;
            pack_ok = false;
            release_graph();
        }
    }
    const void *pack_key[2] = {nullptr, nullptr};
    uint64_t pack_tag = ~0ull;
    int pack_merge = -1, pack_vbytes = 0;
    // (re)builds the pack when its key changed; false when the matrix does
    // not pack compactly and the plain kernels must be used.  Synchronises:
    // call outside stream capture.
    bool ensure_pack(const int *rp, const int *ci, const void *val, const void *D, int vbytes, int merge_rows,
                     uint64_t tag, cudaStream_t st);

    // sync-free form of the pack (SMAX_SOLVE_SYNCFREE): every level its own
    // step, entries naming source rows; unfit when padding is too large or an
    // entry reads a row that is not solved before it
    LevelPack sf_pack;
    bool sf_ok = false, sf_unfit = false;
    const void *sf_key[2] = {nullptr, nullptr};
    uint64_t sf_tag = ~0ull;
    int sf_vbytes = 0;
    bool ensure_syncfree(const int *rp, const int *ci, const void *val, const void *D, int vbytes, uint64_t tag,
                         cudaStream_t st);

    // dependency levels of the matrix itself (plain solve)
    void build_own(const DevCRS &a, bool upper, cudaStream_t st);
    // caller-given contiguous levels (permuted, level-scheduled solve)
    void build_given(const std::vector<int> &lvl_ptr, int64_t n, bool upper, cudaStream_t st);
    // the same level sets swept in the opposite direction (the schedule of
    // the transposed solve)
    void assign_reverse(const TriPlan &src, cudaStream_t st);
    void finish(cudaStream_t st);
    void schedule(int64_t k, int merge_rows);
    // schedules and uploads the merged-run ranges ahead of a stream capture
    void prepare(int64_t k, int merge_rows, cudaStream_t st);
    void release_graph();
    int n_levels() const { return lvl_ptr.empty() ? 0 : (int)lvl_ptr.size() - 1; }
    ~TriPlan();
};

// X = A^{-1} B for k right-hand sides (row-major: element (r, v) at r*k+v;
// column-major: at r + v*ld).  merge_rows: levels with at most this many
// (row, vector) pairs are merged into single-CTA runs (0 disables merging).
// `tag` identifies the current values of (val, D): a caller that changes the
// values in place passes a new tag so the level-ordered pack is rebuilt.
// With k == 1 the solve runs on the pack (levelpack.cu); tri_solve_raw does
// not build it (it may run inside a stream capture): call ensure_pack first.
template <typename VT>
void tri_solve(TriPlan &p, const DevCRS &a, const VT *D, const VT *B, VT *X, int64_t k, bool row_major, int64_t ld,
               int merge_rows, uint64_t tag, cudaStream_t st);
// tri_solve on raw arrays (rp/ci of the matrix the plan was built for, with
// any values of type VT, e.g. a float copy of double values).
template <typename VT>
void tri_solve_raw(TriPlan &p, const int *rp, const int *ci, const VT *val, const VT *D, const VT *B, VT *X,
                   int64_t k, bool row_major, int64_t ld, int merge_rows, uint64_t tag, cudaStream_t st);
// The sync-free solve of one right-hand side (pack_solve_syncfree).  Returns
// false, launching nothing, when it does not apply: the matrix does not pack,
// an entry reads a row not solved before it, or B and X overlap.
// Whether the default scheme (SMAX_SOLVE_AUTO) runs sync-free.  One
// right-hand side: at least 2^17 rows in levels of 32768 rows or more on
// average (few wide levels, whose launches the sync-free solve saves).  k > 1:
// at least 2^16 rows in 64 levels or more of at most 16384 rows on average
// (many narrow levels, launch-bound as level launches).
bool syncfree_suits(const TriPlan &p, int64_t k = 1);
// k > 1 runs the row kernel (solve_syncfree_rows), in either block layout.
template <typename VT>
bool tri_solve_syncfree(TriPlan &p, const DevCRS &a, const VT *D, const VT *B, VT *X, uint64_t tag, DevBuf &ctl,
                        long long limit, bool force_timeout, DevStatus *st, cudaStream_t s, int64_t k = 1,
                        bool row_major = true);
// The same launch sequence, captured once into a CUDA graph and replayed.
template <typename VT>
void tri_solve_graph(TriPlan &p, const DevCRS &a, const VT *D, const VT *B, VT *X, int64_t k, bool row_major,
                     int64_t ld, int merge_rows, uint64_t tag, cudaStream_t st);

}  // namespace smax
