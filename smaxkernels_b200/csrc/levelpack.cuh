// levelpack.cuh -- level-ordered packed triangular matrices and the sweep
// kernels over them (levelpack.cu).
#pragma once

#include <vector>

#include "common.cuh"

namespace smax {

// Rows in sweep order ("positions"), each level stored as a dense
// column-major block of its rows' off-diagonal entries (ELL per level): the
// i-th entry of the t-th row of level s sits at ent_base[s] + i*m[s] + t, so a
// warp reads its rows' i-th entries with one coalesced load.  Each entry's
// source is encoded for the single-CTA sweep:
//   src <  0, != kPad : the solution is in slot (-src-1) % kRing of the
//                       shared-memory ring of CTA (-src-1) / kRing of the run's
//                       cluster (0 for single-CTA runs); it was written by the
//                       same run at most kRing positions ago and is not
//                       overwritten by the current level
//   src >= 0          : the solution's position in the position-ordered x
//   src == kPad       : padding (the row has fewer entries than the level width)
struct LevelPack {
    static constexpr int kPad = -0x7fffffff - 1;
    static constexpr int kRing = 8192;  // shared-memory ring of recent solutions (positions; a power of 2)

    struct Level {
        int pos, m, w;      // first position, rows, width (max off-diagonals)
        int base;           // first entry (packs are limited to 2^31 entries)
    };
    int64_t n = 0, ents = 0;
    int vbytes = 8;
    std::vector<Level> h_lv;
    // launch geometry of the run each step belongs to: x = CTAs in the cluster
    // (1: a single CTA), y = threads per CTA; ring entries name the CTA that
    // owns the solution when x > 1
    std::vector<int2> h_geo;
    DevBuf lv;      // Level[n_levels]
    DevBuf prow;    // int[n]: row of each position
    DevBuf psrc;    // int[ents]
    DevBuf pval;    // VT[ents]
    DevBuf pinv;    // VT[n]: 1 / diagonal
    DevBuf bp, xp;  // VT[n]: right-hand side and solution in position order
    bool needs_x_init = false;  // some entry reads a solution not computed before it
    // sync-free packs (row_sources): entries name the source ROW in the
    // caller's numbering, never a ring slot, and `tasks` lists the warp tasks
    // in sweep order, up to 32 rows of one level each, so a warp's rows never
    // depend on one another
    bool row_sources = false;
    DevBuf tasks;  // int4[n_tasks]: first position, rows | width << 6, level rows, first entry
    int n_tasks = 0;
    int n_levels() const { return (int)h_lv.size(); }
};

// Builds the pack of a triangular CRS matrix (diagonal last in each row, D its
// diagonal) for a sweep whose step s solves the rows order[src_begin[s] ..
// src_begin[s] + count[s]) (order == nullptr: the identity).  seg_begin[s] is
// the first sweep step of the single-CTA run step s belongs to (s itself for
// a level solved by its own grid launch): only solutions produced inside the
// same run may come from the ring.
// Returns false (building nothing) when the per-level padding would make the
// pack more than about three times the off-diagonal entries.  allow_cluster:
// runs with levels wider than one CTA covers may be solved by a thread-block
// cluster (single matrices; the batch kernel is one CTA per matrix).
// row_sources: build the sync-free form (every step its own level, entries
// naming source rows, the task table).
bool build_level_pack(LevelPack &pk, const int *rp, const int *ci, const void *val, const void *D, int vbytes,
                      int64_t n, const int *order, const std::vector<int> &src_begin, const std::vector<int> &count,
                      const std::vector<int> &seg_begin, bool allow_cluster, cudaStream_t st,
                      bool row_sources = false);

// Solves with the pack: gathers B into position order, runs each step --
// wide levels as one grid launch each, runs of narrow levels as one
// single-CTA sweep -- and scatters the solution to X.  steps: (first sweep
// step, number of steps, kind 0 wide / 1 run).
struct PackStep {
    int first, count, kind;
};
template <typename VT>
void pack_solve(const LevelPack &pk, const std::vector<PackStep> &steps, const VT *B, VT *X, cudaStream_t st);

// Sync-free solve on a row_sources pack: X is first filled with a pending
// marker (a signalling-NaN pattern that no arithmetic result has), then one
// launch of warps takes 32-row tasks in sweep order (a CTA claims a chunk of
// tasks with one atomic) and each row waits on its sources' values in X,
// with no barrier between levels.  A row's sources lie in earlier tasks, which
// were claimed by running CTAs, so the earliest unfinished task can always
// finish.  Each wait gives up after `limit` polls: SMAX_ERR_TIMEOUT in st, an
// abort flag that ends the other waits, and NaN for the missing value.
// B and X must not overlap.  ctl: device scratch of at least 64 bytes.
// force_timeout (test only): the first row also waits on a word nothing writes.
template <typename VT>
void pack_solve_syncfree(const LevelPack &pk, const VT *B, VT *X, void *ctl, long long limit, bool force_timeout,
                         DevStatus *st, cudaStream_t s);

// The sync-free solve for k > 1 right-hand sides, on the matrix's own CRS
// arrays (diagonal last in each row) with the rows in the sweep order of a
// row_sources pack: a warp per row, lanes over vectors, bounded waits as
// above.  Blocks are row-major (r*k + v) or column-major (r + v*n, the
// matrix's row count as the leading dimension).  B and X (n * k values each)
// must not overlap.
template <typename VT>
void solve_syncfree_rows(const LevelPack &pk, const int *rp, const int *ci, const VT *val, const VT *D, const VT *B,
                         VT *X, int64_t k, bool row_major, void *ctl, long long limit, DevStatus *st, cudaStream_t s);

// One single-CTA sweep per matrix of a batch, matrices taken from a device
// work queue: mat_steps[m] .. mat_steps[m+1] are matrix m's sweep steps.
template <typename VT>
void pack_solve_batch(const LevelPack &pk, const int *mat_steps, const int *queue_order, int n_mats, int *queue,
                      const VT *B, VT *X, cudaStream_t st);

}  // namespace smax
