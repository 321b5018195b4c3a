// sptrsv.cu -- level-scheduled SpTRSV / SpTRSM on sm_100a.
//
// Reference semantics:
//   * peel_diag_crs (src/kernels/sptrsv/sptrsv_cpu/sptrsv_cpu_crs_helpers_impl.hpp:9-38):
//     D[r] = A[r][r] (the last diagonal entry of the row), swapped to the last
//     slot of its row; |D| < 1e-16 or a missing diagonal is an error.
//   * naive_crs_sptrsv / crs_sptrsv_lvl (sptrsv_cpu_crs_impl.hpp:9-55,
//     sptrsv_lvl_cpu_crs_impl.hpp:11-82) and the SpTRSM loops
//     (src/kernels/sptrsm/sptrsm_cpu/sptrsm_cpu_crs_impl.hpp:9-102):
//     x[r] = (b[r] - sum_{j < end-1} val[j] x[col[j]]) / D[r].
//
// Schedule.  A solve is a sequence of levels; the rows of one level are
// independent.  With the permuted (level-scheduled) flag the levels are the
// caller's contiguous row ranges (generate_perm's lvl_ptr), swept ascending for
// lower and descending for upper triangles, as the reference does.  Without
// it the platform computes the dependency levels of the matrix itself
// (levels.cu: RS levels of A+A^T, reversed for upper triangles) and keeps a
// row order, so the plain solve runs level-parallel with the reference's
// per-row arithmetic and summation order.
//
// Kernels.  One thread per (row, right-hand side) sums its row sequentially.
//   * wide level: one grid launch per level;
//   * run of narrow levels (<= merge threshold rows * k each): one CTA sweeps
//     the whole run, with __syncthreads() as the level barrier (global writes
//     of the CTA are visible to the CTA after the barrier);
// The launch sequence of a solve can be captured once into a CUDA graph and
// replayed (tri_solve_graph).
#include "sptrsv.cuh"

#include <algorithm>

namespace smax {

namespace {

constexpr int kSegThreads = 1024;

// ------------------------------------------------------------ peel diag ----
template <typename VT>
__global__ void peel_diag_kernel(const int *__restrict__ rp, int *__restrict__ col, VT *__restrict__ val, int64_t n,
                                 VT *__restrict__ D, DevStatus *st) {
    const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n) return;
    const int s = rp[r], e = rp[r + 1] - 1;
    int dj = -1;
    for (int j = s; j <= e; ++j)
        if (col[j] == (int)r) dj = j;  // the last diagonal entry wins, as in the reference
    if (dj < 0) {
        report(st, SMAX_ERR_NO_DIAG, r);
        return;
    }
    const VT d = val[dj];
    if (fabs((double)d) < 1e-16) report(st, SMAX_ERR_ZERO_DIAG, r);
    D[r] = d;
    if (dj != e) {
        const int tc = col[dj];
        col[dj] = col[e];
        col[e] = tc;
        const VT tv = val[dj];
        val[dj] = val[e];
        val[e] = tv;
    }
}

// D[r] = the last entry of row r, which the peel made the diagonal
template <typename VT>
__global__ void refresh_diag_kernel(const int *__restrict__ rp, const int *__restrict__ col,
                                    const VT *__restrict__ val, int64_t n, VT *__restrict__ D, DevStatus *st) {
    const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n) return;
    const int e = rp[r + 1] - 1;
    if (e < rp[r] || col[e] != (int)r) {
        report(st, SMAX_ERR_NO_DIAG, r);
        return;
    }
    const VT d = val[e];
    if (fabs((double)d) < 1e-16) report(st, SMAX_ERR_ZERO_DIAG, r);
    D[r] = d;
}

// ------------------------------------------------------------ the row op ---
// Element (row r, vector v) of X / B lives at r*rs + v*vs.
template <typename VT>
__device__ __forceinline__ void solve_row(const int *__restrict__ rp, const int *__restrict__ col,
                                          const VT *__restrict__ val, const VT *__restrict__ D, const VT *B, VT *X,
                                          int r, int64_t v, int64_t rs, int64_t vs) {
    const int s = rp[r], e = rp[r + 1] - 1;  // the diagonal sits at e
    VT sum = VT(0);
    const int64_t vo = v * vs;
    for (int j = s; j < e; ++j) sum += val[j] * X[(int64_t)col[j] * rs + vo];
    X[(int64_t)r * rs + vo] = (B[(int64_t)r * rs + vo] - sum) / D[r];
}

// thread t -> (i-th row of the level, vector v); rows vary fastest for
// column-major blocks, vectors for row-major ones (coalesced X accesses)
__device__ __forceinline__ void split_work(int64_t t, int64_t m, int64_t k, bool row_major, int64_t &i,
                                           int64_t &v) {
    if (row_major) { i = t / k; v = t % k; }
    else { i = t % m; v = t / m; }
}

template <typename VT>
__global__ void level_kernel(const int *__restrict__ rp, const int *__restrict__ col, const VT *__restrict__ val,
                             const VT *__restrict__ D, const int *__restrict__ order, int row0, int m, int64_t k,
                             bool row_major, int64_t rs, int64_t vs, const VT *B, VT *X) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (int64_t)m * k) return;
    int64_t i, v;
    split_work(t, m, k, row_major, i, v);
    const int r = order ? order[row0 + i] : row0 + (int)i;
    solve_row<VT>(rp, col, val, D, B, X, r, v, rs, vs);
}

// One CTA sweeps levels seg_lvl[0..n_lvls) (given as [begin, end) row ranges
// into `order`, or contiguous rows when order is null).
template <typename VT>
__global__ void __launch_bounds__(kSegThreads) segment_kernel(const int *__restrict__ rp, const int *__restrict__ col,
                                                              const VT *__restrict__ val, const VT *__restrict__ D,
                                                              const int *__restrict__ order,
                                                              const int2 *__restrict__ ranges, int n_lvls, int64_t k,
                                                              bool row_major, int64_t rs, int64_t vs, const VT *B,
                                                              VT *X) {
    for (int l = 0; l < n_lvls; ++l) {
        const int2 rg = ranges[l];
        const int64_t m = rg.y - rg.x;
        for (int64_t t = threadIdx.x; t < m * k; t += blockDim.x) {
            int64_t i, v;
            split_work(t, m, k, row_major, i, v);
            const int r = order ? order[rg.x + i] : rg.x + (int)i;
            solve_row<VT>(rp, col, val, D, B, X, r, v, rs, vs);
        }
        __syncthreads();
    }
}

}  // namespace

void peel_diag(DevCRS &a, int vbytes, DevBuf &D, DevStatus *st, cudaStream_t s) {
    D.alloc((size_t)vbytes * (a.n_rows ? a.n_rows : 1));
    if (a.n_rows == 0) return;
    const unsigned g = ceil_div_u(a.n_rows, 256);
    if (vbytes == 8)
        peel_diag_kernel<double><<<g, 256, 0, s>>>(a.rp(), a.col.as<int>(), a.val.as<double>(), a.n_rows,
                                                   D.as<double>(), st);
    else
        peel_diag_kernel<float><<<g, 256, 0, s>>>(a.rp(), a.col.as<int>(), a.val.as<float>(), a.n_rows,
                                                  D.as<float>(), st);
    SMAX_CUDA(cudaGetLastError());
}

void refresh_diag(const DevCRS &a, int vbytes, DevBuf &D, DevStatus *st, cudaStream_t s) {
    if (a.n_rows == 0) return;
    const unsigned g = ceil_div_u(a.n_rows, 256);
    if (vbytes == 8)
        refresh_diag_kernel<double><<<g, 256, 0, s>>>(a.rp(), a.ci(), a.val.as<double>(), a.n_rows, D.as<double>(), st);
    else
        refresh_diag_kernel<float><<<g, 256, 0, s>>>(a.rp(), a.ci(), a.val.as<float>(), a.n_rows, D.as<float>(), st);
    SMAX_CUDA(cudaGetLastError());
}

void TriPlan::build_own(const DevCRS &a, bool upper, cudaStream_t st) {
    DevBuf srp, scol, lvl;
    int64_t snnz = 0;
    build_symmetric(a, srp, scol, snnz, st);
    const int nl = rs_levels(srp.as<int>(), scol.as<int>(), a.n_rows, lvl, st, upper);
    level_order(lvl.as<int>(), a.n_rows, nl, order, lvl_ptr, st);
    if (a.n_rows > 0 && lvl_ptr.back() != a.n_rows) fail(SMAX_ERR_STATE, "dependency levels do not cover all rows");
    has_order = true;
    descending = false;
    n_rows = a.n_rows;
    finish(st);
}

void TriPlan::build_given(const std::vector<int> &lp, int64_t n, bool upper, cudaStream_t st) {
    if (lp.empty() || lp.front() != 0 || lp.back() != n) fail(SMAX_ERR_STATE, "level pointer does not match the matrix");
    for (size_t i = 1; i < lp.size(); ++i)
        if (lp[i] < lp[i - 1]) fail(SMAX_ERR_BAD_ARG, "level pointer is not monotone");
    lvl_ptr = lp;
    order.release();
    has_order = false;
    descending = upper;  // crs_sptrsv_lvl<false> walks levels from last to first
    n_rows = n;
    finish(st);
}

void TriPlan::assign_reverse(const TriPlan &src, cudaStream_t st) {
    release_graph();
    n_rows = src.n_rows;
    lvl_ptr = src.lvl_ptr;
    has_order = src.has_order;
    descending = !src.descending;
    if (src.has_order) {
        order.alloc(sizeof(int) * (n_rows > 0 ? n_rows : 1));
        if (n_rows) SMAX_CUDA(cudaMemcpyAsync(order.p, src.order.p, sizeof(int) * n_rows, cudaMemcpyDeviceToDevice, st));
    } else {
        order.release();
    }
    scheduled_k = -1;
    scheduled_merge = -1;
    finish(st);
}

void TriPlan::finish(cudaStream_t) {
    graph_valid = false;
    pack_ok = false;
    pack_unfit = false;
    pack = LevelPack();
    sf_ok = false;
    sf_unfit = false;
    sf_pack = LevelPack();
}

bool TriPlan::ensure_pack(const int *rp, const int *ci, const void *val, const void *D, int vbytes, int merge_rows,
                          uint64_t tag, cudaStream_t st) {
    if (scheduled_k != 1 || scheduled_merge != merge_rows) schedule(1, merge_rows);
    if (pack_ok && pack_key[0] == val && pack_key[1] == D && pack_tag == tag && pack_merge == merge_rows &&
        pack_vbytes == vbytes)
        return true;
    if (pack_unfit) return false;  // a property of the pattern and the level sets
    const int L = n_levels();
    std::vector<int> src_begin(L), count(L), seg_begin(L);
    pack_steps.clear();
    for (const Step &s : steps) {
        for (int i = 0; i < s.sweep_count; ++i) {
            const int sw = s.sweep_first + i;
            const int lv = descending ? L - 1 - sw : sw;
            src_begin[sw] = lvl_ptr[lv];
            count[sw] = lvl_ptr[lv + 1] - lvl_ptr[lv];
            seg_begin[sw] = s.kind == 1 ? s.sweep_first : sw;
        }
        pack_steps.push_back(PackStep{s.sweep_first, s.sweep_count, s.kind});
    }
    release_graph();
    pack_ok = false;
    const bool ok = build_level_pack(pack, rp, ci, val, D, vbytes, n_rows, has_order ? order.as<int>() : nullptr,
                                     src_begin, count, seg_begin, allow_cluster, st);
    if (!ok) {
        pack_unfit = true;
        return false;
    }
    pack_ok = true;
    pack_key[0] = val;
    pack_key[1] = D;
    pack_tag = tag;
    pack_merge = merge_rows;
    pack_vbytes = vbytes;
    return true;
}

bool TriPlan::ensure_syncfree(const int *rp, const int *ci, const void *val, const void *D, int vbytes, uint64_t tag,
                              cudaStream_t st) {
    if (sf_ok && sf_key[0] == val && sf_key[1] == D && sf_tag == tag && sf_vbytes == vbytes) return true;
    if (sf_unfit) return false;  // a property of the pattern and the level sets
    const int L = n_levels();
    std::vector<int> src_begin(L), count(L), seg_begin(L);
    for (int sw = 0; sw < L; ++sw) {
        const int lv = descending ? L - 1 - sw : sw;
        src_begin[sw] = lvl_ptr[lv];
        count[sw] = lvl_ptr[lv + 1] - lvl_ptr[lv];
        seg_begin[sw] = sw;
    }
    sf_ok = false;
    const bool ok = build_level_pack(sf_pack, rp, ci, val, D, vbytes, n_rows, has_order ? order.as<int>() : nullptr,
                                     src_begin, count, seg_begin, false, st, true);
    if (!ok || sf_pack.needs_x_init) {
        sf_pack = LevelPack();
        sf_unfit = true;
        return false;
    }
    sf_ok = true;
    sf_key[0] = val;
    sf_key[1] = D;
    sf_tag = tag;
    sf_vbytes = vbytes;
    return true;
}

void TriPlan::prepare(int64_t k, int merge_rows, cudaStream_t st) {
    if (scheduled_k != k || scheduled_merge != merge_rows) schedule(k, merge_rows);
    if (!ranges_uploaded && !seg_ranges.empty()) {
        SMAX_CUDA(cudaMemcpyAsync(d_ranges.p, seg_ranges.data(), sizeof(int2) * seg_ranges.size(),
                                  cudaMemcpyHostToDevice, st));
        ranges_uploaded = true;
        SMAX_CUDA(cudaStreamSynchronize(st));
    }
}

// Sequence of steps: wide levels alone, runs of narrow levels merged.
void TriPlan::schedule(int64_t k, int merge_rows) {
    steps.clear();
    seg_ranges.clear();
    const int L = (int)lvl_ptr.size() - 1;
    int l = 0;
    auto level_at = [&](int idx) { return descending ? L - 1 - idx : idx; };
    while (l < L) {
        const int lv = level_at(l);
        const int64_t m = lvl_ptr[lv + 1] - lvl_ptr[lv];
        if (merge_rows > 0 && m * k <= merge_rows) {
            const int l0 = l;
            while (l < L) {
                const int lv2 = level_at(l);
                const int64_t m2 = lvl_ptr[lv2 + 1] - lvl_ptr[lv2];
                if (m2 * k > merge_rows) break;
                ++l;
            }
            // One right-hand side: the run's single-CTA sweep is sized by its
            // widest level (256 / 512 / 1024 threads for up to 512 / 1024 /
            // more rows), and every warp of it passes every level.  Long
            // stretches of narrower levels become runs of their own, on fewer
            // threads; stretches shorter than kMinStretch levels stay with a
            // neighbour (a run boundary costs a launch, and the first level of
            // a run reads its sources from global memory instead of the ring).
            std::vector<std::pair<int, int>> parts;  // (first sweep step, width class)
            auto width_class = [&](int idx) {
                const int lv2 = level_at(idx);
                const int64_t m2 = lvl_ptr[lv2 + 1] - lvl_ptr[lv2];
                return k == 1 ? (m2 <= 512 ? 0 : (m2 <= 1024 ? 1 : 2)) : 0;
            };
            for (int i = l0; i < l; ++i) {
                const int c = width_class(i);
                if (parts.empty() || parts.back().second != c) parts.push_back({i, c});
            }
            constexpr int kMinStretch = 64;
            for (bool changed = true; changed && parts.size() > 1;) {
                changed = false;
                for (size_t i = 0; i < parts.size(); ++i) {
                    const int end = i + 1 < parts.size() ? parts[i + 1].first : l;
                    if (end - parts[i].first >= kMinStretch) continue;
                    // merge the short stretch into its wider neighbour
                    size_t j;
                    if (i == 0) j = 1;
                    else if (i + 1 == parts.size()) j = i - 1;
                    else j = parts[i - 1].second >= parts[i + 1].second ? i - 1 : i + 1;
                    const size_t lo = std::min(i, j);
                    parts[lo].second = std::max(parts[i].second, parts[j].second);
                    parts.erase(parts.begin() + (long)(lo + 1));
                    // neighbours of equal class join
                    if (lo + 1 < parts.size() && parts[lo + 1].second == parts[lo].second)
                        parts.erase(parts.begin() + (long)(lo + 1));
                    if (lo > 0 && parts[lo - 1].second == parts[lo].second) parts.erase(parts.begin() + (long)lo);
                    changed = true;
                    break;
                }
            }
            for (size_t pi = 0; pi < parts.size(); ++pi) {
                const int a = parts[pi].first, b = pi + 1 < parts.size() ? parts[pi + 1].first : l;
                Step s;
                s.kind = 1;
                s.seg_first = (int)seg_ranges.size();
                s.sweep_first = a;
                for (int i = a; i < b; ++i) {
                    const int lv2 = level_at(i);
                    seg_ranges.push_back({lvl_ptr[lv2], lvl_ptr[lv2 + 1]});
                }
                s.seg_count = (int)seg_ranges.size() - s.seg_first;
                s.sweep_count = s.seg_count;
                steps.push_back(s);
            }
        } else {
            Step s;
            s.kind = 0;
            s.row0 = lvl_ptr[lv];
            s.m = (int)m;
            s.sweep_first = l;
            s.sweep_count = 1;
            steps.push_back(s);
            ++l;
        }
    }
    d_ranges.alloc(sizeof(int2) * (seg_ranges.empty() ? 1 : seg_ranges.size()));
    scheduled_k = k;
    scheduled_merge = merge_rows;
    ranges_uploaded = false;
    graph_valid = false;
}

template <typename VT>
void tri_solve(TriPlan &p, const DevCRS &a, const VT *D, const VT *B, VT *X, int64_t k, bool row_major, int64_t ld,
               int merge_rows, uint64_t tag, cudaStream_t st) {
    if (k == 1 && p.n_rows > 0) p.ensure_pack(a.rp(), a.ci(), a.val.p, D, sizeof(VT), merge_rows, tag, st);
    tri_solve_raw<VT>(p, a.rp(), a.ci(), a.val.as<VT>(), D, B, X, k, row_major, ld, merge_rows, tag, st);
}

template <typename VT>
void tri_solve_raw(TriPlan &p, const int *rp, const int *ci, const VT *val, const VT *D, const VT *B, VT *X,
                   int64_t k, bool row_major, int64_t ld, int merge_rows, uint64_t tag, cudaStream_t st) {
    if (p.n_rows == 0) return;
    if (k == 1 && p.pack_ok && p.pack_key[0] == val && p.pack_key[1] == D && p.pack_tag == tag &&
        p.pack_merge == merge_rows && p.pack_vbytes == (int)sizeof(VT)) {
        pack_solve<VT>(p.pack, p.pack_steps, B, X, st);
        return;
    }
    if (p.scheduled_k != k || p.scheduled_merge != merge_rows) p.schedule(k, merge_rows);
    if (!p.ranges_uploaded && !p.seg_ranges.empty()) {
        SMAX_CUDA(cudaMemcpyAsync(p.d_ranges.p, p.seg_ranges.data(), sizeof(int2) * p.seg_ranges.size(),
                                  cudaMemcpyHostToDevice, st));
        p.ranges_uploaded = true;
    }
    const int64_t rs = row_major ? k : 1, vs = row_major ? 1 : ld;
    const int *order = p.has_order ? p.order.as<int>() : nullptr;
    const int2 *ranges = p.d_ranges.as<int2>();
    for (const auto &s : p.steps) {
        if (s.kind == 0) {
            const int64_t work = (int64_t)s.m * k;
            level_kernel<VT><<<ceil_div_u(work, 256), 256, 0, st>>>(rp, ci, val, D, order, s.row0, s.m, k, row_major,
                                                                    rs, vs, B, X);
        } else {
            segment_kernel<VT><<<1, kSegThreads, 0, st>>>(rp, ci, val, D, order, ranges + s.seg_first, s.seg_count, k,
                                                          row_major, rs, vs, B, X);
        }
    }
    SMAX_CUDA(cudaGetLastError());
}

template <typename VT>
void tri_solve_graph(TriPlan &p, const DevCRS &a, const VT *D, const VT *B, VT *X, int64_t k, bool row_major,
                     int64_t ld, int merge_rows, uint64_t tag, cudaStream_t caller) {
    if (p.n_rows == 0) return;
    // the pack is built outside the capture (it synchronises); a rebuild drops the graph
    if (k == 1) p.ensure_pack(a.rp(), a.ci(), a.val.p, D, sizeof(VT), merge_rows, tag, caller);
    // graphs are captured (and replayed) on a capturable stream
    const bool fenced = !is_capturable(caller);
    cudaStream_t st = fenced ? p.aux.enter(caller) : caller;
    struct Leave {
        TriPlan &p;
        bool fenced;
        cudaStream_t caller;
        ~Leave() {
            if (fenced) {
                cudaEventRecord(p.aux.out, p.aux.s);
                cudaStreamWaitEvent(caller, p.aux.out, 0);
            }
        }
    } leave{p, fenced, caller};
    if (p.scheduled_k != k || p.scheduled_merge != merge_rows) p.schedule(k, merge_rows);
    const void *key[4] = {B, X, D, a.val.p};
    if (!p.graph_valid || p.graph_key[0] != key[0] || p.graph_key[1] != key[1] || p.graph_key[2] != key[2] ||
        p.graph_key[3] != key[3] || p.graph_row_major != row_major || p.graph_ld != ld) {
        if (!p.ranges_uploaded && !p.seg_ranges.empty()) {
            SMAX_CUDA(cudaMemcpyAsync(p.d_ranges.p, p.seg_ranges.data(), sizeof(int2) * p.seg_ranges.size(),
                                      cudaMemcpyHostToDevice, st));
            p.ranges_uploaded = true;
        }
        SMAX_CUDA(cudaStreamSynchronize(st));
        p.release_graph();
        cudaGraph_t g = nullptr;
        SMAX_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
        try {
            tri_solve_raw<VT>(p, a.rp(), a.ci(), a.val.as<VT>(), D, B, X, k, row_major, ld, merge_rows, tag, st);
        } catch (...) {
            cudaStreamEndCapture(st, &g);
            if (g) cudaGraphDestroy(g);
            throw;
        }
        SMAX_CUDA(cudaStreamEndCapture(st, &g));
        cudaGraphExec_t ge = nullptr;
        cudaError_t e = cudaGraphInstantiate(&ge, g, 0);
        cudaGraphDestroy(g);
        cuda_check(e, "cudaGraphInstantiate");
        p.graph = ge;
        p.graph_valid = true;
        p.graph_key[0] = key[0];
        p.graph_key[1] = key[1];
        p.graph_key[2] = key[2];
        p.graph_key[3] = key[3];
        p.graph_row_major = row_major;
        p.graph_ld = ld;
    }
    SMAX_CUDA(cudaGraphLaunch(p.graph, st));
}

void TriPlan::release_graph() {
    if (graph) cudaGraphExecDestroy(graph);
    graph = nullptr;
    graph_valid = false;
}

TriPlan::~TriPlan() { release_graph(); }

bool syncfree_suits(const TriPlan &p, int64_t k) {
    const int64_t L = p.n_levels();
    if (L <= 0) return false;
    if (k == 1) return p.n_rows >= (1 << 17) && p.n_rows >= L * 32768;
    return p.n_rows >= (1 << 16) && L >= 64 && p.n_rows <= L * 16384;
}

template <typename VT>
bool tri_solve_syncfree(TriPlan &p, const DevCRS &a, const VT *D, const VT *B, VT *X, uint64_t tag, DevBuf &ctl,
                        long long limit, bool force_timeout, DevStatus *st, cudaStream_t s, int64_t k,
                        bool row_major) {
    if (p.n_rows == 0 || k == 0) return true;
    const uintptr_t b0 = reinterpret_cast<uintptr_t>(B), x0 = reinterpret_cast<uintptr_t>(X);
    const uintptr_t len = sizeof(VT) * (uintptr_t)p.n_rows * (uintptr_t)k;
    if (b0 < x0 + len && x0 < b0 + len) return false;  // B is read while X fills
    if (!p.ensure_syncfree(a.rp(), a.ci(), a.val.p, D, sizeof(VT), tag, s)) return false;
    ctl.ensure(64);
    if (k == 1)
        pack_solve_syncfree<VT>(p.sf_pack, B, X, ctl.p, limit, force_timeout, st, s);
    else
        solve_syncfree_rows<VT>(p.sf_pack, a.rp(), a.ci(), a.val.as<VT>(), D, B, X, k, row_major, ctl.p, limit, st,
                                s);
    return true;
}

template bool tri_solve_syncfree<double>(TriPlan &, const DevCRS &, const double *, const double *, double *, uint64_t,
                                         DevBuf &, long long, bool, DevStatus *, cudaStream_t, int64_t, bool);
template bool tri_solve_syncfree<float>(TriPlan &, const DevCRS &, const float *, const float *, float *, uint64_t,
                                        DevBuf &, long long, bool, DevStatus *, cudaStream_t, int64_t, bool);
template void tri_solve<double>(TriPlan &, const DevCRS &, const double *, const double *, double *, int64_t, bool,
                                int64_t, int, uint64_t, cudaStream_t);
template void tri_solve<float>(TriPlan &, const DevCRS &, const float *, const float *, float *, int64_t, bool,
                               int64_t, int, uint64_t, cudaStream_t);
template void tri_solve_raw<double>(TriPlan &, const int *, const int *, const double *, const double *,
                                    const double *, double *, int64_t, bool, int64_t, int, uint64_t, cudaStream_t);
template void tri_solve_raw<float>(TriPlan &, const int *, const int *, const float *, const float *, const float *,
                                   float *, int64_t, bool, int64_t, int, uint64_t, cudaStream_t);
template void tri_solve_graph<double>(TriPlan &, const DevCRS &, const double *, const double *, double *, int64_t,
                                      bool, int64_t, int, uint64_t, cudaStream_t);
template void tri_solve_graph<float>(TriPlan &, const DevCRS &, const float *, const float *, float *, int64_t, bool,
                                     int64_t, int, uint64_t, cudaStream_t);

}  // namespace smax
