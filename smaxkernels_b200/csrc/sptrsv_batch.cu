// sptrsv_batch.cu -- persistent triangular solves.
//
// 1. Batched: many independent triangular matrices of uneven size in ONE
//    persistent launch.  The matrices are packed back to back (global row
//    numbering, their rows sorted by dependency level).  Each CTA takes the
//    next matrix from a device work queue (an atomic counter over the matrices
//    in longest-first order) and sweeps that matrix's levels, with
//    __syncthreads() as the level barrier; when done it takes the next one.
//    The sweep runs on the level-ordered pack of the batch (levelpack.cu:
//    per-level ELL blocks, a shared-memory ring of recent solutions, the next
//    level prefetched into registers); matrices that would pack too sparsely
//    use the plain kernel below.
//    There is no spin-wait anywhere: the queue is a fetch-add and the level
//    barrier is the CTA barrier.  The launch (queue reset + kernel) is
//    captured once into a CUDA graph and replayed.
// 2. Grid-wide persistent (one matrix, wide levels): a cooperative launch of
//    co-resident CTAs sweeps all levels, with a software grid barrier between
//    levels.  The barrier spins with an iteration limit; when the limit is hit
//    it records SMAX_ERR_TIMEOUT in the status word and every CTA returns, so
//    the context stays usable and the host gets an error.  A test knob makes
//    the barrier wait for one arrival more than exists, to exercise that path.
//
// Row arithmetic as in sptrsv.cu (the reference's per-row recurrence and order).
#include <algorithm>
#include <numeric>

#include "sptrsv_batch.cuh"

namespace smax {

namespace {

constexpr int kBatchThreads = 1024;
constexpr int kGridThreads = 512;

template <typename VT>
__device__ __forceinline__ void batch_row(const int *__restrict__ rp, const int *__restrict__ col,
                                          const VT *__restrict__ val, const VT *__restrict__ D, const VT *B, VT *X,
                                          int r) {
    const int s = rp[r], e = rp[r + 1] - 1;
    VT sum = VT(0);
    for (int j = s; j < e; ++j) sum += val[j] * X[col[j]];
    X[r] = (B[r] - sum) / D[r];
}

// Work queue of matrices; each CTA sweeps the levels of its matrix.
template <typename VT>
__global__ void __launch_bounds__(kBatchThreads) batch_persistent(const int *__restrict__ rp, const int *__restrict__ col,
                                                                  const VT *__restrict__ val, const VT *__restrict__ D,
                                                                  const int *__restrict__ order,
                                                                  const int *__restrict__ mat_lvl_off,
                                                                  const int *__restrict__ lvl_rows,
                                                                  const int *__restrict__ queue_order, int n_mats,
                                                                  int *queue, const VT *B, VT *X) {
    __shared__ int m_sh;
    while (true) {
        if (threadIdx.x == 0) m_sh = atomicAdd(queue, 1);
        __syncthreads();
        const int q = m_sh;
        __syncthreads();  // m_sh is rewritten on the next turn
        if (q >= n_mats) return;
        const int m = queue_order[q];
        for (int l = mat_lvl_off[m]; l < mat_lvl_off[m + 1]; ++l) {
            const int a = lvl_rows[l], b = lvl_rows[l + 1];
            for (int i = a + threadIdx.x; i < b; i += blockDim.x) batch_row<VT>(rp, col, val, D, B, X, order[i]);
            __syncthreads();
        }
    }
}

// one launch per level of one matrix (the plain baseline)
template <typename VT>
__global__ void batch_level(const int *__restrict__ rp, const int *__restrict__ col, const VT *__restrict__ val,
                            const VT *__restrict__ D, const int *__restrict__ order, int a, int b, const VT *B, VT *X) {
    const int i = a + blockIdx.x * blockDim.x + threadIdx.x;
    if (i < b) batch_row<VT>(rp, col, val, D, B, X, order[i]);
}

// ------------------------------------------------------- grid barrier ----
struct GridBarrier {
    unsigned *count;
    unsigned *gen;
};

__device__ __forceinline__ unsigned ld_acquire(const unsigned *p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// Returns false (and leaves) once any CTA has timed out.  `expected` is the
// number of arrivals that release the barrier (gridDim.x normally).
__device__ bool grid_sync(GridBarrier gb, unsigned expected, long long limit, DevStatus *st, int *abort_flag) {
    __syncthreads();
    __shared__ int ok;
    if (threadIdx.x == 0) {
        ok = 1;
        __threadfence();
        const unsigned g = ld_acquire(gb.gen);
        const unsigned arrived = atomicAdd(gb.count, 1u) + 1u;
        if (arrived == expected) {
            *gb.count = 0;
            __threadfence();
            atomicAdd(gb.gen, 1u);
        } else {
            long long it = 0;
            while (ld_acquire(gb.gen) == g) {
                if (*(volatile int *)abort_flag) { ok = 0; break; }
                if (++it > limit) {
                    report(st, SMAX_ERR_TIMEOUT, it);
                    atomicExch(abort_flag, 1);
                    ok = 0;
                    break;
                }
                __nanosleep(64);
            }
        }
    }
    __syncthreads();
    return ok != 0;
}

template <typename VT>
__global__ void grid_persistent(const int *__restrict__ rp, const int *__restrict__ col, const VT *__restrict__ val,
                                const VT *__restrict__ D, const int *__restrict__ order,
                                const int *__restrict__ lvl_rows, int n_levels, int descending, const VT *B, VT *X,
                                GridBarrier gb, unsigned expected, long long limit, DevStatus *st, int *abort_flag) {
    const int64_t tid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t nth = (int64_t)gridDim.x * blockDim.x;
    for (int t = 0; t < n_levels; ++t) {
        const int l = descending ? n_levels - 1 - t : t;
        const int a = lvl_rows[l], b = lvl_rows[l + 1];
        for (int64_t i = a + tid; i < b; i += nth) {
            const int r = order ? order[i] : (int)i;
            // dependencies were written by other CTAs: read them through L2
            const int s = rp[r], e = rp[r + 1] - 1;
            VT sum = VT(0);
            for (int j = s; j < e; ++j) sum += val[j] * __ldcg(X + col[j]);
            X[r] = (__ldcg(B + r) - sum) / D[r];
        }
        if (t + 1 < n_levels && !grid_sync(gb, expected, limit, st, abort_flag)) return;
    }
}

}  // namespace

// ------------------------------------------------------------- the batch ---
void TriBatch::build(int vbytes_, const std::vector<RegCRS> &mats, cudaStream_t st) {
    vbytes = vbytes_;
    n_mats = (int)mats.size();
    // pack the matrices as one block-diagonal CRS with global column indices
    std::vector<int64_t> roff(n_mats + 1, 0), zoff(n_mats + 1, 0);
    for (int m = 0; m < n_mats; ++m) {
        if (mats[m].n_rows != mats[m].n_cols) fail(SMAX_ERR_BAD_ARG, "triangular matrices must be square");
        roff[m + 1] = roff[m] + (int64_t)mats[m].n_rows;
        zoff[m + 1] = zoff[m] + (int64_t)mats[m].nnz;
    }
    n_rows = roff[n_mats];
    nnz = zoff[n_mats];
    if (n_rows >= (1ll << 31) || nnz >= (1ll << 31)) fail(SMAX_ERR_UNSUPPORTED, "batch exceeds int32 indexing");
    std::vector<int> rp(n_rows + 1), cl(nnz);
    std::vector<char> vv((size_t)vbytes * nnz);
    for (int m = 0; m < n_mats; ++m) {
        const int *mrp = static_cast<const int *>(mats[m].row_ptr);
        const int *mcl = static_cast<const int *>(mats[m].col);
        for (uint64_t r = 0; r < mats[m].n_rows; ++r) rp[roff[m] + r] = (int)(zoff[m] + mrp[r]);
        for (uint64_t j = 0; j < mats[m].nnz; ++j) {
            const int c = mcl[j];
            if (c < 0 || (uint64_t)c >= mats[m].n_cols) fail(SMAX_ERR_COL_OOB, "column index out of range");
            cl[zoff[m] + j] = (int)(c + roff[m]);
        }
        if (mats[m].nnz)
            std::memcpy(vv.data() + (size_t)vbytes * zoff[m], mats[m].val, (size_t)vbytes * mats[m].nnz);
        if (mrp[0] != 0 || (uint64_t)mrp[mats[m].n_rows] != mats[m].nnz)
            fail(SMAX_ERR_BAD_ARG, "row_ptr does not match nnz");
    }
    rp[n_rows] = (int)nnz;
    RegCRS packed{true, (uint64_t)n_rows, (uint64_t)n_rows, (uint64_t)nnz, cl.data(), rp.data(), vv.data()};
    upload_crs(A, packed, vbytes, st);
    DevBuf status(sizeof(DevStatus));
    SMAX_CUDA(cudaMemsetAsync(status.p, 0, sizeof(DevStatus), st));
    validate_crs(A, status.as<DevStatus>(), st);
    peel_diag(A, vbytes, D, status.as<DevStatus>(), st);
    DevStatus h{};
    SMAX_CUDA(cudaMemcpyAsync(&h, status.p, sizeof(h), cudaMemcpyDeviceToHost, st));
    SMAX_CUDA(cudaStreamSynchronize(st));
    if (h.code) fail(h.code, "batch matrix rejected at packed row/entry " + std::to_string(h.index));
    // dependency levels of the block-diagonal matrix, split back per matrix:
    // a level of the packed matrix restricted to one block is that matrix's level
    DevBuf srp, scol, lvl;
    int64_t snnz = 0;
    build_symmetric(A, srp, scol, snnz, st);
    const int nl = rs_levels(srp.as<int>(), scol.as<int>(), n_rows, lvl, st, false);
    std::vector<int> hl(n_rows);
    SMAX_CUDA(cudaMemcpyAsync(hl.data(), lvl.p, sizeof(int) * n_rows, cudaMemcpyDeviceToHost, st));
    SMAX_CUDA(cudaStreamSynchronize(st));
    // per matrix: rows sorted by (level, row); level boundaries
    std::vector<int> ord(n_rows), lrows, moff(n_mats + 1, 0);
    mat_levels.assign(n_mats, 0);
    for (int m = 0; m < n_mats; ++m) {
        int mx = -1;
        for (int64_t r = roff[m]; r < roff[m + 1]; ++r) mx = std::max(mx, hl[r]);
        const int L = mx + 1;
        std::vector<int> cnt(L + 1, 0);
        for (int64_t r = roff[m]; r < roff[m + 1]; ++r) cnt[hl[r] + 1]++;
        for (int l = 0; l < L; ++l) cnt[l + 1] += cnt[l];
        for (int l = 0; l < L; ++l) lrows.push_back((int)(roff[m] + cnt[l]));
        std::vector<int> pos(cnt.begin(), cnt.end() - 1);
        for (int64_t r = roff[m]; r < roff[m + 1]; ++r) ord[roff[m] + pos[hl[r]]++] = (int)r;
        moff[m + 1] = moff[m] + L;
        mat_levels[m] = L;
    }
    lrows.push_back((int)n_rows);
    (void)nl;
    // longest critical path first
    std::vector<int> qo(n_mats);
    std::iota(qo.begin(), qo.end(), 0);
    std::stable_sort(qo.begin(), qo.end(), [&](int a, int b) {
        if (mat_levels[a] != mat_levels[b]) return mat_levels[a] > mat_levels[b];
        return roff[a + 1] - roff[a] > roff[b + 1] - roff[b];
    });
    total_levels = moff[n_mats];
    auto up = [&](DevBuf &d, const std::vector<int> &h) {
        d.alloc(sizeof(int) * (h.empty() ? 1 : h.size()));
        if (!h.empty()) SMAX_CUDA(cudaMemcpyAsync(d.p, h.data(), sizeof(int) * h.size(), cudaMemcpyHostToDevice, st));
    };
    up(order, ord);
    up(mat_lvl_off, moff);
    up(lvl_rows, lrows);
    up(queue_order, qo);
    queue.alloc(sizeof(int));
    h_lvl_rows = lrows;
    h_mat_lvl_off = moff;
    row_off = roff;
    SMAX_CUDA(cudaStreamSynchronize(st));
    // sweep steps = every matrix's levels in order; each matrix is one run
    const int L = total_levels;
    std::vector<int> src_begin(L), count(L), seg_begin(L);
    for (int m = 0; m < n_mats; ++m)
        for (int l = moff[m]; l < moff[m + 1]; ++l) {
            src_begin[l] = lrows[l];
            count[l] = lrows[l + 1] - lrows[l];
            seg_begin[l] = moff[m];
        }
    pack_ok = build_level_pack(pack, A.rp(), A.ci(), A.val.p, D.p, vbytes, n_rows, order.as<int>(), src_begin, count,
                               seg_begin, false, st);
}

template <typename VT>
void TriBatch::solve_persistent(const VT *B, VT *X, cudaStream_t st) {
    if (n_mats == 0) return;
    if (pack_ok) {
        pack_solve_batch<VT>(pack, mat_lvl_off.as<int>(), queue_order.as<int>(), n_mats, queue.as<int>(), B, X, st);
        return;
    }
    int per_sm = 0;
    SMAX_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, batch_persistent<VT>, kBatchThreads, 0));
    const int grid = std::max(1, std::min(n_mats, per_sm * sm_count()));
    SMAX_CUDA(cudaMemsetAsync(queue.p, 0, sizeof(int), st));
    batch_persistent<VT><<<grid, kBatchThreads, 0, st>>>(A.rp(), A.ci(), A.val.as<VT>(), D.as<VT>(), order.as<int>(),
                                                         mat_lvl_off.as<int>(), lvl_rows.as<int>(),
                                                         queue_order.as<int>(), n_mats, queue.as<int>(), B, X);
    SMAX_CUDA(cudaGetLastError());
}

template <typename VT>
void TriBatch::solve_graph(const VT *B, VT *X, cudaStream_t caller) {
    if (n_mats == 0) return;
    const bool fenced = !is_capturable(caller);
    cudaStream_t st = fenced ? aux.enter(caller) : caller;
    struct Leave {
        AuxStream &aux;
        bool fenced;
        cudaStream_t caller;
        ~Leave() {
            if (fenced) {
                cudaEventRecord(aux.out, aux.s);
                cudaStreamWaitEvent(caller, aux.out, 0);
            }
        }
    } leave{aux, fenced, caller};
    if (!graph || graph_b != B || graph_x != X) {
        if (graph) cudaGraphExecDestroy(graph);
        graph = nullptr;
        SMAX_CUDA(cudaStreamSynchronize(st));
        cudaGraph_t g = nullptr;
        SMAX_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
        try {
            solve_persistent<VT>(B, X, st);
        } catch (...) {
            cudaStreamEndCapture(st, &g);
            if (g) cudaGraphDestroy(g);
            throw;
        }
        SMAX_CUDA(cudaStreamEndCapture(st, &g));
        cudaError_t e = cudaGraphInstantiate(&graph, g, 0);
        cudaGraphDestroy(g);
        cuda_check(e, "cudaGraphInstantiate");
        graph_b = B;
        graph_x = X;
    }
    SMAX_CUDA(cudaGraphLaunch(graph, st));
}

template <typename VT>
void TriBatch::solve_per_level(const VT *B, VT *X, cudaStream_t st) {
    for (int m = 0; m < n_mats; ++m)
        for (int l = h_mat_lvl_off[m]; l < h_mat_lvl_off[m + 1]; ++l) {
            const int a = h_lvl_rows[l], b = h_lvl_rows[l + 1];
            batch_level<VT><<<ceil_div_u(b - a, 256), 256, 0, st>>>(A.rp(), A.ci(), A.val.as<VT>(), D.as<VT>(),
                                                                    order.as<int>(), a, b, B, X);
        }
    SMAX_CUDA(cudaGetLastError());
}

TriBatch::~TriBatch() {
    if (graph) cudaGraphExecDestroy(graph);
}

template void TriBatch::solve_persistent<double>(const double *, double *, cudaStream_t);
template void TriBatch::solve_persistent<float>(const float *, float *, cudaStream_t);
template void TriBatch::solve_graph<double>(const double *, double *, cudaStream_t);
template void TriBatch::solve_graph<float>(const float *, float *, cudaStream_t);
template void TriBatch::solve_per_level<double>(const double *, double *, cudaStream_t);
template void TriBatch::solve_per_level<float>(const float *, float *, cudaStream_t);

// ---------------------------------------------------- grid-wide persistent --
template <typename VT>
void tri_solve_persistent(const TriPlan &p, const DevCRS &a, const VT *D, const VT *B, VT *X, DevStatus *st,
                          DevBuf &scratch, bool force_timeout, long long spin_limit, cudaStream_t s) {
    if (p.n_rows == 0) return;
    // level row ranges of the sweep, in the plan's row numbering
    const int L = p.n_levels();
    scratch.ensure(sizeof(int) * (L + 1) + 4 * sizeof(unsigned) + 256);
    int *lvl_rows = scratch.as<int>();
    unsigned *bar = reinterpret_cast<unsigned *>(static_cast<char *>(scratch.p) + sizeof(int) * (L + 1));
    bar = reinterpret_cast<unsigned *>((reinterpret_cast<uintptr_t>(bar) + 15) & ~uintptr_t(15));
    SMAX_CUDA(cudaMemcpyAsync(lvl_rows, p.lvl_ptr.data(), sizeof(int) * (L + 1), cudaMemcpyHostToDevice, s));
    SMAX_CUDA(cudaMemsetAsync(bar, 0, 4 * sizeof(unsigned), s));
    int per_sm = 0;
    SMAX_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, grid_persistent<VT>, kGridThreads, 0));
    if (per_sm < 1) fail(SMAX_ERR_UNSUPPORTED, "persistent solve kernel cannot be resident");
    const int grid = std::min(per_sm, 2) * sm_count();  // co-resident by construction (cooperative launch)
    GridBarrier gb{bar, bar + 1};
    int *abort_flag = reinterpret_cast<int *>(bar + 2);
    const unsigned expected = (unsigned)grid + (force_timeout ? 1u : 0u);
    const int *order = p.has_order ? p.order.as<int>() : nullptr;
    const VT *val = a.val.as<VT>();
    const int *rp = a.rp(), *ci = a.ci();
    int desc = p.descending ? 1 : 0;
    void *args[] = {(void *)&rp, (void *)&ci, (void *)&val, (void *)&D, (void *)&order, (void *)&lvl_rows,
                    (void *)&L, (void *)&desc, (void *)&B, (void *)&X, (void *)&gb, (void *)&expected,
                    (void *)&spin_limit, (void *)&st, (void *)&abort_flag};
    SMAX_CUDA(cudaLaunchCooperativeKernel((const void *)grid_persistent<VT>, dim3(grid), dim3(kGridThreads), args, 0,
                                          s));
}

template void tri_solve_persistent<double>(const TriPlan &, const DevCRS &, const double *, const double *, double *,
                                           DevStatus *, DevBuf &, bool, long long, cudaStream_t);
template void tri_solve_persistent<float>(const TriPlan &, const DevCRS &, const float *, const float *, float *,
                                          DevStatus *, DevBuf &, bool, long long, cudaStream_t);

}  // namespace smax
