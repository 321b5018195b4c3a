// colour.cu -- the colouring permutations of Utils::generate_perm ("SC",
// "PC", "PC_BAL") and Utils::sanity_check_perm, on the GPU.
//
// Reference: src/utils/permutations.hpp.
//   * generate_color_perm (:588-647, "SC"): roots (rows without a lower
//     neighbour in A+A^T) queued in ascending order, then a FIFO
//     breadth-first search in which each dequeued node u takes the smallest
//     colour not used by its neighbours dequeued before it.
//   * generate_color_perm_par (:649-714, "PC"): with one OpenMP thread, rows
//     in ascending order, each taking the smallest colour not used by its
//     lower neighbours (the higher ones are still uncoloured).
//   * generate_color_perm_bal (:716-792, "PC_BAL", after PC): b = n / colours
//     (integer division); rows in ascending order; a row whose colour class
//     holds more than b rows moves to the smallest colour that no neighbour
//     has and whose class holds fewer than b rows, if one exists.
//   * sanity_check_perm (:794-818): no row shares a non-zero colour with a
//     lower neighbour.
// With more than one thread the reference's colourings depend on thread
// timing; these are the one-thread results, reproduced exactly.
//
// GPU: a greedy colouring in a fixed order is the same as colouring by
// dependency levels -- a node's colour depends only on the colours of its
// neighbours earlier in the order, and those all lie in earlier levels of
// the longest-path levels over "earlier" edges.  PC uses the RS levels
// (earlier = lower index); SC computes its queue order (hop distances from
// the roots, each level ordered by first discoverer) and uses levels over
// "earlier in the queue".  Each level's nodes are coloured in parallel with a
// 64-bit mask of the neighbours' colours (a scan above 64 colours); runs of
// small levels share one CTA with __syncthreads between levels.  The PC_BAL
// pass is sequential by definition (every move changes the class sizes the
// next rows test), so one warp walks the rows whose class starts oversized
// (the only ones that can move: a class never grows past b), with the class
// sizes and the colours a row's neighbours forbid in shared memory.
#include <cub/device/device_select.cuh>
#include <thrust/iterator/counting_iterator.h>

#include <vector>

#include "levels.cuh"

namespace smax {

namespace {

constexpr int kSmallNodes = 4096;  // levels up to this size share one CTA
constexpr int kSmallThreads = 1024;
constexpr int kMaxBalanceColours = 12288;  // class sizes + marks of the PC_BAL pass in shared memory

// the node is earlier in the colouring order than u
__device__ __forceinline__ bool earlier(int v, int u, const int *prio) {
    return prio ? prio[v] < prio[u] : v < u;
}

// smallest colour not held by an earlier neighbour of u
__device__ int mex_colour(const int *__restrict__ srp, const int *__restrict__ scol, const int *prio, const int *colour,
                          int u) {
    unsigned long long mask = 0ull;
    const int b = srp[u], e = srp[u + 1];
    for (int j = b; j < e; ++j) {
        const int v = scol[j];
        if (earlier(v, u, prio)) {
            const int c = __ldcg(colour + v);
            if (c < 64) mask |= 1ull << c;
        }
    }
    if (~mask) return __ffsll((long long)~mask) - 1;
    for (int c = 64;; ++c) {  // all of 0..63 are taken: scan upward (ends within deg + 1 colours)
        bool used = false;
        for (int j = b; j < e && !used; ++j) {
            const int v = scol[j];
            used = earlier(v, u, prio) && __ldcg(colour + v) == c;
        }
        if (!used) return c;
    }
}

__global__ void __launch_bounds__(kSmallThreads)
    colour_small_levels(const int *__restrict__ srp, const int *__restrict__ scol, const int *prio,
                        const int *__restrict__ lvl_ptr, const int *__restrict__ order, int l0, int l1, int *colour) {
    for (int l = l0; l < l1; ++l) {
        const int a = lvl_ptr[l], b = lvl_ptr[l + 1];
        for (int i = a + threadIdx.x; i < b; i += blockDim.x) {
            const int u = order[i];
            colour[u] = mex_colour(srp, scol, prio, colour, u);
        }
        __syncthreads();  // this level's colours are visible before the next level reads them
    }
}

__global__ void colour_level(const int *__restrict__ srp, const int *__restrict__ scol, const int *prio,
                             const int *__restrict__ order, int a, int b, int *colour) {
    const int i = a + blockIdx.x * blockDim.x + threadIdx.x;
    if (i < b) {
        const int u = order[i];
        colour[u] = mex_colour(srp, scol, prio, colour, u);
    }
}

__global__ void max_reduce(const int *__restrict__ a, int64_t n, int *out) {
    int m = 0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        m = max(m, a[i]);
    for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) atomicMax(out, m);
}

// ---- SC: hop distances from the roots
__global__ void sc_roots(const int *__restrict__ srp, const int *__restrict__ scol, int64_t n, int *__restrict__ dist,
                         int *__restrict__ frontier, int *__restrict__ count) {
    const int64_t u = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (u >= n) return;
    bool root = true;
    for (int j = srp[u]; j < srp[u + 1] && root; ++j) root = scol[j] >= (int)u;
    dist[u] = root ? 0 : -1;
    if (root) frontier[atomicAdd(count, 1)] = (int)u;
}

__global__ void sc_expand(const int *__restrict__ srp, const int *__restrict__ scol, const int *__restrict__ cur,
                          int cur_count, int *__restrict__ nxt, int *__restrict__ nxt_count, int *dist, int level) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < cur_count; i += stride) {
        const int u = cur[i];
        for (int j = srp[u]; j < srp[u + 1]; ++j) {
            const int v = scol[j];
            if (atomicCAS(dist + v, -1, level + 1) == -1) nxt[atomicAdd(nxt_count, 1)] = v;
        }
    }
}

// ---- PC_BAL
__global__ void oversized_flags(const int *__restrict__ colour, int64_t n, const int *__restrict__ size, double b,
                                unsigned char *__restrict__ flag) {
    const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (r < n) flag[r] = (double)size[colour[r]] > b;
}

__global__ void class_sizes(const int *__restrict__ colour, int64_t n, int *__restrict__ size) {
    const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (r < n) atomicAdd(size + colour[r], 1);
}

// One warp walks the candidate rows in ascending order (generate_color_perm_bal
// with one thread).  mark[c] == row + 1 means a neighbour of `row` has colour c.
__global__ void __launch_bounds__(32)
    balance_walk(const int *__restrict__ srp, const int *__restrict__ scol, const int *__restrict__ cand, int n_cand,
                 int *colour, const int *__restrict__ size0, int n_colours, double b) {
    extern __shared__ int sh[];
    int *size = sh, *mark = sh + n_colours;
    const int lane = threadIdx.x;
    for (int c = lane; c < n_colours; c += 32) {
        size[c] = size0[c];
        mark[c] = 0;
    }
    __syncwarp();
    for (int k = 0; k < n_cand; ++k) {
        const int row = cand[k];
        const int cur = colour[row];  // this row's own colour is only changed by this walk
        if ((double)size[cur] <= b) continue;  // uniform: size[] is shared and synchronised
        const int s = srp[row], e = srp[row + 1];
        for (int j = s + lane; j < e; j += 32) mark[colour[scol[j]]] = row + 1;
        __syncwarp();
        int spec = -1;
        for (int c0 = 0; c0 < n_colours && spec < 0; c0 += 32) {
            const int c = c0 + lane;
            const bool ok = c < n_colours && mark[c] != row + 1 && (double)size[c] < b;
            const unsigned bal = __ballot_sync(0xffffffffu, ok);
            if (bal) spec = c0 + __ffs(bal) - 1;
        }
        if (spec >= 0 && lane == 0) {
            size[cur] -= 1;
            colour[row] = spec;
            size[spec] += 1;
        }
        __syncwarp();
    }
}

// ---- sanity_check_perm
__global__ void colour_conflicts(const int *__restrict__ rp, const int *__restrict__ col, int64_t n,
                                 const int *__restrict__ colour, int *__restrict__ first_bad) {
    const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n) return;
    const int cr = colour[r];
    for (int j = rp[r]; j < rp[r + 1]; ++j) {
        const int c = col[j];
        if (c >= (int)r) continue;
        if (colour[c] == cr && cr != 0) {
            atomicMin(first_bad, (int)r);
            return;
        }
    }
}

// greedy colours by dependency levels (`order`/`lvl_ptr` group the nodes by level)
int colour_by_levels(const int *srp, const int *scol, int64_t n, const int *prio, const std::vector<int> &lvl_ptr,
                     const int *order, DevBuf &colour, cudaStream_t st) {
    colour.alloc(sizeof(int) * (n ? n : 1));
    if (n == 0) return 1;  // the reference returns ++max_color with max_color = 0
    const int L = (int)lvl_ptr.size() - 1;
    DevBuf dlp(sizeof(int) * (L + 1));
    SMAX_CUDA(cudaMemcpyAsync(dlp.p, lvl_ptr.data(), sizeof(int) * (L + 1), cudaMemcpyHostToDevice, st));
    int l = 0;
    while (l < L) {
        if (lvl_ptr[l + 1] - lvl_ptr[l] <= kSmallNodes) {
            int l1 = l;
            while (l1 < L && lvl_ptr[l1 + 1] - lvl_ptr[l1] <= kSmallNodes) ++l1;
            colour_small_levels<<<1, kSmallThreads, 0, st>>>(srp, scol, prio, dlp.as<int>(), order, l, l1,
                                                             colour.as<int>());
            l = l1;
        } else {
            const int a = lvl_ptr[l], b = lvl_ptr[l + 1];
            colour_level<<<ceil_div_u(b - a, 256), 256, 0, st>>>(srp, scol, prio, order, a, b, colour.as<int>());
            ++l;
        }
        SMAX_CUDA(cudaGetLastError());
    }
    DevBuf mx(sizeof(int));
    SMAX_CUDA(cudaMemsetAsync(mx.p, 0, sizeof(int), st));
    max_reduce<<<std::min<int64_t>(ceil_div_u(n, 256), sm_count() * 4), 256, 0, st>>>(colour.as<int>(), n, mx.as<int>());
    SMAX_CUDA(cudaGetLastError());
    int h = 0;
    SMAX_CUDA(cudaMemcpyAsync(&h, mx.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    SMAX_CUDA(cudaStreamSynchronize(st));
    return h + 1;
}

}  // namespace

int colour_pc(const int *srp, const int *scol, int64_t n, DevBuf &colour, cudaStream_t st) {
    DevBuf lvl, order;
    std::vector<int> lvl_ptr;
    const int nl = rs_levels(srp, scol, n, lvl, st);
    level_order(lvl.as<int>(), n, nl, order, lvl_ptr, st);
    if (n > 0 && lvl_ptr.back() != n) fail(SMAX_ERR_STATE, "colouring levels do not cover all rows");
    return colour_by_levels(srp, scol, n, nullptr, lvl_ptr, order.as<int>(), colour, st);
}

int colour_sc(const int *srp, const int *scol, int64_t n, DevBuf &colour, cudaStream_t st) {
    if (n == 0) {
        colour.alloc(sizeof(int));
        return 1;
    }
    // hop distances from the roots, one level per step
    DevBuf dist(sizeof(int) * n), f0(sizeof(int) * n), f1(sizeof(int) * n), cnt(sizeof(int) * 2);
    SMAX_CUDA(cudaMemsetAsync(cnt.p, 0, sizeof(int) * 2, st));
    sc_roots<<<ceil_div_u(n, 256), 256, 0, st>>>(srp, scol, n, dist.as<int>(), f0.as<int>(), cnt.as<int>());
    SMAX_CUDA(cudaGetLastError());
    int h = 0;
    SMAX_CUDA(cudaMemcpyAsync(&h, cnt.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    SMAX_CUDA(cudaStreamSynchronize(st));
    int *cur = f0.as<int>(), *nxt = f1.as<int>();
    int level = 0, reached = h;
    const int grid = 4 * sm_count();
    while (h > 0) {
        if (level > n) fail(SMAX_ERR_STATE, "breadth-first search did not terminate");
        SMAX_CUDA(cudaMemsetAsync(cnt.as<int>() + 1, 0, sizeof(int), st));
        sc_expand<<<grid, 256, 0, st>>>(srp, scol, cur, h, nxt, cnt.as<int>() + 1, dist.as<int>(), level);
        SMAX_CUDA(cudaGetLastError());
        SMAX_CUDA(cudaMemcpyAsync(&h, cnt.as<int>() + 1, sizeof(int), cudaMemcpyDeviceToHost, st));
        SMAX_CUDA(cudaStreamSynchronize(st));
        std::swap(cur, nxt);
        reached += h;
        ++level;
    }
    if (reached != n) fail(SMAX_ERR_STATE, "breadth-first search did not reach every row");
    // the queue order: roots ascending, then each level by first discoverer
    DevBuf lorder, queue, pos(sizeof(int) * n), lvl2, order2;
    std::vector<int> lvl_ptr, lvl_ptr2;
    level_order(dist.as<int>(), n, level, lorder, lvl_ptr, st);
    bfs_order(srp, scol, n, lvl_ptr, lorder.as<int>(), queue, st, true);
    inverse_perm(queue.as<int>(), n, pos.as<int>(), st);
    // greedy colouring in queue order
    const int nl = rs_levels(srp, scol, n, lvl2, st, false, pos.as<int>());
    level_order(lvl2.as<int>(), n, nl, order2, lvl_ptr2, st);
    if (lvl_ptr2.back() != n) fail(SMAX_ERR_STATE, "colouring levels do not cover all rows");
    return colour_by_levels(srp, scol, n, pos.as<int>(), lvl_ptr2, order2.as<int>(), colour, st);
}

int colour_balance(const int *srp, const int *scol, int64_t n, DevBuf &colour, int n_colours, cudaStream_t st) {
    if (n == 0) return n_colours;
    if (n_colours > kMaxBalanceColours)
        fail(SMAX_ERR_UNSUPPORTED, "PC_BAL handles at most " + std::to_string(kMaxBalanceColours) + " colours");
    const double b = (double)(n / n_colours);  // integer division, as the reference
    DevBuf size(sizeof(int) * n_colours), flag(n), cand(sizeof(int) * n), nc(sizeof(int));
    SMAX_CUDA(cudaMemsetAsync(size.p, 0, sizeof(int) * n_colours, st));
    class_sizes<<<ceil_div_u(n, 256), 256, 0, st>>>(colour.as<int>(), n, size.as<int>());
    oversized_flags<<<ceil_div_u(n, 256), 256, 0, st>>>(colour.as<int>(), n, size.as<int>(), b,
                                                        flag.as<unsigned char>());
    SMAX_CUDA(cudaGetLastError());
    thrust::counting_iterator<int> it(0);
    size_t tb = 0;
    SMAX_CUDA(cub::DeviceSelect::Flagged(nullptr, tb, it, flag.as<unsigned char>(), cand.as<int>(), nc.as<int>(),
                                         (int)n, st));
    DevBuf tmp(tb);
    SMAX_CUDA(cub::DeviceSelect::Flagged(tmp.p, tb, it, flag.as<unsigned char>(), cand.as<int>(), nc.as<int>(),
                                         (int)n, st));
    int h = 0;
    SMAX_CUDA(cudaMemcpyAsync(&h, nc.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    SMAX_CUDA(cudaStreamSynchronize(st));
    if (h > 0) {
        const size_t shm = sizeof(int) * 2 * (size_t)n_colours;
        SMAX_CUDA(cudaFuncSetAttribute(balance_walk, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shm));
        balance_walk<<<1, 32, shm, st>>>(srp, scol, cand.as<int>(), h, colour.as<int>(), size.as<int>(), n_colours,
                                         b);
        SMAX_CUDA(cudaGetLastError());
        SMAX_CUDA(cudaStreamSynchronize(st));
    }
    return n_colours;
}

bool colours_valid(const int *rp, const int *col, int64_t n, const int *colour, int64_t *first_bad_row,
                   cudaStream_t st) {
    if (first_bad_row) *first_bad_row = -1;
    if (n == 0) return true;
    DevBuf bad(sizeof(int));
    const int big = 0x7fffffff;
    SMAX_CUDA(cudaMemcpyAsync(bad.p, &big, sizeof(int), cudaMemcpyHostToDevice, st));
    colour_conflicts<<<ceil_div_u(n, 256), 256, 0, st>>>(rp, col, n, colour, bad.as<int>());
    SMAX_CUDA(cudaGetLastError());
    int h = big;
    SMAX_CUDA(cudaMemcpyAsync(&h, bad.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    SMAX_CUDA(cudaStreamSynchronize(st));
    if (h == big) return true;
    if (first_bad_row) *first_bad_row = h;
    return false;
}

}  // namespace smax
