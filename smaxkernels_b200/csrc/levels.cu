// levels.cu -- level sets, permutations and A+A^T on the GPU.
//
// Reference: src/utils/permutations.hpp.
//   * build_symmetric_crs (:236-392, the _parallel_adapted variant): row c of
//     A+A^T is A's row c as stored, then every r with c in row r, c != r, whose
//     own row c lacks r -- appended in ascending r (the order one OpenMP thread,
//     or any static schedule, produces).  GPU: a flag per entry (linear search
//     of the transposed row), a radix sort of the missing (c, r) pairs, a
//     per-row count, a scan and a fill.
//   * generate_perm_row_sweep (:394-414): lvl[r] = 1 + max lvl of the
//     neighbours c < r of the symmetric pattern.  GPU: Kahn's algorithm level
//     by level -- a node enters level l+1 when its last lower neighbour leaves
//     level l.  Frontiers of up to kSmallCap nodes are processed by a single CTA
//     that sweeps many levels per launch with __syncthreads between levels;
//     larger frontiers use one grid-wide launch per level.
//   * generate_perm_BFS (:416-483) with one thread: roots in ascending order;
//     a node v is queued while its last-dequeued lower neighbour w* is being
//     visited, in the order of w*'s symmetric row.  Hence the queue order of
//     level l+1 is the order of the keys (position of w*, first index of v in
//     w*'s row), which this file computes level by level (single CTA with a
//     shared-memory sort for small levels, a device radix sort otherwise).
//   * generate_perm (:485-584) for non-BFS types: stable sort of the identity
//     by level = radix sort of (level, row) keys; inv_perm; lvl_ptr by counting.
//   * apply_mat_perm (:820-861), apply_vec_perm (:863-874): gathers.
#include "levels.cuh"

#include <cub/block/block_radix_sort.cuh>
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>
#include <cub/device/device_select.cuh>

#include <vector>

namespace smax {

namespace {

constexpr int kSmallCap = 4096;    // frontier capacity of the single-CTA sweeps
constexpr int kSmallThreads = 1024;

// ------------------------------------------------------------ A + A^T ----
__global__ void sym_missing_flags(const int *__restrict__ rp, const int *__restrict__ col, int64_t n,
                                  unsigned char *__restrict__ miss) {
    const int64_t r = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (r >= n) return;
    for (int j = rp[r] + lane; j < rp[r + 1]; j += 32) {
        const int c = col[j];
        unsigned char m = 0;
        if (c != r && c >= 0 && c < n) {
            m = 1;
            for (int k = rp[c]; k < rp[c + 1]; ++k)
                if (col[k] == (int)r) { m = 0; break; }
        }
        miss[j] = m;
    }
}

// key = (c << 32) | r for every missing transpose r -> row c
__global__ void sym_missing_keys(const int *__restrict__ rp, const int *__restrict__ col, int64_t n,
                                 const unsigned char *__restrict__ miss, unsigned long long *__restrict__ keys) {
    const int64_t r = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (r >= n) return;
    for (int j = rp[r] + lane; j < rp[r + 1]; j += 32)
        keys[j] = miss[j] ? (((unsigned long long)(unsigned)col[j] << 32) | (unsigned)r) : ~0ull;
}

__global__ void sym_count(const unsigned long long *__restrict__ sorted, int64_t m, int *__restrict__ extra) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m) return;
    atomicAdd(extra + (int)(sorted[i] >> 32), 1);
}

__global__ void sym_rowlen(const int *__restrict__ rp, const int *__restrict__ extra, int64_t n,
                           int *__restrict__ len) {
    const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (r < n) len[r] = rp[r + 1] - rp[r] + extra[r];
}

__global__ void sym_fill(const int *__restrict__ rp, const int *__restrict__ col, int64_t n,
                         const int *__restrict__ srp, const unsigned long long *__restrict__ sorted,
                         const int *__restrict__ extra_off, int *__restrict__ scol) {
    const int64_t r = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (r >= n) return;
    const int own = rp[r + 1] - rp[r];
    for (int j = lane; j < own; j += 32) scol[srp[r] + j] = col[rp[r] + j];
    const int ne = srp[r + 1] - srp[r] - own;
    const int eo = extra_off[r];
    for (int j = lane; j < ne; j += 32) scol[srp[r] + own + j] = (int)(sorted[eo + j] & 0xffffffffull);
}

// ------------------------------------------------------------ RS levels ----
// deg[v] = number of entries v > u over all symmetric rows u, i.e. exactly
// the releases v receives in the sweep (duplicates counted on both sides)
// With rev, edges run from higher to lower rows (levels of an upper
// triangular dependency structure).
// With prio, "ahead" is a larger priority instead of a larger row index.
__device__ __forceinline__ bool ahead(int v, int u, bool rev, const int *prio) {
    if (prio) return prio[v] > prio[u];
    return rev ? v < u : v > u;
}

__global__ void incoming_degree(const int *__restrict__ srp, const int *__restrict__ scol, int64_t n,
                                int *__restrict__ deg, bool rev, const int *__restrict__ prio) {
    const int64_t u = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (u >= n) return;
    for (int j = srp[u]; j < srp[u + 1]; ++j) {
        const int v = scol[j];
        if (ahead(v, (int)u, rev, prio)) atomicAdd(deg + v, 1);
    }
}

__global__ void fill_int(int *__restrict__ a, int64_t n, int value) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) a[i] = value;
}

__global__ void roots_kernel(const int *__restrict__ deg, int64_t n, int *__restrict__ frontier,
                             int *__restrict__ count, int *__restrict__ lvl) {
    const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n || deg[r] != 0) return;
    lvl[r] = 0;
    frontier[atomicAdd(count, 1)] = (int)r;
}

// One level, grid-wide: every node of the frontier releases its upper
// neighbours; the last release of a node puts it into the next frontier.
__global__ void level_step(const int *__restrict__ srp, const int *__restrict__ scol, const int *__restrict__ cur,
                           const int *__restrict__ cur_count, int *__restrict__ nxt, int *__restrict__ nxt_count,
                           int *__restrict__ deg, int *__restrict__ lvl, int level, bool rev,
                           const int *__restrict__ prio) {
    const int cnt = *cur_count;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < cnt; i += stride) {
        const int u = cur[i];
        for (int j = srp[u]; j < srp[u + 1]; ++j) {
            const int v = scol[j];
            if (ahead(v, u, rev, prio) && atomicSub(deg + v, 1) == 1) {
                lvl[v] = level + 1;
                nxt[atomicAdd(nxt_count, 1)] = v;
            }
        }
    }
}

// Many levels in one CTA while the frontier fits in shared memory.  On exit
// frontier/count hold the frontier of level *level_io (possibly too large for
// the next small sweep), or count == 0 when all levels are done.
__global__ void __launch_bounds__(kSmallThreads) level_sweep_small(const int *__restrict__ srp,
                                                                   const int *__restrict__ scol,
                                                                   int *__restrict__ frontier,
                                                                   int *__restrict__ count, int *__restrict__ deg,
                                                                   int *__restrict__ lvl, int *__restrict__ level_io,
                                                                   bool rev, const int *__restrict__ prio) {
    __shared__ int buf[2][kSmallCap];
    __shared__ int cnt[2];
    __shared__ int overflow;
    const int tid = threadIdx.x;
    int level = *level_io;
    int c = *count;
    for (int i = tid; i < c; i += blockDim.x) buf[0][i] = frontier[i];
    if (tid == 0) { cnt[0] = c; overflow = 0; }
    __syncthreads();
    int cur = 0;
    while (true) {
        const int cc = cnt[cur];
        if (cc == 0) break;
        if (tid == 0) cnt[cur ^ 1] = 0;
        __syncthreads();
        for (int i = tid; i < cc; i += blockDim.x) {
            const int u = buf[cur][i];
            for (int j = srp[u]; j < srp[u + 1]; ++j) {
                const int v = scol[j];
                if (ahead(v, u, rev, prio) && atomicSub(deg + v, 1) == 1) {
                    lvl[v] = level + 1;
                    const int p = atomicAdd(&cnt[cur ^ 1], 1);
                    if (p < kSmallCap) buf[cur ^ 1][p] = v;
                    else frontier[p] = v;  // spills: kept in global memory for the grid-wide step
                }
            }
        }
        __syncthreads();
        const int nc = cnt[cur ^ 1];
        if (nc > kSmallCap) {
            // hand the (large) next frontier back to the grid-wide path
            for (int i = tid; i < kSmallCap; i += blockDim.x) frontier[i] = buf[cur ^ 1][i];
            if (tid == 0) { overflow = 1; *count = nc; *level_io = level + 1; }
            __syncthreads();
            return;
        }
        cur ^= 1;
        ++level;
    }
    if (tid == 0) { *count = 0; *level_io = level; }
}

// ------------------------------------------------------------ orderings ----
__global__ void level_keys(const int *__restrict__ lvl, int64_t n, unsigned long long *__restrict__ keys,
                           int *__restrict__ idx) {
    const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n) return;
    keys[r] = ((unsigned long long)(unsigned)lvl[r] << 32) | (unsigned long long)r;
    idx[r] = (int)r;
}

__global__ void level_counts(const int *__restrict__ lvl, int64_t n, int *__restrict__ cnt) {
    const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (r < n) atomicAdd(cnt + lvl[r], 1);
}

__global__ void inverse_kernel(const int *__restrict__ perm, int64_t n, int *__restrict__ inv) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) inv[perm[i]] = (int)i;
}

// BFS key of v: (position of its last-dequeued lower neighbour w*, first index
// of v in w*'s symmetric row).  pos[] holds the final positions of all nodes
// of earlier levels; it is written by the same kernel, so it is read through
// L2 (__ldcg), never through the non-coherent read-only path.
// With First, w* is instead v's first-dequeued neighbour of any index among
// the nodes placed before this level (pos < placed_end; unplaced nodes hold
// INT_MAX): the queue order of a FIFO breadth-first search from a root set.
template <bool First>
__device__ __forceinline__ unsigned long long bfs_key(const int *__restrict__ srp, const int *__restrict__ scol,
                                                      const int *pos, int v, int placed_end) {
    int best = First ? 0x7fffffff : -1, wstar = -1;
    for (int j = srp[v]; j < srp[v + 1]; ++j) {
        const int w = scol[j];
        if constexpr (First) {
            const int p = __ldcg(pos + w);
            if (p < placed_end && p < best) { best = p; wstar = w; }
        } else if (w < v) {
            const int p = __ldcg(pos + w);
            if (p > best) { best = p; wstar = w; }
        }
    }
    if (wstar < 0) return ~0ull;  // no lower neighbour: not reachable for levels >= 1
    int k = 0;
    for (int j = srp[wstar]; j < srp[wstar + 1]; ++j)
        if (scol[j] == v) { k = j - srp[wstar]; break; }
    return ((unsigned long long)(unsigned)best << 32) | (unsigned)k;
}

// Small levels [l0, l1): one CTA; each level's nodes (contiguous in `order`,
// the (level, row)-sorted nodes) are sorted by their BFS keys in shared memory.
template <bool First>
__global__ void __launch_bounds__(kSmallThreads) bfs_small_levels(const int *__restrict__ srp,
                                                                  const int *__restrict__ scol,
                                                                  const int *__restrict__ lvl_ptr,
                                                                  const int *__restrict__ order, int l0, int l1,
                                                                  int *pos, int *__restrict__ perm) {
    using Sort = cub::BlockRadixSort<unsigned long long, kSmallThreads, kSmallCap / kSmallThreads, int>;
    __shared__ typename Sort::TempStorage tmp;
    constexpr int IPT = kSmallCap / kSmallThreads;
    for (int l = l0; l < l1; ++l) {
        const int a = lvl_ptr[l], b = lvl_ptr[l + 1];
        const int m = b - a;
        unsigned long long keys[IPT];
        int vals[IPT];
#pragma unroll
        for (int i = 0; i < IPT; ++i) {
            const int e = threadIdx.x * IPT + i;  // blocked arrangement
            if (e < m) {
                const int v = order[a + e];
                keys[i] = bfs_key<First>(srp, scol, pos, v, a);
                vals[i] = v;
            } else {
                keys[i] = ~0ull;
                vals[i] = -1;
            }
        }
        Sort(tmp).Sort(keys, vals);
#pragma unroll
        for (int i = 0; i < IPT; ++i) {
            const int e = threadIdx.x * IPT + i;
            if (e < m) {
                perm[a + e] = vals[i];
                pos[vals[i]] = a + e;
            }
        }
        __syncthreads();  // positions of level l are visible before level l+1 reads them
    }
}

template <bool First>
__global__ void bfs_keys_level(const int *__restrict__ srp, const int *__restrict__ scol,
                               const int *__restrict__ order, int a, int m, const int *pos,
                               unsigned long long *__restrict__ keys, int *__restrict__ vals) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m) return;
    const int v = order[a + i];
    keys[i] = bfs_key<First>(srp, scol, pos, v, a);
    vals[i] = v;
}

__global__ void bfs_place_level(const int *__restrict__ sorted_vals, int a, int m, int *__restrict__ pos,
                                int *__restrict__ perm) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m) return;
    const int v = sorted_vals[i];
    perm[a + i] = v;
    pos[v] = a + i;
}

__global__ void set_pos_kernel(const int *__restrict__ perm, int64_t a, int64_t b, int *__restrict__ pos) {
    const int64_t i = a + (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < b) pos[perm[i]] = (int)i;
}

// ------------------------------------------------------------ apply perm ----
__global__ void perm_rowlen(const int *__restrict__ rp, const int *__restrict__ perm, int64_t n,
                            int *__restrict__ len) {
    const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (r < n) len[r] = rp[perm[r] + 1] - rp[perm[r]];
}

template <typename VT>
__global__ void perm_fill(const int *__restrict__ rp, const int *__restrict__ col, const VT *__restrict__ val,
                          const int *__restrict__ prp, const int *__restrict__ perm, const int *__restrict__ inv,
                          int64_t n, int *__restrict__ pcol, VT *__restrict__ pval) {
    const int64_t r = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (r >= n) return;
    const int o = rp[perm[r]];
    const int len = prp[r + 1] - prp[r];
    for (int j = lane; j < len; j += 32) {
        pcol[prp[r] + j] = inv[col[o + j]];
        pval[prp[r] + j] = val[o + j];
    }
}

template <typename VT>
__global__ void vec_perm_kernel(const VT *__restrict__ v, const int *__restrict__ perm, int64_t n,
                                VT *__restrict__ out) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = v[perm[i]];
}

// exclusive scan of n ints into out[0..n] (out[n] = total) with CUB
void exclusive_scan_total(const int *in, int64_t n, int *out, cudaStream_t st) {
    SMAX_CUDA(cudaMemsetAsync(out, 0, sizeof(int), st));
    if (n == 0) return;
    size_t tb = 0;
    SMAX_CUDA(cub::DeviceScan::InclusiveSum(nullptr, tb, in, out + 1, (int)n, st));
    DevBuf tmp(tb);
    SMAX_CUDA(cub::DeviceScan::InclusiveSum(tmp.p, tb, in, out + 1, (int)n, st));
}

}  // namespace

void build_symmetric(const DevCRS &a, DevBuf &srp, DevBuf &scol, int64_t &sym_nnz, cudaStream_t st) {
    const int64_t n = a.n_rows, nnz = a.nnz;
    srp.alloc(sizeof(int) * (n + 1));
    if (n == 0) {
        SMAX_CUDA(cudaMemsetAsync(srp.p, 0, sizeof(int), st));
        scol.alloc(sizeof(int));
        sym_nnz = 0;
        return;
    }
    DevBuf miss(nnz ? nnz : 1), keys(sizeof(unsigned long long) * (nnz ? nnz : 1)),
        sorted(sizeof(unsigned long long) * (nnz ? nnz : 1));
    DevBuf extra(sizeof(int) * n), len(sizeof(int) * n), eoff(sizeof(int) * (n + 1));
    SMAX_CUDA(cudaMemsetAsync(extra.p, 0, sizeof(int) * n, st));
    int64_t m = 0;
    if (nnz > 0) {
        const unsigned g = ceil_div_u((uint64_t)n * 32, 256);
        sym_missing_flags<<<g, 256, 0, st>>>(a.rp(), a.ci(), n, miss.as<unsigned char>());
        sym_missing_keys<<<g, 256, 0, st>>>(a.rp(), a.ci(), n, miss.as<unsigned char>(),
                                            keys.as<unsigned long long>());
        SMAX_CUDA(cudaGetLastError());
        size_t tb = 0;
        SMAX_CUDA(cub::DeviceRadixSort::SortKeys(nullptr, tb, keys.as<unsigned long long>(),
                                                 sorted.as<unsigned long long>(), (int)nnz, 0, 64, st));
        DevBuf tmp(tb);
        SMAX_CUDA(cub::DeviceRadixSort::SortKeys(tmp.p, tb, keys.as<unsigned long long>(),
                                                 sorted.as<unsigned long long>(), (int)nnz, 0, 64, st));
        // missing pairs are the keys below ~0: count them
        DevBuf nm(sizeof(int));
        DevBuf flags(nnz);
        size_t tb2 = 0;
        SMAX_CUDA(cub::DeviceSelect::Flagged(nullptr, tb2, miss.as<unsigned char>(), miss.as<unsigned char>(),
                                             flags.as<unsigned char>(), nm.as<int>(), (int)nnz, st));
        DevBuf tmp2(tb2);
        SMAX_CUDA(cub::DeviceSelect::Flagged(tmp2.p, tb2, miss.as<unsigned char>(), miss.as<unsigned char>(),
                                             flags.as<unsigned char>(), nm.as<int>(), (int)nnz, st));
        int hm = 0;
        SMAX_CUDA(cudaMemcpyAsync(&hm, nm.p, sizeof(int), cudaMemcpyDeviceToHost, st));
        SMAX_CUDA(cudaStreamSynchronize(st));
        m = hm;
        if (m > 0) {
            sym_count<<<ceil_div_u(m, 256), 256, 0, st>>>(sorted.as<unsigned long long>(), m, extra.as<int>());
            SMAX_CUDA(cudaGetLastError());
        }
    }
    sym_rowlen<<<ceil_div_u(n, 256), 256, 0, st>>>(a.rp(), extra.as<int>(), n, len.as<int>());
    SMAX_CUDA(cudaGetLastError());
    exclusive_scan_total(len.as<int>(), n, srp.as<int>(), st);
    exclusive_scan_total(extra.as<int>(), n, eoff.as<int>(), st);
    int total = 0;
    SMAX_CUDA(cudaMemcpyAsync(&total, srp.as<int>() + n, sizeof(int), cudaMemcpyDeviceToHost, st));
    SMAX_CUDA(cudaStreamSynchronize(st));
    sym_nnz = total;
    scol.alloc(sizeof(int) * (total ? total : 1));
    sym_fill<<<ceil_div_u((uint64_t)n * 32, 256), 256, 0, st>>>(a.rp(), a.ci(), n, srp.as<int>(),
                                                                sorted.as<unsigned long long>(), eoff.as<int>(),
                                                                scol.as<int>());
    SMAX_CUDA(cudaGetLastError());
    SMAX_CUDA(cudaStreamSynchronize(st));
}

int rs_levels(const int *srp, const int *scol, int64_t n, DevBuf &lvl, cudaStream_t st, bool rev, const int *prio) {
    lvl.alloc(sizeof(int) * (n ? n : 1));
    if (n == 0) return 1;  // the reference reports one level for an empty matrix
    DevBuf deg(sizeof(int) * n), fr0(sizeof(int) * n), fr1(sizeof(int) * n), cnts(sizeof(int) * 4);
    const unsigned g = ceil_div_u(n, 256);
    SMAX_CUDA(cudaMemsetAsync(deg.p, 0, sizeof(int) * n, st));
    incoming_degree<<<g, 256, 0, st>>>(srp, scol, n, deg.as<int>(), rev, prio);
    fill_int<<<g, 256, 0, st>>>(lvl.as<int>(), n, -1);
    SMAX_CUDA(cudaMemsetAsync(cnts.p, 0, sizeof(int) * 4, st));
    roots_kernel<<<g, 256, 0, st>>>(deg.as<int>(), n, fr0.as<int>(), cnts.as<int>(), lvl.as<int>());
    SMAX_CUDA(cudaGetLastError());
    int *cnt = cnts.as<int>();  // cnt[0], cnt[1]: frontier sizes; cnt[2]: level
    int *cur = fr0.as<int>(), *nxt = fr1.as<int>();
    int *ccur = cnt, *cnxt = cnt + 1;
    int level = 0;
    const int grid = 4 * sm_count();
    int h[2] = {0, 0};
    SMAX_CUDA(cudaMemcpyAsync(h, ccur, sizeof(int), cudaMemcpyDeviceToHost, st));
    SMAX_CUDA(cudaStreamSynchronize(st));
    int64_t guard = 0;
    while (h[0] > 0) {
        if (++guard > 4 * n + 8) fail(SMAX_ERR_STATE, "level sweep did not terminate");
        if (h[0] <= kSmallCap) {
            SMAX_CUDA(cudaMemcpyAsync(cnt + 2, &level, sizeof(int), cudaMemcpyHostToDevice, st));
            level_sweep_small<<<1, kSmallThreads, 0, st>>>(srp, scol, cur, ccur, deg.as<int>(), lvl.as<int>(),
                                                           cnt + 2, rev, prio);
            SMAX_CUDA(cudaGetLastError());
            SMAX_CUDA(cudaMemcpyAsync(h, ccur, sizeof(int), cudaMemcpyDeviceToHost, st));
            SMAX_CUDA(cudaMemcpyAsync(h + 1, cnt + 2, sizeof(int), cudaMemcpyDeviceToHost, st));
            SMAX_CUDA(cudaStreamSynchronize(st));
            level = h[1];
        } else {
            SMAX_CUDA(cudaMemsetAsync(cnxt, 0, sizeof(int), st));
            level_step<<<grid, 256, 0, st>>>(srp, scol, cur, ccur, nxt, cnxt, deg.as<int>(), lvl.as<int>(), level,
                                             rev, prio);
            SMAX_CUDA(cudaGetLastError());
            std::swap(cur, nxt);
            std::swap(ccur, cnxt);
            ++level;
            SMAX_CUDA(cudaMemcpyAsync(h, ccur, sizeof(int), cudaMemcpyDeviceToHost, st));
            SMAX_CUDA(cudaStreamSynchronize(st));
        }
    }
    // levels 0..level-1 were produced; a node never reached (only possible on
    // malformed input) would keep lvl == -1
    return level;
}

void level_order(const int *lvl, int64_t n, int n_levels, DevBuf &order, std::vector<int> &lvl_ptr, cudaStream_t st) {
    order.alloc(sizeof(int) * (n ? n : 1));
    lvl_ptr.assign((size_t)n_levels + 1, 0);
    if (n == 0) return;
    DevBuf keys(sizeof(unsigned long long) * n), skeys(sizeof(unsigned long long) * n), idx(sizeof(int) * n);
    level_keys<<<ceil_div_u(n, 256), 256, 0, st>>>(lvl, n, keys.as<unsigned long long>(), idx.as<int>());
    SMAX_CUDA(cudaGetLastError());
    size_t tb = 0;
    SMAX_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tb, keys.as<unsigned long long>(),
                                              skeys.as<unsigned long long>(), idx.as<int>(), order.as<int>(), (int)n,
                                              0, 64, st));
    DevBuf tmp(tb);
    SMAX_CUDA(cub::DeviceRadixSort::SortPairs(tmp.p, tb, keys.as<unsigned long long>(),
                                              skeys.as<unsigned long long>(), idx.as<int>(), order.as<int>(), (int)n,
                                              0, 64, st));
    DevBuf cnt(sizeof(int) * (n_levels + 1)), ptr(sizeof(int) * (n_levels + 1));
    SMAX_CUDA(cudaMemsetAsync(cnt.p, 0, sizeof(int) * (n_levels + 1), st));
    level_counts<<<ceil_div_u(n, 256), 256, 0, st>>>(lvl, n, cnt.as<int>());
    SMAX_CUDA(cudaGetLastError());
    exclusive_scan_total(cnt.as<int>(), n_levels, ptr.as<int>(), st);
    SMAX_CUDA(cudaMemcpyAsync(lvl_ptr.data(), ptr.p, sizeof(int) * (n_levels + 1), cudaMemcpyDeviceToHost, st));
    SMAX_CUDA(cudaStreamSynchronize(st));
}

void bfs_order(const int *srp, const int *scol, int64_t n, const std::vector<int> &lvl_ptr, const int *order,
               DevBuf &perm, cudaStream_t st, bool first_discoverer) {
    perm.alloc(sizeof(int) * (n ? n : 1));
    if (n == 0) return;
    const int L = (int)lvl_ptr.size() - 1;
    DevBuf pos(sizeof(int) * n), dlp(sizeof(int) * (L + 1));
    if (first_discoverer) {
        fill_int<<<ceil_div_u(n, 256), 256, 0, st>>>(pos.as<int>(), n, 0x7fffffff);
        SMAX_CUDA(cudaGetLastError());
    }
    SMAX_CUDA(cudaMemcpyAsync(dlp.p, lvl_ptr.data(), sizeof(int) * (L + 1), cudaMemcpyHostToDevice, st));
    // level 0: the roots, queued in ascending order == (level, row) order
    const int m0 = lvl_ptr[1] - lvl_ptr[0];
    SMAX_CUDA(cudaMemcpyAsync(perm.p, order, sizeof(int) * m0, cudaMemcpyDeviceToDevice, st));
    set_pos_kernel<<<ceil_div_u(m0 > 0 ? m0 : 1, 256), 256, 0, st>>>(perm.as<int>(), 0, m0, pos.as<int>());
    SMAX_CUDA(cudaGetLastError());
    DevBuf kin, kout, vin, vout, tmp;
    size_t tmp_bytes = 0;
    int l = 1;
    while (l < L) {
        if (lvl_ptr[l + 1] - lvl_ptr[l] <= kSmallCap) {
            int l1 = l;
            while (l1 < L && lvl_ptr[l1 + 1] - lvl_ptr[l1] <= kSmallCap) ++l1;
            if (first_discoverer)
                bfs_small_levels<true><<<1, kSmallThreads, 0, st>>>(srp, scol, dlp.as<int>(), order, l, l1,
                                                                    pos.as<int>(), perm.as<int>());
            else
                bfs_small_levels<false><<<1, kSmallThreads, 0, st>>>(srp, scol, dlp.as<int>(), order, l, l1,
                                                                     pos.as<int>(), perm.as<int>());
            SMAX_CUDA(cudaGetLastError());
            l = l1;
        } else {
            const int a = lvl_ptr[l], m = lvl_ptr[l + 1] - a;
            kin.ensure(sizeof(unsigned long long) * m);
            kout.ensure(sizeof(unsigned long long) * m);
            vin.ensure(sizeof(int) * m);
            vout.ensure(sizeof(int) * m);
            if (first_discoverer)
                bfs_keys_level<true><<<ceil_div_u(m, 256), 256, 0, st>>>(srp, scol, order, a, m, pos.as<int>(),
                                                                         kin.as<unsigned long long>(), vin.as<int>());
            else
                bfs_keys_level<false><<<ceil_div_u(m, 256), 256, 0, st>>>(srp, scol, order, a, m, pos.as<int>(),
                                                                          kin.as<unsigned long long>(), vin.as<int>());
            SMAX_CUDA(cudaGetLastError());
            size_t tb = 0;
            SMAX_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tb, kin.as<unsigned long long>(),
                                                      kout.as<unsigned long long>(), vin.as<int>(), vout.as<int>(), m,
                                                      0, 64, st));
            if (tb > tmp_bytes) {
                tmp.alloc(tb);
                tmp_bytes = tb;
            }
            SMAX_CUDA(cub::DeviceRadixSort::SortPairs(tmp.p, tb, kin.as<unsigned long long>(),
                                                      kout.as<unsigned long long>(), vin.as<int>(), vout.as<int>(), m,
                                                      0, 64, st));
            bfs_place_level<<<ceil_div_u(m, 256), 256, 0, st>>>(vout.as<int>(), a, m, pos.as<int>(), perm.as<int>());
            SMAX_CUDA(cudaGetLastError());
            ++l;
        }
    }
    SMAX_CUDA(cudaStreamSynchronize(st));
}

void inverse_perm(const int *perm, int64_t n, int *inv, cudaStream_t st) {
    if (n == 0) return;
    inverse_kernel<<<ceil_div_u(n, 256), 256, 0, st>>>(perm, n, inv);
    SMAX_CUDA(cudaGetLastError());
}

void apply_mat_perm(const DevCRS &a, const int *perm, const int *inv, int vbytes, DevCRS &out, cudaStream_t st) {
    const int64_t n = a.n_rows;
    out.n_rows = n;
    out.n_cols = a.n_cols;
    out.nnz = a.nnz;
    out.row_ptr.alloc(sizeof(int) * (n + 1));
    out.col.alloc(sizeof(int) * (a.nnz ? a.nnz : 1));
    out.val.alloc((size_t)vbytes * (a.nnz ? a.nnz : 1));
    if (n == 0) {
        SMAX_CUDA(cudaMemsetAsync(out.row_ptr.p, 0, sizeof(int), st));
        return;
    }
    DevBuf len(sizeof(int) * n);
    perm_rowlen<<<ceil_div_u(n, 256), 256, 0, st>>>(a.rp(), perm, n, len.as<int>());
    SMAX_CUDA(cudaGetLastError());
    exclusive_scan_total(len.as<int>(), n, out.row_ptr.as<int>(), st);
    const unsigned g = ceil_div_u((uint64_t)n * 32, 256);
    if (vbytes == 8)
        perm_fill<double><<<g, 256, 0, st>>>(a.rp(), a.ci(), a.val.as<double>(), out.row_ptr.as<int>(), perm, inv, n,
                                             out.col.as<int>(), out.val.as<double>());
    else
        perm_fill<float><<<g, 256, 0, st>>>(a.rp(), a.ci(), a.val.as<float>(), out.row_ptr.as<int>(), perm, inv, n,
                                            out.col.as<int>(), out.val.as<float>());
    SMAX_CUDA(cudaGetLastError());
}

void apply_vec_perm(const void *vec, const int *perm, int64_t n, int vbytes, void *out, cudaStream_t st) {
    if (n == 0) return;
    if (vbytes == 8)
        vec_perm_kernel<double><<<ceil_div_u(n, 256), 256, 0, st>>>(static_cast<const double *>(vec), perm, n,
                                                                    static_cast<double *>(out));
    else
        vec_perm_kernel<float><<<ceil_div_u(n, 256), 256, 0, st>>>(static_cast<const float *>(vec), perm, n,
                                                                   static_cast<float *>(out));
    SMAX_CUDA(cudaGetLastError());
}

}  // namespace smax
