// spgemm.cu -- Gustavson SpGEMM C = A*B on sm_100a.
//
// Reference semantics (src/kernels/spgemm/spgemm_cpu/): padded_symbolic_phase
// (symbolic_phase_impl.hpp:9-177) stores each row's distinct columns of B in
// FIRST-TOUCH order -- the order in which the products (j over A's row, k over
// B's row col[j]) first reach them; basic_numerical_phase
// (numerical_phase_impl.hpp:9-91) accumulates every product in that (j, k)
// order.  C_n_rows = A_n_rows, C_n_cols = B_n_cols.
//
// Design.  When every row of B has increasing columns, a row of A with at most
// 8 entries and 64 products takes the merge path: one thread merges the row's
// B lists in registers (no table; see gustavson_merge).  If every row of A
// qualifies, C is written directly by a counting pass and a writing pass.
// Other rows take one fused hash pass, binned by their product count P_i:
//   * P_i <= 64:    a team of 8 lanes, hash table in shared memory (128 slots),
//                   persistent teams that reset only the slots a row used;
//   * P_i <= 256:   one warp, hash table in shared memory (512 slots);
//   * P_i <= 4096:  one CTA, hash table in shared memory (8192 slots);
//   * larger:       one CTA, hash table in a global workspace (2*P_i slots).
// The row's products are visited B-row by B-row in the reference's order; the
// columns of one B row are distinct, so the lanes of one step never collide
// and every table slot accumulates its products in (j, k) order --
// deterministic, and the same summation order as the reference.  A column's
// slot records the product index p of its first touch; since these indices
// are distinct, posmap[p] = slot followed by an ordered compaction of posmap
// yields the columns in first-touch order without a comparison sort.  Each row
// writes its columns/values at its product offset (an upper bound, as the
// reference's padded buffer), then a scan of the counts gives C's row_ptr and
// a compaction pass packs C_col / C_val.
#include "spgemm.cuh"

#include <cub/device/device_scan.cuh>

#include <algorithm>

namespace smax {

namespace {

constexpr int kSmallP = 64, kSmallTS = 128;    // small-row path: products, table slots
constexpr int kSmallTeam = 8;                  // lanes per row of the small-row path
constexpr int kSmallWarps = 4;                 // warps per CTA: 16 teams, 1.8 KB of tables each
constexpr int kWarpP = 256, kWarpTS = 512;     // warp path
constexpr int kCtaP = 4096, kCtaTS = 8192;     // CTA path
constexpr int kCtaThreads = 512;
constexpr int kWarpsPerCta = 4;
constexpr int kMergeLists = 8;                 // merge path: at most this many entries in the row of A
constexpr int kBins = 5;                       // small (hash), warp, CTA, global, merge
constexpr int kMergeWriteThreads = 128;        // direct write pass: 4 warps, each staging its rows in shared memory

__device__ __forceinline__ unsigned hash_col(int c) { return (unsigned)c * 0x9E3779B1u; }

constexpr int kRowGroup = 8;  // lanes per row of the per-row helper passes (short rows)

unsigned grid_cap(int64_t items) {  // a grid-stride launch of 256-thread blocks, at most 8 per SM
    const int64_t want = (items + 255) / 256, cap = 8ll * sm_count();
    return (unsigned)(want < 1 ? 1 : (want < cap ? want : cap));
}

// product count of every row of A (kRowGroup lanes per row)
__global__ void row_products(const int *__restrict__ arp, const int *__restrict__ acol, const int *__restrict__ brp,
                             int64_t n, long long *__restrict__ P) {
    const int64_t i = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) / kRowGroup;
    const int lane = threadIdx.x % kRowGroup;
    long long s = 0;
    if (i < n)
        for (int j = arp[i] + lane; j < arp[i + 1]; j += kRowGroup) {
            const int c = acol[j];
            s += brp[c + 1] - brp[c];
        }
#pragma unroll
    for (int o = kRowGroup / 2; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (i < n && lane == 0) P[i] = s;
}

// b_sorted = 1 unless some row of B has columns that do not strictly increase
__global__ void b_sorted_kernel(const int *__restrict__ brp, const int *__restrict__ bcol, int64_t n,
                                int *__restrict__ b_sorted) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < n; r += stride)
        for (int j = brp[r] + 1; j < brp[r + 1]; ++j)
            if (bcol[j] <= bcol[j - 1]) {
                atomicAnd(b_sorted, 0);
                return;
            }
}

// rows into five lists: the merge path (B's rows sorted, at most kMergeLists
// entries in the row of A and kSmallP products), then by product count the
// small-row, warp, CTA and global hash paths; the order inside a list is
// irrelevant (rows are independent)
__global__ void bin_rows(const long long *__restrict__ P, const int *__restrict__ arp, int64_t n,
                         const int *__restrict__ b_sorted, int *__restrict__ lists, int *counts) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const bool valid = i < n;
    const long long p = valid ? P[i] : 0;
    const bool merge = valid && *b_sorted && p <= kSmallP && arp[i + 1] - arp[i] <= kMergeLists;
    const int bin = merge ? 4 : (p <= kSmallP ? 0 : (p <= kWarpP ? 1 : (p <= kCtaP ? 2 : 3)));
    const unsigned active = __ballot_sync(0xffffffffu, valid);
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int b = 0; b < kBins; ++b) {
        const unsigned mask = __ballot_sync(0xffffffffu, valid && bin == b) & active;
        if (!mask) continue;
        const int leader = __ffs(mask) - 1;
        int base = 0;
        if (lane == leader) base = atomicAdd(counts + b, __popc(mask));
        base = __shfl_sync(0xffffffffu, base, leader);
        if (valid && bin == b) lists[(int64_t)b * n + base + __popc(mask & ((1u << lane) - 1u))] = (int)i;
    }
}

// The body shared by all three paths: a team of `tsize` threads (`t` its
// rank) fills a table of `TS` slots for row i.  sync() orders the steps.
template <typename VT, typename Sync>
__device__ __forceinline__ void gustavson_row(int i, int t, int tsize, const int *__restrict__ arp,
                                              const int *__restrict__ acol, const VT *__restrict__ aval,
                                              const int *__restrict__ brp, const int *__restrict__ bcol,
                                              const VT *__restrict__ bval, int *keys, int *first, VT *vals,
                                              int *posmap, unsigned TS, long long P, long long out_off,
                                              int *__restrict__ pcol, VT *__restrict__ pval, int *__restrict__ count,
                                              Sync sync) {
    for (unsigned h = t; h < TS; h += tsize) {
        keys[h] = -1;
        vals[h] = VT(0);
    }
    for (long long q = t; q < P; q += tsize) posmap[q] = -1;
    sync();
    long long base = 0;  // product index of the first product of the current B row
    for (int j = arp[i]; j < arp[i + 1]; ++j) {
        const int c = acol[j];
        const VT av = aval[j];
        const int bs = brp[c], be = brp[c + 1];
        for (int k = bs + t; k < be; k += tsize) {
            const int col = bcol[k];
            const VT prod = av * bval[k];
            unsigned h = hash_col(col) & (TS - 1);
            while (true) {
                const int old = atomicCAS(keys + h, -1, col);
                if (old == -1) {
                    first[h] = (int)(base + (k - bs));
                    break;
                }
                if (old == col) break;
                h = (h + 1) & (TS - 1);
            }
            vals[h] += prod;  // one product per slot per step: the (j, k) order
        }
        base += be - bs;
        sync();
    }
    for (unsigned h = t; h < TS; h += tsize)
        if (keys[h] != -1) posmap[first[h]] = (int)h;
    sync();
    // ordered compaction of posmap: entries in first-touch order
    __shared__ int team_total[kCtaThreads / 32];
    int written = 0;
    for (long long q0 = 0; q0 < P; q0 += tsize) {
        const long long q = q0 + t;
        const int h = q < P ? posmap[q] : -1;
        const int take = h >= 0;
        // team-wide exclusive scan of `take` (warp ballots, then warps in
        // order); a team smaller than a warp uses only its own lanes' bits
        const int lane = (int)(threadIdx.x & 31), warp = t >> 5;
        const unsigned tmask =
            tsize >= 32 ? 0xffffffffu : (((1u << tsize) - 1u) << ((unsigned)lane & ~(unsigned)(tsize - 1)));
        const unsigned bal = __ballot_sync(tmask, take) & tmask;
        const int before_in_warp = __popc(bal & ((1u << lane) - 1u));
        int before = before_in_warp, total = __popc(bal);
        if (tsize > 32) {
            if (lane == 0) team_total[warp] = total;
            sync();
            before = before_in_warp;
            total = 0;
            for (int w = 0; w < tsize / 32; ++w) {
                if (w < warp) before += team_total[w];
                total += team_total[w];
            }
            sync();
        }
        if (take) {
            pcol[out_off + written + before] = keys[h];
            pval[out_off + written + before] = vals[h];
        }
        written += total;
    }
    if (t == 0) count[i] = written;
}

// the lanes of one team inside a warp (the whole warp for a team of 32)
struct GroupSync {
    unsigned mask;
    __device__ void operator()() const { __syncwarp(mask); }
};
struct CtaSync {
    __device__ void operator()() const { __syncthreads(); }
};

// A team of G lanes (G <= 32, a power of two) per row of at most WP products,
// with a WTS-slot table (load at most 1/2); WARPS warps per CTA, 32 / G rows
// per warp.  Small teams suit rows whose B rows are short: a team covers one
// B row per step of the product loop.
template <typename VT, int WP, int WTS, int WARPS, int G>
__global__ void __launch_bounds__(WARPS * 32) gustavson_warp(
    const int *__restrict__ rows, int n_rows_bin, const long long *__restrict__ P, const long long *__restrict__ Poff,
    const int *__restrict__ arp, const int *__restrict__ acol, const VT *__restrict__ aval,
    const int *__restrict__ brp, const int *__restrict__ bcol, const VT *__restrict__ bval, int *__restrict__ pcol,
    VT *__restrict__ pval, int *__restrict__ count) {
    constexpr int TEAMS = WARPS * 32 / G;
    __shared__ int keys[TEAMS][WTS];
    __shared__ int first[TEAMS][WTS];
    __shared__ VT vals[TEAMS][WTS];
    __shared__ int posmap[TEAMS][WP];
    const int g = threadIdx.x / G;
    const int64_t r = (int64_t)blockIdx.x * TEAMS + g;
    if (r >= n_rows_bin) return;  // uniform per team; teams never touch CTA barriers
    const int i = rows[r];
    const unsigned mask = G == 32 ? 0xffffffffu : (((1u << G) - 1u) << ((threadIdx.x & 31) & ~(unsigned)(G - 1)));
    gustavson_row<VT>(i, (int)(threadIdx.x % G), G, arp, acol, aval, brp, bcol, bval, keys[g], first[g], vals[g],
                      posmap[g], WTS, P[i], Poff[i], pcol, pval, count, GroupSync{mask});
}

// The small-row path as persistent teams of G lanes: a team keeps its WTS-slot
// table across the rows it takes (rows r, r + teams in the grid, ...), clears
// it once, records the slots a row inserts, builds the first-touch map from
// that list and resets only those slots afterwards -- a row of ~25 distinct
// columns touches ~25 slots instead of clearing and scanning all WTS.  The
// steps, the first-touch bookkeeping and the summation order are those of
// gustavson_row.  Product indices (< WP <= 255) and slots (< WTS <= 128) are
// stored in bytes.
template <typename VT, int WP, int WTS, int WARPS, int G>
__global__ void __launch_bounds__(WARPS * 32) gustavson_small(
    const int *__restrict__ rows, int n_rows_bin, const long long *__restrict__ P, const long long *__restrict__ Poff,
    const int *__restrict__ arp, const int *__restrict__ acol, const VT *__restrict__ aval,
    const int *__restrict__ brp, const int *__restrict__ bcol, const VT *__restrict__ bval, int *__restrict__ pcol,
    VT *__restrict__ pval, int *__restrict__ count) {
    static_assert(WP <= 255 && WTS <= 128 && (WTS & (WTS - 1)) == 0, "byte-sized product indices and slots");
    constexpr int TEAMS = WARPS * 32 / G;
    __shared__ int keys[TEAMS][WTS];
    __shared__ VT vals[TEAMS][WTS];
    __shared__ unsigned char first[TEAMS][WTS];
    __shared__ signed char posmap[TEAMS][WP];
    __shared__ unsigned char used[TEAMS][WP];
    __shared__ int nused[TEAMS];
    const int g = threadIdx.x / G, t = (int)(threadIdx.x % G);
    const int lane = (int)(threadIdx.x & 31);
    const unsigned mask = G == 32 ? 0xffffffffu : (((1u << G) - 1u) << ((unsigned)lane & ~(unsigned)(G - 1)));
    for (int h = t; h < WTS; h += G) {
        keys[g][h] = -1;
        vals[g][h] = VT(0);
    }
    if (t == 0) nused[g] = 0;
    __syncwarp(mask);
    const int64_t stride = (int64_t)gridDim.x * TEAMS;
    for (int64_t r = (int64_t)blockIdx.x * TEAMS + g; r < n_rows_bin; r += stride) {  // uniform per team
        const int i = rows[r];
        const int Pi = (int)P[i];
        const long long out_off = Poff[i];
        for (int q = t; q < Pi; q += G) posmap[g][q] = -1;
        __syncwarp(mask);
        int base = 0;
        for (int j = arp[i]; j < arp[i + 1]; ++j) {
            const int c = acol[j];
            const VT av = aval[j];
            const int bs = brp[c], be = brp[c + 1];
            for (int k = bs + t; k < be; k += G) {
                const int col = bcol[k];
                const VT prod = av * bval[k];
                unsigned h = hash_col(col) & (WTS - 1);
                while (true) {
                    const int old = atomicCAS(&keys[g][h], -1, col);
                    if (old == -1) {
                        first[g][h] = (unsigned char)(base + (k - bs));
                        used[g][atomicAdd(&nused[g], 1)] = (unsigned char)h;
                        break;
                    }
                    if (old == col) break;
                    h = (h + 1) & (WTS - 1);
                }
                vals[g][h] += prod;  // one product per slot per step: the (j, k) order
            }
            base += be - bs;
            __syncwarp(mask);
        }
        const int nu = nused[g];
        for (int u = t; u < nu; u += G) {
            const int h = used[g][u];
            posmap[g][first[g][h]] = (signed char)h;
        }
        __syncwarp(mask);
        // ordered compaction of posmap: entries in first-touch order
        int written = 0;
        for (int q0 = 0; q0 < Pi; q0 += G) {
            const int q = q0 + t;
            const int h = q < Pi ? posmap[g][q] : -1;
            const int take = h >= 0;
            const unsigned bal = __ballot_sync(mask, take) & mask;
            const int before = __popc(bal & ((1u << lane) - 1u));
            if (take) {
                pcol[out_off + written + before] = keys[g][h];
                pval[out_off + written + before] = vals[g][h];
            }
            written += __popc(bal);
        }
        __syncwarp(mask);
        for (int u = t; u < nu; u += G) {
            const int h = used[g][u];
            keys[g][h] = -1;
            vals[g][h] = VT(0);
        }
        if (t == 0) {
            count[i] = written;
            nused[g] = 0;
        }
        __syncwarp(mask);
    }
}

// The merge path: one thread per row of A with at most kMergeLists entries
// and kSmallP products, when every row of B has strictly increasing columns.
// The row's products are then the union of at most kMergeLists sorted lists
// (the B rows its entries select), merged in registers.
//   Pass 1 marks, for every distinct column, the product index p of its first
//   touch in a 64-bit mask (the column's first occurrence in the lowest list
//   holding it: lists are in the reference's (j, k) order).
//   Pass 2 merges again; a column's value is 0 plus its products added in
//   ascending list order -- the product order of the reference's zeroed
//   accumulator -- and it is written at its first-touch rank, the number of
//   mask bits below its p.
// No atomics on the data; a warp serves 32 rows.
template <typename VT>
struct MergeLists {  // list j: B entries [kb, ke); its products start at index off + kb
    int kb[kMergeLists], ke[kMergeLists], off[kMergeLists];
    VT av[kMergeLists];
};

// Fills the lists of row i from its first kMergeLists entries; returns the
// products of those entries.
template <typename VT>
__device__ __forceinline__ int merge_lists(int i, const int *__restrict__ arp, const int *__restrict__ acol,
                                           const VT *__restrict__ aval, const int *__restrict__ brp,
                                           MergeLists<VT> &L) {
    const int a0 = arp[i], la = arp[i + 1] - a0;
    int o = 0;
#pragma unroll
    for (int j = 0; j < kMergeLists; ++j) {
        L.kb[j] = L.ke[j] = L.off[j] = 0;
        L.av[j] = VT(0);
        if (j < la) {
            const int c = acol[a0 + j];
            L.av[j] = aval[a0 + j];
            L.kb[j] = brp[c];
            L.ke[j] = brp[c + 1];
            L.off[j] = o - L.kb[j];
            o += L.ke[j] - L.kb[j];
        }
    }
    return o;
}

// Visits the union of the lists in ascending column order: f(col, p, sum)
// with p the column's first product index and (SUM) its products summed in
// list order.  Returns false if some list does not strictly increase (the
// walk then still ends, and every p stays below the row's product count).
template <bool SUM, typename VT, typename F>
__device__ __forceinline__ bool merge_walk(const MergeLists<VT> &L, const int *__restrict__ bcol,
                                           const VT *__restrict__ bval, F f) {
    bool increasing = true;
    constexpr int K = kMergeLists;
    constexpr int INF = 0x7fffffff;
    int k[K], h[K];
#pragma unroll
    for (int j = 0; j < K; ++j) {
        k[j] = L.kb[j];
        h[j] = k[j] < L.ke[j] ? bcol[k[j]] : INF;
    }
    while (true) {
        int m = INF;
#pragma unroll
        for (int j = 0; j < K; ++j) m = min(m, h[j]);
        if (m == INF) break;
        int fp = -1;
        VT sum = VT(0);
#pragma unroll
        for (int j = 0; j < K; ++j)
            if (h[j] == m) {
                if (fp < 0) fp = L.off[j] + k[j];
                if (SUM) sum += L.av[j] * bval[k[j]];
                ++k[j];
                h[j] = k[j] < L.ke[j] ? bcol[k[j]] : INF;
                increasing &= h[j] > m;
            }
        f(m, fp, sum);
    }
    return increasing;
}

__device__ __forceinline__ int first_touch_rank(unsigned long long mask, int p) {
    return __popcll(mask & ((1ull << p) - 1ull));
}

// MODE 0: both passes for the rows of a bin list, written at each row's
// product offset.  MODE 1: pass 1 for every row of A in order; stores the
// mask and the count, raises *warp_max to the largest number of C entries
// that one warp's 32 rows hold (the staging size of the write pass), and
// sets *off_path if a row does not qualify for the merge path (more than
// kMergeLists entries, more than kSmallP products, or a B list that does
// not strictly increase) -- then the masks are not used.
template <typename VT, int MODE>
__global__ void __launch_bounds__(256) gustavson_merge(
    const int *__restrict__ rows, int64_t n_rows_bin, const long long *__restrict__ Poff, const int *__restrict__ arp,
    const int *__restrict__ acol, const VT *__restrict__ aval, const int *__restrict__ brp,
    const int *__restrict__ bcol, const VT *__restrict__ bval, int *__restrict__ pcol, VT *__restrict__ pval,
    int *__restrict__ count, unsigned long long *__restrict__ masks, int *__restrict__ warp_max,
    int *__restrict__ off_path) {
    const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (MODE == 0 && r >= n_rows_bin) return;
    const bool valid = r < n_rows_bin;
    const int i = rows ? rows[r] : (int)r;
    unsigned long long mask = 0ull;
    MergeLists<VT> L;
    if (valid) {
        const int o = merge_lists<VT>(i, arp, acol, aval, brp, L);
        if (MODE == 1 && (arp[i + 1] - arp[i] > kMergeLists || o > kSmallP)) {
            *off_path = 1;
        } else {
            const bool inc = merge_walk<false>(L, bcol, bval, [&](int, int fp, VT) { mask |= 1ull << fp; });
            if (MODE == 1 && !inc) *off_path = 1;
        }
    }
    const int cnt = __popcll(mask);
    if (MODE == 1) {
        if (valid) {
            masks[i] = mask;
            count[i] = cnt;
        }
        int t = cnt;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
        if ((threadIdx.x & 31) == 0 && t > 0) atomicMax(warp_max, t);
        return;
    }
    const long long out = Poff[i];
    merge_walk<true>(L, bcol, bval, [&](int m, int fp, VT sum) {
        const int pos = first_touch_rank(mask, fp);
        pcol[out + pos] = m;
        pval[out + pos] = sum;
    });
    count[i] = cnt;
}

// Pass 2 of the direct path (every row of A on the merge path): each warp
// stages its 32 rows' entries -- a contiguous range of C -- in shared memory
// and writes that range with coalesced stores.  `stage` entries per warp
// (at least the largest range, so every warp fits).
template <typename VT>
__global__ void __launch_bounds__(kMergeWriteThreads) gustavson_merge_write(
    int64_t n, int stage, const int *__restrict__ arp, const int *__restrict__ acol, const VT *__restrict__ aval,
    const int *__restrict__ brp, const int *__restrict__ bcol, const VT *__restrict__ bval,
    const unsigned long long *__restrict__ masks, const int *__restrict__ crp, int *__restrict__ ccol,
    VT *__restrict__ cval) {
    extern __shared__ __align__(16) unsigned char smem[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    VT *sval = reinterpret_cast<VT *>(smem) + (int64_t)warp * stage;
    int *scol = reinterpret_cast<int *>(reinterpret_cast<VT *>(smem) + (int64_t)(blockDim.x >> 5) * stage) +
                (int64_t)warp * stage;
    const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t w0 = r - lane;  // the warp's first row
    if (w0 >= n) return;          // the whole warp
    const int64_t w1 = w0 + 32 < n ? w0 + 32 : n;
    const long long base = crp[w0];
    const int total = (int)(crp[w1] - base);
    if (r < n) {
        const int i = (int)r;
        const unsigned long long mask = masks[i];
        MergeLists<VT> L;
        merge_lists<VT>(i, arp, acol, aval, brp, L);
        const int at = (int)(crp[i] - base);
        merge_walk<true>(L, bcol, bval, [&](int m, int fp, VT sum) {
            const int pos = at + first_touch_rank(mask, fp);
            if (pos < total) {  // always: the row's ranks are below its count
                scol[pos] = m;
                sval[pos] = sum;
            }
        });
    }
    __syncwarp();
    for (int t = lane; t < total; t += 32) {
        ccol[base + t] = scol[t];
        cval[base + t] = sval[t];
    }
}

template <typename VT>
__global__ void __launch_bounds__(kCtaThreads) gustavson_cta(
    const int *__restrict__ rows, int n_rows_bin, const long long *__restrict__ P, const long long *__restrict__ Poff,
    const int *__restrict__ arp, const int *__restrict__ acol, const VT *__restrict__ aval,
    const int *__restrict__ brp, const int *__restrict__ bcol, const VT *__restrict__ bval, int *__restrict__ pcol,
    VT *__restrict__ pval, int *__restrict__ count) {
    extern __shared__ __align__(16) unsigned char smem[];
    VT *vals = reinterpret_cast<VT *>(smem);
    int *keys = reinterpret_cast<int *>(vals + kCtaTS);
    int *first = keys + kCtaTS;
    int *posmap = first + kCtaTS;
    const int i = rows[blockIdx.x];
    gustavson_row<VT>(i, threadIdx.x, kCtaThreads, arp, acol, aval, brp, bcol, bval, keys, first, vals, posmap,
                      kCtaTS, P[i], Poff[i], pcol, pval, count, CtaSync());
}

// rows with more than kCtaP products: tables in a global workspace
template <typename VT>
__global__ void __launch_bounds__(kCtaThreads) gustavson_global(
    const int *__restrict__ rows, const long long *__restrict__ ws_off, const unsigned *__restrict__ ws_ts,
    const long long *__restrict__ P, const long long *__restrict__ Poff, const int *__restrict__ arp,
    const int *__restrict__ acol, const VT *__restrict__ aval, const int *__restrict__ brp,
    const int *__restrict__ bcol, const VT *__restrict__ bval, int *__restrict__ pcol, VT *__restrict__ pval,
    int *__restrict__ count, int *ws_keys, int *ws_first, VT *ws_vals, int *ws_pos) {
    const int b = blockIdx.x;
    const int i = rows[b];
    const long long o = ws_off[b];
    gustavson_row<VT>(i, threadIdx.x, kCtaThreads, arp, acol, aval, brp, bcol, bval, ws_keys + o, ws_first + o,
                      ws_vals + o, ws_pos + Poff[i], ws_ts[b], P[i], Poff[i], pcol, pval, count, CtaSync());
}

__global__ void ws_sizes(const int *__restrict__ rows, int m, const long long *__restrict__ P,
                         unsigned *__restrict__ ts, long long *__restrict__ sz) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= m) return;
    unsigned t = 1;
    while ((long long)t < 2 * P[rows[b]]) t <<= 1;
    ts[b] = t;
    sz[b] = t;
}

template <typename VT>
__global__ void compact_kernel(const int *__restrict__ crp, const long long *__restrict__ Poff, int64_t n,
                               const int *__restrict__ pcol, const VT *__restrict__ pval, int *__restrict__ ccol,
                               VT *__restrict__ cval) {
    const int64_t i = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) / kRowGroup;
    const int lane = threadIdx.x % kRowGroup;
    if (i >= n) return;
    const int s = crp[i], len = crp[i + 1] - s;
    const long long o = Poff[i];
    for (int t = lane; t < len; t += kRowGroup) {
        ccol[s + t] = pcol[o + t];
        cval[s + t] = pval[o + t];
    }
}

template <typename T> void excl_scan(const T *in, T *out, int64_t n, DevBuf &tmp, cudaStream_t st) {
    SMAX_CUDA(cudaMemsetAsync(out, 0, sizeof(T), st));
    if (n == 0) return;
    size_t tb = 0;
    SMAX_CUDA(cub::DeviceScan::InclusiveSum(nullptr, tb, in, out + 1, (int)n, st));
    tmp.ensure(tb);
    SMAX_CUDA(cub::DeviceScan::InclusiveSum(tmp.p, tb, in, out + 1, (int)n, st));
}

}  // namespace

namespace {

void record_times(cudaEvent_t *ev, SpgemmTimes *times) {
    if (!times) return;
    float a = 0, b = 0, c = 0, d = 0;
    cudaEventElapsedTime(&a, ev[0], ev[1]);
    cudaEventElapsedTime(&b, ev[1], ev[2]);
    cudaEventElapsedTime(&c, ev[2], ev[3]);
    cudaEventElapsedTime(&d, ev[3], ev[4]);
    times->setup = a * 1e-3;
    times->fused = b * 1e-3;
    times->alloc = c * 1e-3;
    times->compress = d * 1e-3;
}

// Pass 2 of the direct merge path into C (C's row pointer and arrays ready;
// `stage` the largest number of C entries of one warp's 32 rows).
template <typename VT>
void merge_write(const DevCRS &A, const DevCRS &B, DevCRS &C, SpgemmWork &w, int stage, cudaStream_t st) {
    const int64_t n = A.n_rows;
    // a warp's 32 rows hold at most 32 * kSmallP entries
    stage = std::max(8, (stage + 7) / 8 * 8);
    if (stage > 32 * kSmallP) fail(SMAX_ERR_STATE, "SpGEMM merge path: staging size out of range");
    constexpr int kMaxSmem = kMergeWriteThreads / 32 * 32 * kSmallP * (int)(sizeof(VT) + sizeof(int));
    // set on every call: the attribute belongs to the current device
    SMAX_CUDA(cudaFuncSetAttribute(gustavson_merge_write<VT>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxSmem));
    const size_t smem = (size_t)kMergeWriteThreads / 32 * stage * (sizeof(VT) + sizeof(int));
    gustavson_merge_write<VT><<<ceil_div_u(n, kMergeWriteThreads), kMergeWriteThreads, smem, st>>>(
        n, stage, A.rp(), A.ci(), A.val.as<VT>(), B.rp(), B.ci(), B.val.as<VT>(), w.masks.as<unsigned long long>(),
        C.rp(), C.col.as<int>(), C.val.as<VT>());
    SMAX_CUDA(cudaGetLastError());
}

}  // namespace

template <typename VT>
void spgemm(const DevCRS &A, const DevCRS &B, DevCRS &C, SpgemmWork &w, SpgemmTimes *times, cudaStream_t st) {
    if (A.n_cols != B.n_rows) fail(SMAX_ERR_BAD_ARG, "A.n_cols must equal B.n_rows");
    const int64_t n = A.n_rows;
    C.n_rows = n;
    C.n_cols = B.n_cols;
    C.row_ptr.ensure(sizeof(int) * (n + 1));
    // phase boundaries for the timers, only when they are wanted
    struct PhaseEvents {
        cudaEvent_t ev[5] = {};
        explicit PhaseEvents(bool on) {
            if (on)
                for (auto &e : ev) SMAX_CUDA(cudaEventCreate(&e));
        }
        void mark(int i, cudaStream_t s) {
            if (ev[i]) SMAX_CUDA(cudaEventRecord(ev[i], s));
        }
        ~PhaseEvents() {
            for (auto &e : ev)
                if (e) cudaEventDestroy(e);
        }
    } pe(times != nullptr);
    cudaEvent_t *ev = pe.ev;
    pe.mark(0, st);
    // The last apply took the direct merge path: try it first.  Pass 1
    // checks every row (off_path); only if one fails are the rows classified.
    if (w.direct_hint && n > 0) {
        w.counts.ensure(sizeof(int) * (kBins + 3));
        w.count.ensure(sizeof(int) * n);
        w.masks.ensure(sizeof(unsigned long long) * n);
        int *flags = w.counts.as<int>() + kBins;  // b_sorted (unused here), warp_max, off_path
        SMAX_CUDA(cudaMemsetAsync(flags, 0, sizeof(int) * 3, st));
        pe.mark(1, st);
        gustavson_merge<VT, 1><<<ceil_div_u(n, 256), 256, 0, st>>>(
            nullptr, n, nullptr, A.rp(), A.ci(), A.val.as<VT>(), B.rp(), B.ci(), B.val.as<VT>(), nullptr, nullptr,
            w.count.as<int>(), w.masks.as<unsigned long long>(), flags + 1, flags + 2);
        SMAX_CUDA(cudaGetLastError());
        pe.mark(2, st);
        excl_scan<int>(w.count.as<int>(), C.row_ptr.as<int>(), n, w.scan_tmp, st);
        int nnz = 0, hf[2] = {0, 0};
        SMAX_CUDA(cudaMemcpyAsync(&nnz, C.row_ptr.as<int>() + n, sizeof(int), cudaMemcpyDeviceToHost, st));
        SMAX_CUDA(cudaMemcpyAsync(hf, flags + 1, sizeof(int) * 2, cudaMemcpyDeviceToHost, st));
        SMAX_CUDA(cudaStreamSynchronize(st));
        if (hf[1] == 0) {
            C.nnz = nnz;
            C.col.ensure(sizeof(int) * (nnz ? nnz : 1));
            C.val.ensure(sizeof(VT) * (nnz ? nnz : 1));
            pe.mark(3, st);
            merge_write<VT>(A, B, C, w, hf[0], st);
            pe.mark(4, st);
            SMAX_CUDA(cudaStreamSynchronize(st));
            record_times(ev, times);
            return;
        }
        w.direct_hint = false;  // a row left the merge path: classify them all
        pe.mark(0, st);
    }
    // --- setup: product counts, their offsets, row bins
    w.P.ensure(sizeof(long long) * (n ? n : 1));
    w.Poff.ensure(sizeof(long long) * (n + 1));
    w.lists.ensure(sizeof(int) * kBins * (n ? n : 1));
    w.counts.ensure(sizeof(int) * (kBins + 3));  // the bin counts, then b_sorted, warp_max, off_path
    w.count.ensure(sizeof(int) * (n ? n : 1));
    long long *P = w.P.as<long long>(), *Poff = w.Poff.as<long long>();
    SMAX_CUDA(cudaMemsetAsync(w.counts.p, 0, sizeof(int) * (kBins + 3), st));
    int *b_sorted = w.counts.as<int>() + kBins, *warp_max = b_sorted + 1, *off_path = b_sorted + 2;
    const int one = 1;
    SMAX_CUDA(cudaMemcpyAsync(b_sorted, &one, sizeof(int), cudaMemcpyHostToDevice, st));
    if (n > 0) {
        row_products<<<ceil_div_u((uint64_t)n * kRowGroup, 256), 256, 0, st>>>(A.rp(), A.ci(), B.rp(), n, P);
        if (B.n_rows > 0)
            b_sorted_kernel<<<grid_cap(B.n_rows), 256, 0, st>>>(B.rp(), B.ci(), B.n_rows, b_sorted);
        bin_rows<<<ceil_div_u(n, 256), 256, 0, st>>>(P, A.rp(), n, b_sorted, w.lists.as<int>(),
                                                     w.counts.as<int>());
        SMAX_CUDA(cudaGetLastError());
    }
    excl_scan<long long>(P, Poff, n, w.scan_tmp, st);
    struct {
        long long total_p;
        int counts[kBins];
    } h{};
    SMAX_CUDA(cudaMemcpyAsync(&h.total_p, Poff + n, sizeof(long long), cudaMemcpyDeviceToHost, st));
    SMAX_CUDA(cudaMemcpyAsync(h.counts, w.counts.p, sizeof(int) * kBins, cudaMemcpyDeviceToHost, st));
    SMAX_CUDA(cudaStreamSynchronize(st));
    const long long total_p = h.total_p;
    const int ns = h.counts[0], nw = h.counts[1], nc = h.counts[2], ng = h.counts[3], nm = h.counts[4];
    const int *rs = w.lists.as<int>(), *rw = rs + n, *rc = rs + 2 * n, *rg = rs + 3 * n, *rm = rs + 4 * n;
    pe.mark(1, st);
    // --- fused Gustavson pass into product-offset (padded) buffers
    if (nm != n || n == 0) {  // the direct merge path writes C itself
        w.pcol.ensure(sizeof(int) * (total_p ? total_p : 1));
        w.pval.ensure(sizeof(VT) * (total_p ? total_p : 1));
    }
    int *pcol = w.pcol.as<int>(), *count = w.count.as<int>();
    VT *pval = w.pval.as<VT>();
    if (ns > 0) {
        // persistent teams: as many CTAs as are resident at once, or fewer
        auto kern = gustavson_small<VT, kSmallP, kSmallTS, kSmallWarps, kSmallTeam>;
        static int per_sm[2] = {0, 0};
        int &ps = per_sm[sizeof(VT) == 8 ? 1 : 0];
        if (ps == 0) {
            SMAX_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&ps, kern, kSmallWarps * 32, 0));
            if (ps < 1) ps = 1;
        }
        const int64_t teams_per_cta = kSmallWarps * 32 / kSmallTeam;
        const int64_t need = (ns + teams_per_cta - 1) / teams_per_cta;
        const unsigned grid = (unsigned)std::min<int64_t>(need, (int64_t)ps * sm_count());
        kern<<<grid, kSmallWarps * 32, 0, st>>>(rs, ns, P, Poff, A.rp(), A.ci(), A.val.as<VT>(), B.rp(), B.ci(),
                                                B.val.as<VT>(), pcol, pval, count);
    }
    // every row on the merge path: pass 1 counts, C's row pointer by scan,
    // pass 2 writes C directly (no padded buffer, no compaction)
    const bool direct = nm == n && n > 0;
    if (direct) {
        w.masks.ensure(sizeof(unsigned long long) * n);
        gustavson_merge<VT, 1><<<ceil_div_u(n, 256), 256, 0, st>>>(
            nullptr, n, Poff, A.rp(), A.ci(), A.val.as<VT>(), B.rp(), B.ci(), B.val.as<VT>(), nullptr, nullptr, count,
            w.masks.as<unsigned long long>(), warp_max, off_path);
    } else if (nm > 0) {
        gustavson_merge<VT, 0><<<ceil_div_u(nm, 256), 256, 0, st>>>(
            rm, nm, Poff, A.rp(), A.ci(), A.val.as<VT>(), B.rp(), B.ci(), B.val.as<VT>(), pcol, pval, count, nullptr,
            nullptr, nullptr);
    }
    if (nw > 0)
        gustavson_warp<VT, kWarpP, kWarpTS, kWarpsPerCta, 32><<<ceil_div_u(nw, kWarpsPerCta), kWarpsPerCta * 32, 0, st>>>(
            rw, nw, P, Poff, A.rp(), A.ci(), A.val.as<VT>(), B.rp(), B.ci(), B.val.as<VT>(), pcol, pval, count);
    if (nc > 0) {
        const size_t sm = (size_t)kCtaTS * (sizeof(VT) + 2 * sizeof(int)) + sizeof(int) * kCtaP;
        SMAX_CUDA(cudaFuncSetAttribute(gustavson_cta<VT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
        gustavson_cta<VT><<<nc, kCtaThreads, sm, st>>>(rc, nc, P, Poff, A.rp(), A.ci(), A.val.as<VT>(), B.rp(),
                                                       B.ci(), B.val.as<VT>(), pcol, pval, count);
    }
    if (ng > 0) {
        w.wts.ensure(sizeof(unsigned) * ng);
        w.wsz.ensure(sizeof(long long) * ng);
        w.woff.ensure(sizeof(long long) * (ng + 1));
        ws_sizes<<<ceil_div_u(ng, 256), 256, 0, st>>>(rg, ng, P, w.wts.as<unsigned>(), w.wsz.as<long long>());
        SMAX_CUDA(cudaGetLastError());
        excl_scan<long long>(w.wsz.as<long long>(), w.woff.as<long long>(), ng, w.scan_tmp, st);
        long long wtot = 0;
        SMAX_CUDA(cudaMemcpyAsync(&wtot, w.woff.as<long long>() + ng, sizeof(long long), cudaMemcpyDeviceToHost, st));
        SMAX_CUDA(cudaStreamSynchronize(st));
        w.wkeys.ensure(sizeof(int) * wtot);
        w.wfirst.ensure(sizeof(int) * wtot);
        w.wvals.ensure(sizeof(VT) * wtot);
        w.wpos.ensure(sizeof(int) * total_p);
        gustavson_global<VT><<<ng, kCtaThreads, 0, st>>>(rg, w.woff.as<long long>(), w.wts.as<unsigned>(), P, Poff,
                                                         A.rp(), A.ci(), A.val.as<VT>(), B.rp(), B.ci(),
                                                         B.val.as<VT>(), pcol, pval, count, w.wkeys.as<int>(),
                                                         w.wfirst.as<int>(), w.wvals.as<VT>(), w.wpos.as<int>());
    }
    SMAX_CUDA(cudaGetLastError());
    pe.mark(2, st);
    // --- C's row pointer and arrays
    excl_scan<int>(count, C.row_ptr.as<int>(), n, w.scan_tmp, st);
    int nnz = 0, stage = 0;
    SMAX_CUDA(cudaMemcpyAsync(&nnz, C.row_ptr.as<int>() + n, sizeof(int), cudaMemcpyDeviceToHost, st));
    if (direct) SMAX_CUDA(cudaMemcpyAsync(&stage, warp_max, sizeof(int), cudaMemcpyDeviceToHost, st));
    SMAX_CUDA(cudaStreamSynchronize(st));
    C.nnz = nnz;
    C.col.ensure(sizeof(int) * (nnz ? nnz : 1));
    C.val.ensure(sizeof(VT) * (nnz ? nnz : 1));
    pe.mark(3, st);
    if (direct) {
        merge_write<VT>(A, B, C, w, stage, st);
    } else if (n > 0) {
        compact_kernel<VT><<<ceil_div_u((uint64_t)n * kRowGroup, 256), 256, 0, st>>>(C.rp(), Poff, n, pcol, pval,
                                                                              C.col.as<int>(), C.val.as<VT>());
        SMAX_CUDA(cudaGetLastError());
    }
    pe.mark(4, st);
    SMAX_CUDA(cudaStreamSynchronize(st));
    w.direct_hint = direct;
    record_times(ev, times);
}

template void spgemm<double>(const DevCRS &, const DevCRS &, DevCRS &, SpgemmWork &, SpgemmTimes *, cudaStream_t);
template void spgemm<float>(const DevCRS &, const DevCRS &, DevCRS &, SpgemmWork &, SpgemmTimes *, cudaStream_t);

}  // namespace smax
