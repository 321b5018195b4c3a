// levelpack.cu -- level-ordered packed triangular solves on sm_100a.
//
// The per-row recurrence is the reference's (naive_crs_sptrsv / crs_sptrsv_lvl,
// src/kernels/sptrsv/sptrsv_cpu/sptrsv_cpu_crs_impl.hpp:9-55,
// sptrsv_lvl_cpu_crs_impl.hpp:11-82): x[r] = (b[r] - sum_j val[j] x[col[j]]) / D[r]
// with the off-diagonal entries summed in stored order.  What changes is the
// layout, for latency: a level-scheduled solve of a matrix with thousands of
// narrow levels is a chain of dependent steps, and in the plain layout every
// step waits on order -> row_ptr -> col/val -> x, four dependent global loads.
//
// * Rows are renumbered in sweep order ("positions") and each level's
//   off-diagonal entries are stored as a dense column-major block, so a thread
//   finds its row's entries at a fixed offset: no row_ptr hop, coalesced loads.
// * The single-CTA sweep over a run of narrow levels keeps the last kRing
//   solutions in a shared-memory ring indexed by position; an entry whose
//   solution is guaranteed to still be in the ring is encoded with its slot
//   at pack time (the ring slot of position q is q % kRing; it survives until
//   position q + kRing is written, so it is safe while q >= level_end - kRing).
// * While a level is computed, each thread already loads the next level's
//   entries, right-hand sides and diagonals into registers, and the block
//   prefetches the level kL2Ahead steps ahead into L2: the critical path per
//   level is ring reads, a few FMAs, the division and the CTA barrier.
// * Right-hand sides are gathered into position order before the sweep and
//   the solution scattered back after it (two coalesced passes over n).
#include "levelpack.cuh"

#include <algorithm>

#include <cooperative_groups.h>
#include <cub/device/device_segmented_reduce.cuh>

namespace smax {

namespace {

using Level = LevelPack::Level;
constexpr int kPad = LevelPack::kPad;
constexpr int kRing = LevelPack::kRing;
constexpr int kRingShift = 13;     // kRing == 1 << kRingShift
constexpr int kRowsPerThread = 2;  // rows of a level held in registers per thread (default sweeps)
constexpr int kEnts = 2;           // prefetched entries per row (the rest are loaded when used)
#ifndef SMAX_SWEEP_L2_AHEAD
#define SMAX_SWEEP_L2_AHEAD 3
#endif
// levels between a level's L2 prefetch and its sweep (>= 2).  Three: the
// 64-matrix batch 1.464 -> 1.265 ms and the natural 2048^2 sweep 5.41 -> 5.02
// ms against two; four measured the same as three.
constexpr int kL2Ahead = SMAX_SWEEP_L2_AHEAD;
static_assert(kL2Ahead >= 2, "the next level is loaded into registers; L2 prefetch runs further ahead");
constexpr int kClusterCTAs = 8;    // CTAs of a cluster run (portable cluster size)
constexpr int kClusterThreads = 256;
static_assert(kRing == (1 << kRingShift), "ring size");

unsigned grid_for(int64_t work) {
    const int64_t cap = (int64_t)sm_count() * 8;
    int64_t g = (work + 255) / 256;
    return (unsigned)(g < 1 ? 1 : (g > cap ? cap : g));
}

// ---------------------------------------------------------------- build ----
__global__ void positions_kernel(const int *__restrict__ pos_begin, int n_lv, const int *__restrict__ src_begin,
                                 const int *__restrict__ order, int64_t n, int *__restrict__ prow,
                                 int *__restrict__ plev, int *__restrict__ pos_of_row) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += stride) {
        int lo = 0, hi = n_lv - 1;  // last s with pos_begin[s] <= p
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (pos_begin[mid] <= p) lo = mid;
            else hi = mid - 1;
        }
        const int k = src_begin[lo] + (int)(p - pos_begin[lo]);
        const int r = order ? order[k] : k;
        prow[p] = r;
        plev[p] = lo;
        pos_of_row[r] = (int)p;
    }
}

__global__ void off_len_kernel(const int *__restrict__ rp, const int *__restrict__ prow, int64_t n,
                               int *__restrict__ len) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += stride) {
        const int r = prow[p];
        len[p] = rp[r + 1] - rp[r] - 1;
    }
}

template <typename VT>
__global__ void fill_kernel(const int *__restrict__ rp, const int *__restrict__ ci, const VT *__restrict__ val,
                            const VT *__restrict__ D, int64_t n, const int *__restrict__ prow,
                            const int *__restrict__ plev, const int *__restrict__ pos_of_row,
                            const Level *__restrict__ lv, const int *__restrict__ seg_pos,
                            const int2 *__restrict__ geo, int *__restrict__ psrc, VT *__restrict__ pval,
                            VT *__restrict__ pinv, int *needs_init, bool row_src) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += stride) {
        const int s = plev[p];
        const Level L = lv[s];
        const int t = (int)(p - L.pos);
        const int r = prow[p];
        const int j0 = rp[r], len = rp[r + 1] - j0 - 1;
        const int segb = seg_pos[s], le = L.pos + L.m;
        const int2 g2 = geo[s];  // the run's (CTAs, threads per CTA)
        const int G = g2.x * g2.y;
        for (int i = 0; i < L.w; ++i) {
            const long long idx = L.base + (long long)i * L.m + t;
            if (i < len) {
                const int q = pos_of_row[ci[j0 + i]];
                if (q >= L.pos) atomicExch(needs_init, 1);
                const bool ring = q >= segb && q < L.pos && q >= le - kRing;
                int code = q;
                if (ring) {
                    // the thread of the run that solves position q: its row
                    // index in its level modulo the run's thread count
                    const int tq = q - lv[plev[q]].pos;
                    const int owner = (tq % G) / g2.y;
                    code = -((owner << kRingShift) | (q & (kRing - 1))) - 1;
                }
                psrc[idx] = row_src ? ci[j0 + i] : code;
                pval[idx] = val[j0 + i];
            } else {
                psrc[idx] = kPad;
                pval[idx] = VT(0);
            }
        }
        pinv[p] = VT(1) / D[r];
    }
}

// ---------------------------------------------------------------- solve ----
template <typename VT>
__global__ void gather_kernel(const int *__restrict__ prow, int64_t n, const VT *__restrict__ B, VT *__restrict__ bp,
                              const VT *__restrict__ X, VT *__restrict__ xp) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += stride) {
        const int r = prow[p];
        bp[p] = B[r];
        if (xp) xp[p] = X[r];
    }
}

template <typename VT>
__global__ void scatter_kernel(const int *__restrict__ prow, int64_t n, const VT *__restrict__ xp, VT *__restrict__ X) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += stride) X[prow[p]] = xp[p];
}

constexpr int kWideEnts = 4;  // entries of a row whose loads are all issued before the first use

// one wide level: thread per row.  The first kWideEnts entries and their
// solutions are loaded before any is used, so a row costs one entry load and
// one gather of latency instead of one pair per entry.
template <typename VT>
__global__ void wide_level_kernel(Level L, const int *__restrict__ psrc, const VT *__restrict__ pval,
                                  const VT *__restrict__ pinv, const VT *__restrict__ bp, VT *xp) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= L.m) return;
    int src[kWideEnts];
    VT v[kWideEnts], xs[kWideEnts];
#pragma unroll
    for (int i = 0; i < kWideEnts; ++i) {
        src[i] = kPad;
        if (i < L.w) {
            const long long idx = L.base + (long long)i * L.m + t;
            src[i] = psrc[idx];
            v[i] = pval[idx];
        }
    }
#pragma unroll
    for (int i = 0; i < kWideEnts; ++i) xs[i] = src[i] != kPad ? xp[src[i]] : VT(0);
    const int p = L.pos + t;
    const VT bi = bp[p], inv = pinv[p];
    VT sum = VT(0);
    bool more = true;
#pragma unroll
    for (int i = 0; i < kWideEnts; ++i) {
        if (src[i] == kPad) { more = false; break; }
        sum += v[i] * xs[i];
    }
    if (more)
        for (int i = kWideEnts; i < L.w; ++i) {
            const long long idx = L.base + (long long)i * L.m + t;
            const int s = psrc[idx];
            if (s == kPad) break;
            sum += pval[idx] * xp[s];
        }
    xp[p] = (bi - sum) * inv;
}

template <typename VT> struct RowRegs {
    int src[kEnts];
    VT v[kEnts];
    VT b, inv;
};

__device__ __forceinline__ Level load_level(const Level *lv, int s) {
    static_assert(sizeof(Level) == sizeof(int4), "a level is one 16-byte load");
    const int4 v = *reinterpret_cast<const int4 *>(lv + s);
    return Level{v.x, v.y, v.z, v.w};
}

template <typename VT, int T, int CS, int NR>
__device__ __forceinline__ void load_rows(const Level &L, int g, const int *__restrict__ psrc,
                                          const VT *__restrict__ pval, const VT *__restrict__ pinv,
                                          const VT *__restrict__ bp, RowRegs<VT> (&R)[NR]) {
#pragma unroll
    for (int k = 0; k < NR; ++k) {
        const int t = g + k * T * CS;
#pragma unroll
        for (int i = 0; i < kEnts; ++i) R[k].src[i] = kPad;
        if (t < L.m) {
            const int p = L.pos + t;
            R[k].b = bp[p];
            R[k].inv = pinv[p];
#pragma unroll
            for (int i = 0; i < kEnts; ++i)
                if (i < L.w) {
                    const int idx = L.base + i * L.m + t;
                    R[k].src[i] = psrc[idx];
                    R[k].v[i] = pval[idx];
                }
        }
    }
}

// the g-th thread of a run prefetches the g-th 128-byte line of each of level
// L's ranges into L2 (wider levels are prefetched in part)
template <typename VT>
__device__ __forceinline__ void prefetch_level_l2(const Level &L, int g, const int *psrc, const VT *pval,
                                                  const VT *pinv, const VT *bp) {
    const long long o = (long long)g * 128;
    const long long ne = (long long)L.m * L.w;
    if (o < ne * 4) asm volatile("prefetch.global.L2 [%0];" ::"l"(reinterpret_cast<const char *>(psrc + L.base) + o));
    if (o < ne * (long long)sizeof(VT))
        asm volatile("prefetch.global.L2 [%0];" ::"l"(reinterpret_cast<const char *>(pval + L.base) + o));
    if (o < (long long)L.m * (long long)sizeof(VT)) {
        asm volatile("prefetch.global.L2 [%0];" ::"l"(reinterpret_cast<const char *>(pinv + L.pos) + o));
        asm volatile("prefetch.global.L2 [%0];" ::"l"(reinterpret_cast<const char *>(bp + L.pos) + o));
    }
}

// A solution named by an entry: global position, own ring, or (in a cluster
// run) the ring of another CTA through distributed shared memory.
template <typename VT, int CS>
__device__ __forceinline__ VT solution(int src, VT *ring, const VT *xp, unsigned rank) {
    // in a cluster run another SM may have written xp[src]: read it from L2
    // (L1 is not coherent across SMs); one CTA reads its own writes
    if (src >= 0) return CS == 1 ? xp[src] : __ldcg(xp + src);
    const int code = -src - 1;
    if constexpr (CS == 1) {
        return ring[code];
    } else {
        const unsigned owner = (unsigned)code >> kRingShift;
        VT *slot = ring + (code & (kRing - 1));
        if (owner == rank) return *slot;
        return *cooperative_groups::this_cluster().map_shared_rank(slot, owner);
    }
}

template <int CS> __device__ __forceinline__ void run_barrier() {
    if constexpr (CS == 1) __syncthreads();
    else cooperative_groups::this_cluster().sync();  // barrier.cluster arrive.release / wait.acquire
}

// One level s of a run: loads level fill_s's rows (described by Ln) into
// `nxt` and prefetches level s+kL2Ahead into L2 while it solves level s from
// `cur`, then the run's barrier.  Returns level ret_s's descriptor.  With two
// register sets fill_s = s+1 and ret_s = s+2; with three, s+2 and s+3.
template <typename VT, int T, int CS, int NR>
__device__ __forceinline__ Level sweep_level(const Level *__restrict__ lv, int s, int s1, const Level &Lc,
                                             const Level &Ln, int fill_s, int ret_s, const int *__restrict__ psrc,
                                             const VT *__restrict__ pval, const VT *__restrict__ pinv,
                                             const VT *__restrict__ bp, VT *xp, VT *ring, int g, int warp0,
                                             unsigned rank, RowRegs<VT> (&cur)[NR], RowRegs<VT> (&nxt)[NR]) {
    constexpr int G = T * CS;
    const Level Lnn = load_level(lv, ret_s < s1 ? ret_s : s);
    if (fill_s < s1 && warp0 < Ln.m) load_rows<VT, T, CS, NR>(Ln, g, psrc, pval, pinv, bp, nxt);
    if (s + kL2Ahead < s1)
        prefetch_level_l2<VT>(load_level(lv, s + kL2Ahead), g, psrc, pval, pinv, bp);
    if (warp0 < Lc.m) {
#pragma unroll
        for (int k = 0; k < NR; ++k) {
            const int t = g + k * G;
            if (t < Lc.m) {
                VT sum = VT(0);
                bool more = true;
#pragma unroll
                for (int i = 0; i < kEnts; ++i) {
                    const int src = cur[k].src[i];
                    if (src == kPad) { more = false; break; }
                    sum += cur[k].v[i] * solution<VT, CS>(src, ring, xp, rank);
                }
                if (more)
                    for (int i = kEnts; i < Lc.w; ++i) {
                        const int idx = Lc.base + i * Lc.m + t;
                        const int src = psrc[idx];
                        if (src == kPad) break;
                        sum += pval[idx] * solution<VT, CS>(src, ring, xp, rank);
                    }
                const int p = Lc.pos + t;
                const VT x = (cur[k].b - sum) * cur[k].inv;
                ring[p & (kRing - 1)] = x;
                xp[p] = x;
            }
        }
        // rows beyond the register slots (levels wider than the slots cover)
        for (int t = g + NR * G; t < Lc.m; t += G) {
            VT sum = VT(0);
            for (int i = 0; i < Lc.w; ++i) {
                const int idx = Lc.base + i * Lc.m + t;
                const int src = psrc[idx];
                if (src == kPad) break;
                sum += pval[idx] * solution<VT, CS>(src, ring, xp, rank);
            }
            const int p = Lc.pos + t;
            const VT x = (bp[p] - sum) * pinv[p];
            ring[p & (kRing - 1)] = x;
            xp[p] = x;
        }
    }
    // every CTA of a cluster passes this barrier after its last level too,
    // so no CTA leaves while another may still read its ring
    run_barrier<CS>();
    return Lnn;
}

// Sweeps steps [s0, s1) of the pack with CS CTAs of T threads (one CTA or one
// cluster); thread g of the run solves rows g, g + T*CS, ... of every level,
// the first NR of them from registers loaded ahead.  Register sets rotate
// between "this level" and the ones after it, so no set is copied into
// another: two sets (loaded one level ahead), or with THREE three sets
// (two levels ahead; the batched sweep's 512-thread CTAs: 1.265 -> 1.199 ms
// for 64 matrices, while the single solve's sweeps were 3 % slower with it).
template <typename VT, int T, int CS, int NR = kRowsPerThread, bool THREE = false>
__device__ void sweep_run(const Level *__restrict__ lv, int s0, int s1, const int *__restrict__ psrc,
                          const VT *__restrict__ pval, const VT *__restrict__ pinv, const VT *__restrict__ bp, VT *xp,
                          VT *ring) {
    if (s0 >= s1) return;
    unsigned rank = 0;
    if constexpr (CS > 1) rank = cooperative_groups::this_cluster().block_rank();
    const int g = (int)rank * T + (int)threadIdx.x;
    const int warp0 = g & ~31;
    if constexpr (THREE && T * NR <= 1024) {  // 1024-thread CTAs keep two sets (64 registers a thread)
        RowRegs<VT> ra[NR], rb[NR], rc[NR];
        Level La = load_level(lv, s0);
        Level Lb = load_level(lv, s0 + 1 < s1 ? s0 + 1 : s0);
        Level Lc = load_level(lv, s0 + 2 < s1 ? s0 + 2 : s0);
        load_rows<VT, T, CS, NR>(La, g, psrc, pval, pinv, bp, ra);
        if (s0 + 1 < s1) load_rows<VT, T, CS, NR>(Lb, g, psrc, pval, pinv, bp, rb);
        for (int s = s0; s < s1; s += 3) {
            const Level Ld = sweep_level<VT, T, CS, NR>(lv, s, s1, La, Lc, s + 2, s + 3, psrc, pval, pinv, bp, xp,
                                                        ring, g, warp0, rank, ra, rc);
            if (s + 1 >= s1) break;
            const Level Le = sweep_level<VT, T, CS, NR>(lv, s + 1, s1, Lb, Ld, s + 3, s + 4, psrc, pval, pinv, bp,
                                                        xp, ring, g, warp0, rank, rb, ra);
            if (s + 2 >= s1) break;
            const Level Lf = sweep_level<VT, T, CS, NR>(lv, s + 2, s1, Lc, Le, s + 4, s + 5, psrc, pval, pinv, bp,
                                                        xp, ring, g, warp0, rank, rc, rb);
            La = Ld;
            Lb = Le;
            Lc = Lf;
        }
    } else {
        RowRegs<VT> ra[NR], rb[NR];
        Level La = load_level(lv, s0);
        Level Lb = load_level(lv, s0 + 1 < s1 ? s0 + 1 : s0);
        load_rows<VT, T, CS, NR>(La, g, psrc, pval, pinv, bp, ra);
        for (int s = s0; s < s1; s += 2) {
            const Level L2 = sweep_level<VT, T, CS, NR>(lv, s, s1, La, Lb, s + 1, s + 2, psrc, pval, pinv, bp, xp,
                                                        ring, g, warp0, rank, ra, rb);
            if (s + 1 >= s1) break;
            const Level L3 = sweep_level<VT, T, CS, NR>(lv, s + 1, s1, Lb, L2, s + 2, s + 3, psrc, pval, pinv, bp,
                                                        xp, ring, g, warp0, rank, rb, ra);
            La = L2;
            Lb = L3;
        }
    }
}

template <typename VT, int T, int NR>
__global__ void __launch_bounds__(T, 1)
    sweep_kernel(const Level *__restrict__ lv, int s0, int s1, const int *__restrict__ psrc,
                 const VT *__restrict__ pval, const VT *__restrict__ pinv, const VT *__restrict__ bp, VT *xp) {
    extern __shared__ __align__(16) unsigned char smem[];
    sweep_run<VT, T, 1, NR>(lv, s0, s1, psrc, pval, pinv, bp, xp, reinterpret_cast<VT *>(smem));
}

// one run on a cluster of kClusterCTAs CTAs (launched with cluster dimensions)
template <typename VT>
__global__ void __launch_bounds__(kClusterThreads, 1)
    sweep_cluster_kernel(const Level *__restrict__ lv, int s0, int s1, const int *__restrict__ psrc,
                         const VT *__restrict__ pval, const VT *__restrict__ pinv, const VT *__restrict__ bp,
                         VT *xp) {
    extern __shared__ __align__(16) unsigned char smem[];
    sweep_run<VT, kClusterThreads, kClusterCTAs>(lv, s0, s1, psrc, pval, pinv, bp, xp, reinterpret_cast<VT *>(smem));
}

// Work queue of matrices; each CTA sweeps its matrix's steps.
template <typename VT, int T>
__global__ void __launch_bounds__(T, 1)
    sweep_batch_kernel(const Level *__restrict__ lv, const int *__restrict__ mat_steps,
                       const int *__restrict__ queue_order, int n_mats, int *queue, const int *__restrict__ psrc,
                       const VT *__restrict__ pval, const VT *__restrict__ pinv, const VT *__restrict__ bp, VT *xp) {
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ int m_sh;
    while (true) {
        if (threadIdx.x == 0) m_sh = atomicAdd(queue, 1);
        __syncthreads();
        const int q = m_sh;
        __syncthreads();  // m_sh is rewritten on the next turn
        if (q >= n_mats) return;
        const int m = queue_order[q];
        sweep_run<VT, T, 1, kRowsPerThread, true>(lv, mat_steps[m], mat_steps[m + 1], psrc, pval, pinv, bp, xp,
                            reinterpret_cast<VT *>(smem));
    }
}

// ------------------------------------------------------------ sync-free --
constexpr int kSfThreads = 256;
constexpr int kSfChunk = 8;   // warp tasks a CTA claims at once (one per warp)
constexpr int kSfEnts = 4;    // entries of a row loaded before its first wait

// "not solved yet": signalling-NaN patterns; arithmetic never returns a
// signalling NaN, so a computed solution is never mistaken for one
template <typename VT> struct Pending;
template <> struct Pending<double> {
    static constexpr unsigned long long bits = 0x7FF5A5A5A5A5A5A5ull;
    __device__ static bool is(double v) { return (unsigned long long)__double_as_longlong(v) == bits; }
    __device__ static double value() { return __longlong_as_double((long long)bits); }
};
template <> struct Pending<float> {
    static constexpr unsigned bits = 0x7FA5A5A5u;
    __device__ static bool is(float v) { return (unsigned)__float_as_uint(v) == bits; }
    __device__ static float value() { return __uint_as_float(bits); }
};

__device__ __forceinline__ double ld_relaxed(const double *p) {
    double v;
    asm volatile("ld.relaxed.gpu.global.f64 %0, [%1];" : "=d"(v) : "l"(p));
    return v;
}
__device__ __forceinline__ float ld_relaxed(const float *p) {
    float v;
    asm volatile("ld.relaxed.gpu.global.f32 %0, [%1];" : "=f"(v) : "l"(p));
    return v;
}
__device__ __forceinline__ void st_relaxed(double *p, double v) {
    asm volatile("st.relaxed.gpu.global.f64 [%0], %1;" ::"l"(p), "d"(v) : "memory");
}
__device__ __forceinline__ void st_relaxed(float *p, float v) {
    asm volatile("st.relaxed.gpu.global.f32 [%0], %1;" ::"l"(p), "f"(v) : "memory");
}

// The value at p once it is no longer pending.  Bounded: after `limit` polls
// the wait records SMAX_ERR_TIMEOUT and raises the abort flag; once the flag
// is up every wait returns NaN (checked every 64 polls).
template <typename VT>
__device__ __noinline__ VT wait_solved(const VT *p, long long limit, int *abort_flag, DevStatus *st) {
    for (long long it = 1;; ++it) {
        if (it > 32) __nanosleep(64);  // the first polls back to back: most waits are short
        const VT v = ld_relaxed(p);
        if (!Pending<VT>::is(v)) return v;
        if ((it & 63) == 0 && *(volatile int *)abort_flag) return VT(NAN);
        if (it >= limit) {
            report(st, SMAX_ERR_TIMEOUT, it);
            atomicExch(abort_flag, 1);
            return VT(NAN);
        }
    }
}

template <typename VT>
__device__ __forceinline__ VT solved(const VT *p, long long limit, int *abort_flag, DevStatus *st) {
    const VT v = ld_relaxed(p);
    return Pending<VT>::is(v) ? wait_solved(p, limit, abort_flag, st) : v;
}

// X := pending; ctl[0] (task counter) = ctl[1] (abort flag) = 0; ctl[4..] pending
template <typename VT>
__global__ void sf_reset_kernel(VT *__restrict__ X, int64_t n, int *__restrict__ ctl) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    const int64_t i0 = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i0 == 0) {
        ctl[0] = 0;
        ctl[1] = 0;
        *reinterpret_cast<VT *>(ctl + 4) = Pending<VT>::value();
    }
    for (int64_t i = i0; i < n; i += stride) X[i] = Pending<VT>::value();
}

// ctl: [0] task counter, [1] abort flag, [4..] a word that stays pending
// (waited on by the first row when `never` is set: the test knob).
// A task is (first position, rows | width << 6, level rows = entry stride,
// first entry).
template <typename VT>
__global__ void __launch_bounds__(kSfThreads)
    syncfree_kernel(const int4 *__restrict__ tasks, int n_tasks, const int *__restrict__ prow,
                    const int *__restrict__ psrc, const VT *__restrict__ pval, const VT *__restrict__ pinv,
                    const VT *__restrict__ B, VT *X, int *ctl, long long limit, bool never, DevStatus *st) {
    __shared__ int chunk_sh;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    int *abort_flag = ctl + 1;
    while (true) {
        if (threadIdx.x == 0) chunk_sh = atomicAdd(ctl, kSfChunk);
        __syncthreads();
        const int c0 = chunk_sh;
        __syncthreads();  // chunk_sh is rewritten on the next turn
        if (c0 >= n_tasks) return;
        const int c1 = min(c0 + kSfChunk, n_tasks);
        for (int ti = c0 + warp; ti < c1; ti += kSfThreads / 32) {
            const int4 tk = tasks[ti];
            const int w = tk.y >> 6;
            if (lane >= (tk.y & 63)) continue;
            // every load goes out before the first wait: entries, then the
            // sources' values, right-hand side and 1/D
            int src[kSfEnts];
            VT v[kSfEnts], xs[kSfEnts];
#pragma unroll
            for (int i = 0; i < kSfEnts; ++i) {
                src[i] = kPad;
                if (i < w) {
                    const long long idx = tk.w + (long long)i * tk.z + lane;
                    src[i] = psrc[idx];
                    v[i] = pval[idx];
                }
            }
#pragma unroll
            for (int i = 0; i < kSfEnts; ++i) xs[i] = src[i] != kPad ? ld_relaxed(X + src[i]) : VT(0);
            const int p = tk.x + lane;
            const int r = prow[p];
            const VT bi = B[r], inv = pinv[p];
            VT sum = VT(0);
            if (never && ti == 0 && lane == 0)
                sum += VT(0) * solved(reinterpret_cast<const VT *>(ctl + 4), limit, abort_flag, st);
            bool more = true;
#pragma unroll
            for (int i = 0; i < kSfEnts; ++i) {
                if (src[i] == kPad) { more = false; break; }
                const VT xv = Pending<VT>::is(xs[i]) ? wait_solved(X + src[i], limit, abort_flag, st) : xs[i];
                sum += v[i] * xv;
            }
            if (more)
                for (int i = kSfEnts; i < w; ++i) {
                    const long long idx = tk.w + (long long)i * tk.z + lane;
                    const int sc = psrc[idx];
                    if (sc == kPad) break;
                    sum += pval[idx] * solved(X + sc, limit, abort_flag, st);
                }
            st_relaxed(X + r, (bi - sum) * inv);
        }
    }
}

// k > 1 right-hand sides, element (r, v) at r*rs + v*vs (row-major: rs = k,
// vs = 1; column-major: rs = 1, vs = the leading dimension): a warp per
// row with its lanes over the vectors, 32 at a time; a CTA claims 8
// consecutive positions, one per warp, with one atomic.  Per row the plain
// solves' arithmetic: x[r][v] = (b[r][v] - sum_j val[j] x[col[j]][v]) / D[r],
// the off-diagonal entries in stored order (the diagonal is last in each row).
template <typename VT>
__global__ void __launch_bounds__(kSfThreads)
    syncfree_rows_kernel(const int *__restrict__ prow, int n, const int *__restrict__ rp, const int *__restrict__ ci,
                         const VT *__restrict__ val, const VT *__restrict__ D, const VT *__restrict__ B, VT *X,
                         int64_t k, int64_t rs, int64_t vs, int *ctl, long long limit, DevStatus *st) {
    __shared__ int base_sh;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    int *abort_flag = ctl + 1;
    while (true) {
        if (threadIdx.x == 0) base_sh = atomicAdd(ctl, kSfThreads / 32);
        __syncthreads();
        const int p0 = base_sh;
        __syncthreads();  // base_sh is rewritten on the next turn
        if (p0 >= n) return;
        const int p = p0 + warp;
        if (p >= n) continue;
        const int r = prow[p];
        const int s = rp[r], e = rp[r + 1] - 1;
        const VT d = D[r];
        for (int64_t v0 = 0; v0 < k; v0 += 32) {
            const int64_t v = v0 + lane;
            const bool act = v < k;
            VT sum = VT(0);
            for (int j0 = s; j0 < e; j0 += 32) {
                const int jj = j0 + lane;
                const int cj = jj < e ? ci[jj] : 0;
                const VT aj = jj < e ? val[jj] : VT(0);
                const int cnt = min(32, e - j0);
                for (int t = 0; t < cnt; ++t) {
                    const int c = __shfl_sync(0xffffffffu, cj, t);
                    const VT a = __shfl_sync(0xffffffffu, aj, t);
                    if (act) sum += a * solved(X + (int64_t)c * rs + v * vs, limit, abort_flag, st);
                }
            }
            if (act) st_relaxed(X + (int64_t)r * rs + v * vs, (B[(int64_t)r * rs + v * vs] - sum) / d);
        }
    }
}

template <typename VT, int T> void set_smem_attr_t() {
    SMAX_CUDA(cudaFuncSetAttribute(sweep_kernel<VT, T, kRowsPerThread>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)(kRing * sizeof(VT))));
    SMAX_CUDA(cudaFuncSetAttribute(sweep_batch_kernel<VT, T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)(kRing * sizeof(VT))));
}

template <typename VT> void set_smem_attr() {
    static bool done[64] = {};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64 || done[dev]) return;
    set_smem_attr_t<VT, 256>();
    set_smem_attr_t<VT, 512>();
    set_smem_attr_t<VT, 1024>();
    SMAX_CUDA(cudaFuncSetAttribute(sweep_cluster_kernel<VT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)(kRing * sizeof(VT))));
    done[dev] = true;
}

cudaLaunchConfig_t cluster_config(cudaLaunchAttribute &attr, size_t smem, cudaStream_t st) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(kClusterCTAs, 1, 1);
    cfg.blockDim = dim3(kClusterThreads, 1, 1);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    attr.id = cudaLaunchAttributeClusterDimension;
    attr.val.clusterDim.x = kClusterCTAs;
    attr.val.clusterDim.y = 1;
    attr.val.clusterDim.z = 1;
    cfg.attrs = &attr;
    cfg.numAttrs = 1;
    return cfg;
}

// whether a cluster of the sweep can be resident on this device
template <typename VT> bool cluster_ok() {
    static int state[64] = {};  // 0 unknown, 1 yes, 2 no
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64) return false;
    if (state[dev] == 0) {
        set_smem_attr<VT>();
        cudaLaunchAttribute attr;
        cudaLaunchConfig_t cfg = cluster_config(attr, kRing * sizeof(VT), nullptr);
        int clusters = 0;
        const cudaError_t e = cudaOccupancyMaxActiveClusters(&clusters, (void *)sweep_cluster_kernel<VT>, &cfg);
        if (e != cudaSuccess) (void)cudaGetLastError();
        state[dev] = (e == cudaSuccess && clusters > 0) ? 1 : 2;
    }
    return state[dev] == 1;
}

// Launch geometry of a run: (CTAs, threads per CTA) enough for its widest
// level at kRowsPerThread rows each; a cluster for levels wider than 1024 rows
// where allowed and resident, else up to one 1024-thread CTA.
int2 run_geometry(int max_w, bool allow_cluster, int vbytes) {
    const int need = (max_w + kRowsPerThread - 1) / kRowsPerThread;
    if (need <= 256) return make_int2(1, 256);
    if (need <= 512) return make_int2(1, 512);
    if (allow_cluster && (vbytes == 8 ? cluster_ok<double>() : cluster_ok<float>()))
        return make_int2(kClusterCTAs, kClusterThreads);
    return make_int2(1, 1024);
}

template <typename VT>
void launch_run(const LevelPack &pk, int s0, int s1, const int *psrc, const VT *pval, const VT *pinv, const VT *bp,
                VT *xp, cudaStream_t st) {
    const size_t sm = kRing * sizeof(VT);
    const Level *lv = pk.lv.as<Level>();
    const int2 geo = pk.h_geo[s0];
    if (geo.x > 1) {
        cudaLaunchAttribute attr;
        cudaLaunchConfig_t cfg = cluster_config(attr, sm, st);
        SMAX_CUDA(cudaLaunchKernelEx(&cfg, sweep_cluster_kernel<VT>, lv, s0, s1, psrc, pval, pinv, bp, xp));
    } else if (geo.y == 256) {
        sweep_kernel<VT, 256, kRowsPerThread><<<1, 256, sm, st>>>(lv, s0, s1, psrc, pval, pinv, bp, xp);
    } else if (geo.y == 512) {
        sweep_kernel<VT, 512, kRowsPerThread><<<1, 512, sm, st>>>(lv, s0, s1, psrc, pval, pinv, bp, xp);
    } else {
        // 256 threads holding 8 rows each were measured 1.37x slower on the
        // natural 2048^2 triangle: each thread's rows then solve one after another
        sweep_kernel<VT, 1024, kRowsPerThread><<<1, 1024, sm, st>>>(lv, s0, s1, psrc, pval, pinv, bp, xp);
    }
}

}  // namespace

bool build_level_pack(LevelPack &pk, const int *rp, const int *ci, const void *val, const void *D, int vbytes,
                      int64_t n, const int *order, const std::vector<int> &src_begin, const std::vector<int> &count,
                      const std::vector<int> &seg_begin, bool allow_cluster, cudaStream_t st, bool row_sources) {
    const int L = (int)count.size();
    if ((int)src_begin.size() != L || (int)seg_begin.size() != L) fail(SMAX_ERR_STATE, "inconsistent sweep steps");
    pk = LevelPack();
    pk.n = n;
    pk.vbytes = vbytes;
    // the sweep kernels' shared-memory opt-in, set here and not inside a capture
    if (vbytes == 8) set_smem_attr<double>();
    else set_smem_attr<float>();
    std::vector<int> pos_begin(L + 1, 0);
    for (int s = 0; s < L; ++s) pos_begin[s + 1] = pos_begin[s] + count[s];
    if (pos_begin[L] != n) fail(SMAX_ERR_STATE, "sweep steps do not cover all rows");
    const size_t nb = sizeof(int) * (n > 0 ? n : 1);
    pk.prow.alloc(nb);
    pk.pinv.alloc((size_t)vbytes * (n > 0 ? n : 1));
    pk.row_sources = row_sources;
    // a sync-free solve reads B and writes X in the caller's numbering
    const int64_t nv = row_sources ? 1 : (n > 0 ? n : 1);
    pk.bp.alloc((size_t)vbytes * nv);
    pk.xp.alloc((size_t)vbytes * nv);
    if (n == 0 || L == 0) {
        pk.lv.alloc(sizeof(Level));
        pk.psrc.alloc(sizeof(int));
        pk.pval.alloc(vbytes);
        return true;
    }
    DevBuf d_pos(sizeof(int) * (L + 1)), d_src(sizeof(int) * L), plev(nb), pos_of_row(nb), len(nb), wmax(sizeof(int) * L);
    SMAX_CUDA(cudaMemcpyAsync(d_pos.p, pos_begin.data(), sizeof(int) * (L + 1), cudaMemcpyHostToDevice, st));
    SMAX_CUDA(cudaMemcpyAsync(d_src.p, src_begin.data(), sizeof(int) * L, cudaMemcpyHostToDevice, st));
    positions_kernel<<<grid_for(n), 256, 0, st>>>(d_pos.as<int>(), L, d_src.as<int>(), order, n, pk.prow.as<int>(),
                                                  plev.as<int>(), pos_of_row.as<int>());
    off_len_kernel<<<grid_for(n), 256, 0, st>>>(rp, pk.prow.as<int>(), n, len.as<int>());
    SMAX_CUDA(cudaGetLastError());
    size_t tb = 0;
    SMAX_CUDA(cub::DeviceSegmentedReduce::Max(nullptr, tb, len.as<int>(), wmax.as<int>(), L, d_pos.as<int>(),
                                              d_pos.as<int>() + 1, st));
    DevBuf tmp(tb);
    SMAX_CUDA(cub::DeviceSegmentedReduce::Max(tmp.p, tb, len.as<int>(), wmax.as<int>(), L, d_pos.as<int>(),
                                              d_pos.as<int>() + 1, st));
    std::vector<int> w(L);
    SMAX_CUDA(cudaMemcpyAsync(w.data(), wmax.p, sizeof(int) * L, cudaMemcpyDeviceToHost, st));
    int h_rp_end = 0;
    SMAX_CUDA(cudaMemcpyAsync(&h_rp_end, rp + n, sizeof(int), cudaMemcpyDeviceToHost, st));
    SMAX_CUDA(cudaStreamSynchronize(st));
    {
        long long padded = 0;
        for (int s = 0; s < L; ++s) padded += (long long)count[s] * (count[s] > 0 ? std::max(w[s], 0) : 0);
        const long long off = (long long)h_rp_end - n;  // off-diagonal entries
        if (padded > 3 * off + (1ll << 20) || padded >= (1ll << 31)) {
            pk = LevelPack();
            return false;
        }
    }
    pk.h_lv.resize(L);
    long long base = 0;
    std::vector<int> seg_pos(L);
    for (int s = 0; s < L; ++s) {
        const int ws = count[s] > 0 ? std::max(w[s], 0) : 0;
        pk.h_lv[s] = Level{pos_begin[s], count[s], ws, (int)base};
        base += (long long)count[s] * ws;
        if (seg_begin[s] < 0 || seg_begin[s] > s) fail(SMAX_ERR_STATE, "bad run start");
        seg_pos[s] = pos_begin[seg_begin[s]];
    }
    pk.ents = base;
    if (row_sources) {
        // warp tasks: (first position, rows | width << 6, entry stride, first entry)
        std::vector<int4> tk;
        tk.reserve((size_t)(n / 32 + L));
        for (int s = 0; s < L; ++s) {
            const Level &lv_s = pk.h_lv[s];
            if (lv_s.w >= (1 << 25)) {  // does not fit the task encoding
                pk = LevelPack();
                return false;
            }
            for (int t0 = 0; t0 < lv_s.m; t0 += 32)
                tk.push_back(make_int4(lv_s.pos + t0, std::min(32, lv_s.m - t0) | (lv_s.w << 6), lv_s.m,
                                       lv_s.base + t0));
        }
        pk.n_tasks = (int)tk.size();
        pk.tasks.alloc(sizeof(int4) * (tk.empty() ? 1 : tk.size()));
        if (!tk.empty())
            SMAX_CUDA(cudaMemcpyAsync(pk.tasks.p, tk.data(), sizeof(int4) * tk.size(), cudaMemcpyHostToDevice, st));
    }
    // launch geometry per run (steps sharing a run start), from its widest level
    pk.h_geo.assign(L, make_int2(1, 256));
    for (int s = 0; s < L;) {
        int e = s + 1, mw = count[s];
        while (e < L && seg_begin[e] == seg_begin[s]) mw = std::max(mw, count[e++]);
        const int2 g2 = run_geometry(mw, allow_cluster, vbytes);
        for (int k = s; k < e; ++k) pk.h_geo[k] = g2;
        s = e;
    }
    DevBuf d_geo(sizeof(int2) * L);
    SMAX_CUDA(cudaMemcpyAsync(d_geo.p, pk.h_geo.data(), sizeof(int2) * L, cudaMemcpyHostToDevice, st));
    pk.lv.alloc(sizeof(Level) * L);
    SMAX_CUDA(cudaMemcpyAsync(pk.lv.p, pk.h_lv.data(), sizeof(Level) * L, cudaMemcpyHostToDevice, st));
    DevBuf d_seg(sizeof(int) * L), flag(sizeof(int));
    SMAX_CUDA(cudaMemcpyAsync(d_seg.p, seg_pos.data(), sizeof(int) * L, cudaMemcpyHostToDevice, st));
    SMAX_CUDA(cudaMemsetAsync(flag.p, 0, sizeof(int), st));
    pk.psrc.alloc(sizeof(int) * (base > 0 ? base : 1));
    pk.pval.alloc((size_t)vbytes * (base > 0 ? base : 1));
    if (vbytes == 8)
        fill_kernel<double><<<grid_for(n), 256, 0, st>>>(
            rp, ci, static_cast<const double *>(val), static_cast<const double *>(D), n, pk.prow.as<int>(),
            plev.as<int>(), pos_of_row.as<int>(), pk.lv.as<Level>(), d_seg.as<int>(), d_geo.as<int2>(),
            pk.psrc.as<int>(), pk.pval.as<double>(), pk.pinv.as<double>(), flag.as<int>(), row_sources);
    else
        fill_kernel<float><<<grid_for(n), 256, 0, st>>>(
            rp, ci, static_cast<const float *>(val), static_cast<const float *>(D), n, pk.prow.as<int>(),
            plev.as<int>(), pos_of_row.as<int>(), pk.lv.as<Level>(), d_seg.as<int>(), d_geo.as<int2>(),
            pk.psrc.as<int>(), pk.pval.as<float>(), pk.pinv.as<float>(), flag.as<int>(), row_sources);
    SMAX_CUDA(cudaGetLastError());
    int h_flag = 0;
    SMAX_CUDA(cudaMemcpyAsync(&h_flag, flag.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    SMAX_CUDA(cudaStreamSynchronize(st));  // the temporaries die here
    pk.needs_x_init = h_flag != 0;
    return true;
}

template <typename VT>
void pack_solve(const LevelPack &pk, const std::vector<PackStep> &steps, const VT *B, VT *X, cudaStream_t st) {
    if (pk.n == 0) return;
    set_smem_attr<VT>();
    const int *prow = pk.prow.as<int>();
    VT *bp = pk.bp.as<VT>(), *xp = pk.xp.as<VT>();
    gather_kernel<VT><<<grid_for(pk.n), 256, 0, st>>>(prow, pk.n, B, bp, X, pk.needs_x_init ? xp : nullptr);
    const int *psrc = pk.psrc.as<int>();
    const VT *pval = pk.pval.as<VT>(), *pinv = pk.pinv.as<VT>();
    for (const PackStep &s : steps) {
        if (s.kind == 0) {
            for (int l = s.first; l < s.first + s.count; ++l) {
                const Level &L = pk.h_lv[l];
                if (L.m > 0)
                    wide_level_kernel<VT><<<ceil_div_u(L.m, 256), 256, 0, st>>>(L, psrc, pval, pinv, bp, xp);
            }
        } else {
            launch_run<VT>(pk, s.first, s.first + s.count, psrc, pval, pinv, bp, xp, st);
        }
    }
    scatter_kernel<VT><<<grid_for(pk.n), 256, 0, st>>>(prow, pk.n, xp, X);
    SMAX_CUDA(cudaGetLastError());
}

template <typename VT>
void pack_solve_batch(const LevelPack &pk, const int *mat_steps, const int *queue_order, int n_mats, int *queue,
                      const VT *B, VT *X, cudaStream_t st) {
    if (pk.n == 0 || n_mats == 0) return;
    set_smem_attr<VT>();
    const int *prow = pk.prow.as<int>();
    VT *bp = pk.bp.as<VT>(), *xp = pk.xp.as<VT>();
    gather_kernel<VT><<<grid_for(pk.n), 256, 0, st>>>(prow, pk.n, B, bp, X, pk.needs_x_init ? xp : nullptr);
    int threads = 256;
    for (const int2 &g2 : pk.h_geo) threads = std::max(threads, g2.y);
    // one CTA per matrix at a time: as many CTAs as fit (the ring limits residency)
    const int per_sm = threads <= 512 ? 2 : 1;
    const int grid = std::max(1, std::min(n_mats, per_sm * sm_count()));
    SMAX_CUDA(cudaMemsetAsync(queue, 0, sizeof(int), st));
    const size_t sm = kRing * sizeof(VT);
    const Level *lv = pk.lv.as<Level>();
    const int *psrc = pk.psrc.as<int>();
    const VT *pval = pk.pval.as<VT>(), *pinv = pk.pinv.as<VT>();
    if (threads == 256)
        sweep_batch_kernel<VT, 256><<<grid, 256, sm, st>>>(lv, mat_steps, queue_order, n_mats, queue, psrc, pval,
                                                            pinv, bp, xp);
    else if (threads == 512)
        sweep_batch_kernel<VT, 512><<<grid, 512, sm, st>>>(lv, mat_steps, queue_order, n_mats, queue, psrc, pval,
                                                            pinv, bp, xp);
    else
        sweep_batch_kernel<VT, 1024><<<grid, 1024, sm, st>>>(lv, mat_steps, queue_order, n_mats, queue, psrc, pval,
                                                              pinv, bp, xp);
    scatter_kernel<VT><<<grid_for(pk.n), 256, 0, st>>>(prow, pk.n, xp, X);
    SMAX_CUDA(cudaGetLastError());
}

template <typename VT>
void pack_solve_syncfree(const LevelPack &pk, const VT *B, VT *X, void *ctl, long long limit, bool force_timeout,
                         DevStatus *st, cudaStream_t s) {
    if (pk.n == 0) return;
    if (!pk.row_sources) fail(SMAX_ERR_STATE, "the sync-free solve needs a row-sourced pack");
    int *c = static_cast<int *>(ctl);
    sf_reset_kernel<VT><<<grid_for(pk.n), 256, 0, s>>>(X, pk.n, c);
    static int per_sm_cache[64] = {};
    int dev = 0;
    SMAX_CUDA(cudaGetDevice(&dev));
    int per_sm = dev >= 0 && dev < 64 ? per_sm_cache[dev] : 0;
    if (per_sm == 0) {
        SMAX_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, syncfree_kernel<VT>, kSfThreads, 0));
        if (per_sm < 1) per_sm = 1;
        if (dev >= 0 && dev < 64) per_sm_cache[dev] = per_sm;
    }
    const int chunks = (pk.n_tasks + kSfChunk - 1) / kSfChunk;
    // deep, narrow schedules: about four levels' rows in flight, so waiting
    // warps do not flood L2 with polls
    const int64_t avg = pk.n / std::max(1, pk.n_levels());
    const int64_t cap = std::max<int64_t>(8, (4 * avg + kSfThreads - 1) / kSfThreads);
    const int grid = (int)std::max<int64_t>(1, std::min<int64_t>({(int64_t)chunks, (int64_t)per_sm * sm_count(), cap}));
    syncfree_kernel<VT><<<grid, kSfThreads, 0, s>>>(pk.tasks.as<int4>(), pk.n_tasks, pk.prow.as<int>(),
                                                    pk.psrc.as<int>(), pk.pval.as<VT>(), pk.pinv.as<VT>(), B, X, c,
                                                    limit, force_timeout, st);
    SMAX_CUDA(cudaGetLastError());
}

template <typename VT>
void solve_syncfree_rows(const LevelPack &pk, const int *rp, const int *ci, const VT *val, const VT *D, const VT *B,
                         VT *X, int64_t k, bool row_major, void *ctl, long long limit, DevStatus *st, cudaStream_t s) {
    if (pk.n == 0 || k == 0) return;
    if (!pk.row_sources) fail(SMAX_ERR_STATE, "the sync-free solve needs a row-sourced pack");
    int *c = static_cast<int *>(ctl);
    sf_reset_kernel<VT><<<grid_for(pk.n * k), 256, 0, s>>>(X, pk.n * k, c);
    static int per_sm_cache[64] = {};
    int dev = 0;
    SMAX_CUDA(cudaGetDevice(&dev));
    int per_sm = dev >= 0 && dev < 64 ? per_sm_cache[dev] : 0;
    if (per_sm == 0) {
        SMAX_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, syncfree_rows_kernel<VT>, kSfThreads, 0));
        if (per_sm < 1) per_sm = 1;
        if (dev >= 0 && dev < 64) per_sm_cache[dev] = per_sm;
    }
    constexpr int rows_per_claim = kSfThreads / 32;
    const int64_t claims = (pk.n + rows_per_claim - 1) / rows_per_claim;
    // about four levels' rows in flight, as for one right-hand side
    const int64_t avg = pk.n / std::max(1, pk.n_levels());
    const int64_t cap = std::max<int64_t>(8, (4 * avg + rows_per_claim - 1) / rows_per_claim);
    const int grid = (int)std::max<int64_t>(1, std::min<int64_t>({claims, (int64_t)per_sm * sm_count(), cap}));
    // column-major blocks: the leading dimension is the matrix's row count
    const int64_t rs = row_major ? k : 1, vs = row_major ? 1 : pk.n;
    syncfree_rows_kernel<VT><<<grid, kSfThreads, 0, s>>>(pk.prow.as<int>(), (int)pk.n, rp, ci, val, D, B, X, k, rs, vs, c,
                                                         limit, st);
    SMAX_CUDA(cudaGetLastError());
}

template void solve_syncfree_rows<double>(const LevelPack &, const int *, const int *, const double *,
                                          const double *, const double *, double *, int64_t, bool, void *, long long,
                                          DevStatus *, cudaStream_t);
template void solve_syncfree_rows<float>(const LevelPack &, const int *, const int *, const float *, const float *,
                                         const float *, float *, int64_t, bool, void *, long long, DevStatus *,
                                         cudaStream_t);
template void pack_solve_syncfree<double>(const LevelPack &, const double *, double *, void *, long long, bool,
                                          DevStatus *, cudaStream_t);
template void pack_solve_syncfree<float>(const LevelPack &, const float *, float *, void *, long long, bool,
                                         DevStatus *, cudaStream_t);
template void pack_solve<double>(const LevelPack &, const std::vector<PackStep> &, const double *, double *,
                                 cudaStream_t);
template void pack_solve<float>(const LevelPack &, const std::vector<PackStep> &, const float *, float *,
                                cudaStream_t);
template void pack_solve_batch<double>(const LevelPack &, const int *, const int *, int, int *, const double *,
                                       double *, cudaStream_t);
template void pack_solve_batch<float>(const LevelPack &, const int *, const int *, int, int *, const float *, float *,
                                      cudaStream_t);

}  // namespace smax
