// spmv_crs_stream.cu -- CRS SpMV, warp-stream variant (the default on sm_100a).
//
// Reference semantics: SPMV::CPU::naive_crs_spmv
// (src/kernels/spmv/spmv_cpu/spmv_cpu_crs_impl.hpp:9-38): y[i] = sum_j val[j]*x[col[j]].
//
// Design.  The nnz range is cut into fixed slices of W = 512 entries; warp t
// owns slice t, so every warp streams exactly the same number of bytes no
// matter how row lengths are distributed.  A slice is read in chunks of
// 32*U entries, each lane taking U consecutive entries with 128-bit,
// evict-first loads of col and val (the arrays are padded to a multiple of W
// at upload, so the loop has no bounds checks).  Row boundaries come from a
// bit mask built once per matrix: bit e is set when entry e is the last entry
// of its row.  Each lane sums its U products with resets at its row ends; a
// warp-wide segmented scan (shuffles) carries the open partial sum across
// lanes and chunks, and every row that ends inside the slice is written by
// the lane holding its last entry.  The sum a slice holds for the row still
// open at its end is written to carry[t]; a small fix-up pass then adds each
// run of carries to its row in task order (deterministic).  When no row has
// more than 32 entries, a slice instead sums the head of its first row (the
// entries before the slice, at most 31) itself, one entry per lane, and
// neither carries nor the fix-up launch are needed.  Rows without
// entries get y = 0 from a separate list.  HBM traffic: val, col, one bit per
// entry, one int per 512 entries, y; x is gathered through L2.
#include "spmv_crs.cuh"

#include <cub/device/device_reduce.cuh>
#include <cub/device/device_select.cuh>
#include <thrust/iterator/counting_iterator.h>

namespace smax {

namespace {

constexpr int kW = 512;          // entries per warp task
constexpr int kWarpsPerCta = 8;  // 256-thread CTAs

template <typename VT> struct StreamCfg;
template <> struct StreamCfg<double> { static constexpr int U = 4; };
// FP32 lanes take four entries too (16-byte column and value loads): with
// eight, each lane held eight gathers in flight and registers cost occupancy
template <> struct StreamCfg<float> { static constexpr int U = 4; };

// U consecutive entries of col and val starting at a multiple of U.
template <typename VT, int U> struct Chunk;
template <> struct Chunk<double, 4> {
    int c[4];
    double v[4];
    __device__ __forceinline__ void load(const int *col, const double *val, int64_t e) {
        int4 ci = __ldcs(reinterpret_cast<const int4 *>(col + e));
        double2 a = __ldcs(reinterpret_cast<const double2 *>(val + e));
        double2 b = __ldcs(reinterpret_cast<const double2 *>(val + e + 2));
        c[0] = ci.x; c[1] = ci.y; c[2] = ci.z; c[3] = ci.w;
        v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y;
    }
};
template <> struct Chunk<float, 4> {
    int c[4];
    float v[4];
    __device__ __forceinline__ void load(const int *col, const float *val, int64_t e) {
        int4 ci = __ldcs(reinterpret_cast<const int4 *>(col + e));
        float4 a = __ldcs(reinterpret_cast<const float4 *>(val + e));
        c[0] = ci.x; c[1] = ci.y; c[2] = ci.z; c[3] = ci.w;
        v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w;
    }
};

__device__ __forceinline__ int row_of_rank(const int *row_list, int q) { return row_list ? row_list[q] : q; }

// Sum over the entries [rs, base) of the row open at a slice start, one entry
// per lane (base - rs < 32), reduced in a fixed lane order.
template <typename VT>
__device__ __forceinline__ VT head_sum(const int *__restrict__ col, const VT *__restrict__ val,
                                       const VT *__restrict__ x, int64_t rs, int64_t base, int lane) {
    VT h = VT(0);
    if (rs + lane < base) h = __ldg(val + rs + lane) * __ldcg(x + __ldg(col + rs + lane));
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) h += __shfl_xor_sync(0xffffffffu, h, o);
    return h;
}

template <typename VT, bool SHORT>
__global__ void __launch_bounds__(kWarpsPerCta * 32)
    crs_stream_kernel(const int *__restrict__ col, const VT *__restrict__ val,
                      const uint32_t *__restrict__ endbits, const int *__restrict__ task_rank,
                      const int *__restrict__ row_list, const int *__restrict__ row_ptr, int64_t n_tasks,
                      int n_nonempty, const VT *__restrict__ x, VT *__restrict__ y, VT *__restrict__ carry_val,
                      int *__restrict__ carry_rank) {
    constexpr int U = StreamCfg<VT>::U;
    constexpr int CH = 32 * U;  // entries per chunk
    constexpr int NC = kW / CH; // chunks per task
    constexpr unsigned MASK = (1u << U) - 1u;
    const int lane = threadIdx.x & 31;
    const int64_t t = (int64_t)blockIdx.x * kWarpsPerCta + (threadIdx.x >> 5);
    if (t >= n_tasks) return;  // uniform per warp
    const int64_t base = t * kW;
    int q = task_rank[t];      // rank (among non-empty rows) of the row open at the slice start
    VT carry = VT(0);          // partial sum of the open row, from this slice only (SHORT: the whole row)

    Chunk<VT, U> cur;
    int64_t e0 = base + lane * U;
    cur.load(col, val, e0);
    uint32_t word = endbits[e0 >> 5];
    // SHORT: every row has at most 32 entries, so the open row ends in this
    // slice and at most 31 of its entries lie before it
    if constexpr (SHORT) carry = head_sum(col, val, x, (int64_t)row_ptr[row_of_rank(row_list, q)], base, lane);

#pragma unroll
    for (int k = 0; k < NC; ++k) {
        // prefetch the next chunk while this one is reduced
        Chunk<VT, U> nxt;
        uint32_t nword = 0;
        if (k + 1 < NC) {
            nxt.load(col, val, e0 + CH);
            nword = endbits[(e0 + CH) >> 5];
        }
        const unsigned nib = (word >> (unsigned)(e0 & 31)) & MASK;

        VT p[U];
#pragma unroll
        for (int i = 0; i < U; ++i) p[i] = cur.v[i] * __ldcg(x + cur.c[i]);  // L2 only: x lines are not reused in L1

        const int nend = __popc(nib);
        int incl = nend;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            int v = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += v;
        }
        const int excl = incl - nend;
        const int total_ends = __shfl_sync(0xffffffffu, incl, 31);

        // local segments: head (up to and including the first end), complete
        // rows inside the lane, and the open tail after the last end
        VT run = VT(0), head = VT(0);
        int ri = 0;
#pragma unroll
        for (int i = 0; i < U; ++i) {
            run += p[i];
            if ((nib >> i) & 1u) {
                if (ri == 0) head = run;
                else st_stream(y + row_of_rank(row_list, q + excl + ri), run);
                run = VT(0);
                ++ri;
            }
        }

        // segmented inclusive scan of (v, f) over lanes:
        // (v1,f1) then (v2,f2) -> (f2 ? v2 : v1 + v2, f1 | f2)
        VT sv = run;  // tail if the lane has an end, else its whole sum
        int sf = nend > 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            VT vu = __shfl_up_sync(0xffffffffu, sv, o);
            int fu = __shfl_up_sync(0xffffffffu, sf, o);
            if (lane >= o) {
                if (!sf) sv += vu;
                sf |= fu;
            }
        }
        VT ev = __shfl_up_sync(0xffffffffu, sv, 1);
        int ef = __shfl_up_sync(0xffffffffu, sf, 1);
        if (lane == 0) { ev = VT(0); ef = 0; }
        const VT cin = ef ? ev : carry + ev;
        if (nend) st_stream(y + row_of_rank(row_list, q + excl), cin + head);

        const VT v31 = __shfl_sync(0xffffffffu, sv, 31);
        const int f31 = __shfl_sync(0xffffffffu, sf, 31);
        carry = f31 ? v31 : carry + v31;
        q += total_ends;

        if (k + 1 < NC) {
            cur = nxt;
            word = nword;
            e0 += CH;
        }
    }
    if (!SHORT && lane == 0) {
        carry_val[t] = carry;
        carry_rank[t] = q < n_nonempty ? q : -1;
    }
}

// y[row] += the run of carries of one row, summed in task order.
template <typename VT>
__global__ void crs_stream_fixup(const VT *__restrict__ carry_val, const int *__restrict__ carry_rank,
                                 const int *__restrict__ row_list, int64_t n_tasks, VT *__restrict__ y) {
    int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n_tasks) return;
    const int q = carry_rank[t];
    if (q < 0 || (t > 0 && carry_rank[t - 1] == q)) return;
    VT s = VT(0);
    for (int64_t u = t; u < n_tasks && carry_rank[u] == q; ++u) s += carry_val[u];
    y[row_of_rank(row_list, q)] += s;
}

template <typename VT>
__global__ void zero_rows(const int *__restrict__ rows, int64_t n, VT *__restrict__ y) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) y[rows[i]] = VT(0);
}

__global__ void row_flags_kernel(const int *__restrict__ row_ptr, int64_t n, unsigned char *__restrict__ empty,
                                 unsigned char *__restrict__ nonempty, uint32_t *__restrict__ endbits,
                                 int *__restrict__ max_len) {
    int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n) return;
    const int s = row_ptr[r], e = row_ptr[r + 1];
    const bool em = e == s;
    empty[r] = em;
    nonempty[r] = !em;
    if (!em) atomicOr(endbits + ((e - 1) >> 5), 1u << ((e - 1) & 31));
    if (e - s > 32) atomicMax(max_len, e - s);  // only "more than 32" matters
}

// rank of the row holding entry t*W: the largest r with row_ptr[r] <= t*W
// (that row is non-empty), then its position among the non-empty rows.
__global__ void task_rank_kernel(const int *__restrict__ row_ptr, int64_t n, const int *__restrict__ row_list,
                                 int64_t n_nonempty, int64_t n_tasks, int *__restrict__ task_rank) {
    int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n_tasks) return;
    const int64_t e = t * kW;
    int64_t lo = 0, hi = n;  // upper_bound over row_ptr[0..n]
    while (lo < hi) {
        int64_t mid = (lo + hi) >> 1;
        if ((int64_t)row_ptr[mid] <= e) lo = mid + 1; else hi = mid;
    }
    int64_t r = lo - 1;
    if (row_list) {
        int64_t a = 0, b = n_nonempty;  // lower_bound of r in row_list
        while (a < b) {
            int64_t m = (a + b) >> 1;
            if (row_list[m] < r) a = m + 1; else b = m;
        }
        r = a;
    }
    task_rank[t] = (int)r;
}

}  // namespace

int crs_stream_pad() { return kW; }

void CrsStreamPlan::build(const int *d_row_ptr, int64_t n, int64_t nnz_, int vbytes, cudaStream_t st) {
    n_rows = n;
    nnz = nnz_;
    n_tasks = (nnz + kW - 1) / kW;
    int64_t words = (n_tasks * kW) / 32 + 1;
    endbits.alloc(sizeof(uint32_t) * words);
    SMAX_CUDA(cudaMemsetAsync(endbits.p, 0, endbits.bytes, st));
    n_empty = 0;
    n_nonempty = 0;
    row_ptr = d_row_ptr;
    short_rows = true;
    if (n > 0) {
        DevBuf fe(n), fne(n), cnt(sizeof(int) * 3);
        SMAX_CUDA(cudaMemsetAsync(cnt.p, 0, cnt.bytes, st));
        row_flags_kernel<<<ceil_div_u(n, 256), 256, 0, st>>>(d_row_ptr, n, fe.as<unsigned char>(),
                                                             fne.as<unsigned char>(), endbits.as<uint32_t>(),
                                                             cnt.as<int>() + 2);
        SMAX_CUDA(cudaGetLastError());
        thrust::counting_iterator<int> it(0);
        empty_rows.alloc(sizeof(int) * n);
        size_t tb = 0;
        SMAX_CUDA(cub::DeviceSelect::Flagged(nullptr, tb, it, fe.as<unsigned char>(), empty_rows.as<int>(),
                                             cnt.as<int>(), (int)n, st));
        DevBuf tmp(tb);
        SMAX_CUDA(cub::DeviceSelect::Flagged(tmp.p, tb, it, fe.as<unsigned char>(), empty_rows.as<int>(),
                                             cnt.as<int>(), (int)n, st));
        int h[3] = {0, 0, 0};
        SMAX_CUDA(cudaMemcpyAsync(h, cnt.p, sizeof(h), cudaMemcpyDeviceToHost, st));
        SMAX_CUDA(cudaStreamSynchronize(st));
        n_empty = h[0];
        short_rows = h[2] == 0;
        n_nonempty = n - n_empty;
        if (n_empty > 0) {
            row_list.alloc(sizeof(int) * (n_nonempty > 0 ? n_nonempty : 1));
            SMAX_CUDA(cub::DeviceSelect::Flagged(tmp.p, tb, it, fne.as<unsigned char>(), row_list.as<int>(),
                                                 cnt.as<int>() + 1, (int)n, st));
        } else {
            empty_rows.release();
            row_list.release();
        }
        SMAX_CUDA(cudaStreamSynchronize(st));
    }
    task_rank.alloc(sizeof(int) * (n_tasks > 0 ? n_tasks : 1));
    carry_rank.alloc(sizeof(int) * (n_tasks > 0 ? n_tasks : 1));
    carry_val.alloc((size_t)vbytes * (n_tasks > 0 ? n_tasks : 1));
    if (n_tasks > 0) {
        task_rank_kernel<<<ceil_div_u(n_tasks, 256), 256, 0, st>>>(
            d_row_ptr, n, row_list.p ? row_list.as<int>() : nullptr, n_nonempty, n_tasks, task_rank.as<int>());
        SMAX_CUDA(cudaGetLastError());
    }
    SMAX_CUDA(cudaStreamSynchronize(st));
}

template <typename VT>
void crs_spmv_stream(const CrsStreamPlan &p, const int *col, const VT *val, const VT *x, VT *y, cudaStream_t st) {
    const int *rl = p.row_list.p ? p.row_list.as<int>() : nullptr;
    if (p.n_tasks > 0) {
        unsigned grid = ceil_div_u(p.n_tasks, kWarpsPerCta);
        auto launch = [&](auto kern) {
            kern<<<grid, kWarpsPerCta * 32, 0, st>>>(col, val, p.endbits.as<uint32_t>(), p.task_rank.as<int>(), rl,
                                                     p.row_ptr, p.n_tasks, (int)p.n_nonempty, x, y,
                                                     p.carry_val.as<VT>(), p.carry_rank.as<int>());
            SMAX_CUDA(cudaGetLastError());
        };
        if (p.short_rows) {
            launch(crs_stream_kernel<VT, true>);  // no carries: one launch
        } else {
            launch(crs_stream_kernel<VT, false>);
            crs_stream_fixup<VT><<<ceil_div_u(p.n_tasks, 256), 256, 0, st>>>(
                p.carry_val.as<VT>(), p.carry_rank.as<int>(), rl, p.n_tasks, y);
            SMAX_CUDA(cudaGetLastError());
        }
    }
    if (p.n_empty > 0) {
        zero_rows<VT><<<ceil_div_u(p.n_empty, 256), 256, 0, st>>>(p.empty_rows.as<int>(), p.n_empty, y);
        SMAX_CUDA(cudaGetLastError());
    }
}

template void crs_spmv_stream<double>(const CrsStreamPlan &, const int *, const double *, const double *, double *,
                                      cudaStream_t);
template void crs_spmv_stream<float>(const CrsStreamPlan &, const int *, const float *, const float *, float *,
                                     cudaStream_t);

}  // namespace smax
