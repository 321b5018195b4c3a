// spmv_scs.cu -- SELL-C-sigma SpMV and CRS -> SELL-C-sigma conversion on sm_100a.
//
// Layout (the reference's, src/common.hpp:62-88 and src/utils/convert_formats.hpp:16-132):
// chunk c holds rows c*C .. c*C+C-1 of the sigma-sorted order; entry j of
// chunk-row i sits at chunk_ptr[c] + j*C + i; padded entries are col 0 / val 0;
// y is produced in the permuted order (y[perm[r]] is row r of the CRS product).
//
// SpMV (SPMV::CPU::naive_scs_spmv, src/kernels/spmv/spmv_cpu/spmv_cpu_scs_impl.hpp:9-49):
//   * C a multiple of VEC (rows per lane, scs_vec: 1 or 2) and C/VEC <= 32: warp tasks of at
//     most kScsTaskCols chunk columns (a long chunk -- sigma sorting puts the
//     longest rows together -- is split over several warps, whose partial
//     sums a fix-up pass adds in task order, so no warp holds a long tail);
//     each lane owns VEC adjacent rows and reads them with one load per
//     chunk column, so C/VEC lanes cover a chunk column and the warp covers
//     32*VEC/C columns per instruction (chunk-column-major, fully coalesced);
//     the lanes holding the same rows combine with shuffles at the end and y is
//     stored with vector stores.
//   * any other C: one thread per row, consecutive threads on consecutive rows.
//
// Conversion (Utils::convert_crs_to_scs): row lengths, a per-sigma-window sort
// by descending length that leaves rows of equal length in exactly the order
// the reference's std::sort leaves them (scs_window_sort.cuh), chunk lengths
// as the chunk's maximum, chunk_ptr by scan, perm[old] = new, and a scatter
// of col/val into the zero-filled chunk-column-major arrays -- all on the GPU.
// perm, col and val are therefore bit-exact with the reference's for every
// sigma, not only where ties cannot occur.
#include "spmv_formats.cuh"
#include "scs_window_sort.cuh"

#include <vector>

#include <cub/device/device_scan.cuh>

namespace smax {

namespace {

// Rows per lane (VEC): FP64 lanes own one row when a chunk column fits in a
// warp (C <= 32; two rows, 16-byte loads, for C = 64), FP32 lanes two rows
// (8-byte loads).  More rows per lane put more gathers in flight per lane,
// and the registers that costs lost occupancy (FP32 with four rows: 0.440 ms
// against 0.398 ms on the lognormal 2^22 matrix).
int scs_vec(int64_t C, int vbytes) { return vbytes == 8 ? (C <= 32 ? 1 : 2) : 2; }

// VEC adjacent values / column indices from p (8-byte aligned for VEC == 2)
template <typename VT, int VEC> __device__ __forceinline__ void load_vals(const VT *p, VT *o) {
    static_assert(VEC == 1 || VEC == 2, "one or two rows per lane");
    if constexpr (VEC == 1) {
        o[0] = __ldcs(p);
    } else if constexpr (sizeof(VT) == 8) {
        const double2 t = __ldcs(reinterpret_cast<const double2 *>(p));
        o[0] = t.x;
        o[1] = t.y;
    } else {
        const float2 t = __ldcs(reinterpret_cast<const float2 *>(p));
        o[0] = t.x;
        o[1] = t.y;
    }
}
template <int VEC> __device__ __forceinline__ void load_cols(const int *p, int *o) {
    if constexpr (VEC == 1) {
        o[0] = __ldcs(p);
    } else {
        const int2 t = __ldcs(reinterpret_cast<const int2 *>(p));
        o[0] = t.x;
        o[1] = t.y;
    }
}
template <typename VT, int VEC> __device__ __forceinline__ void store_vals(VT *p, const VT *a) {
    if constexpr (VEC == 1) {
        __stcs(p, a[0]);
    } else if constexpr (sizeof(VT) == 8) {
        __stcs(reinterpret_cast<double2 *>(p), make_double2(a[0], a[1]));
    } else {
        __stcs(reinterpret_cast<float2 *>(p), make_float2(a[0], a[1]));
    }
}

// one warp per chunk; LPC = C / VEC lanes per chunk column
template <typename VT, int LPC, int VEC>
__global__ void __launch_bounds__(256) scs_warp_kernel(const int *__restrict__ chunk_ptr,
                                                       const int *__restrict__ chunk_len, int64_t n_chunks,
                                                       const int *__restrict__ col, const VT *__restrict__ val,
                                                       const VT *__restrict__ x, VT *__restrict__ y) {
    constexpr int C = LPC * VEC;
    constexpr int CPI = 32 / LPC;  // chunk columns per warp instruction
    const int lane = threadIdx.x & 31;
    const int64_t c = (int64_t)blockIdx.x * 8 + (threadIdx.x >> 5);
    if (c >= n_chunks) return;
    const int64_t cs = chunk_ptr[c];
    const int len = chunk_len[c];
    const int sub = lane % LPC;  // which VEC rows of the chunk
    const int j0 = lane / LPC;   // first chunk column of this lane
    VT acc[VEC];
#pragma unroll
    for (int i = 0; i < VEC; ++i) acc[i] = VT(0);
    for (int j = j0; j < len; j += CPI) {
        const int64_t idx = cs + (int64_t)j * C + sub * VEC;
        VT v[VEC];
        load_vals<VT, VEC>(val + idx, v);
        int cc[VEC];
        load_cols<VEC>(col + idx, cc);
#pragma unroll
        for (int i = 0; i < VEC; ++i) acc[i] += v[i] * ld_keep(x + cc[i]);
    }
    // lanes with the same `sub` hold partial sums of the same rows
#pragma unroll
    for (int o = LPC; o < 32; o <<= 1)
#pragma unroll
        for (int i = 0; i < VEC; ++i) acc[i] += __shfl_xor_sync(0xffffffffu, acc[i], o);
    if (j0 == 0) store_vals<VT, VEC>(y + c * C + sub * VEC, acc);
}

// One warp per task: chunk columns [j0, min(len, j0 + kScsTaskCols)) of one
// chunk, unrolled four instructions deep so the gathers of several columns
// are in flight together.
template <typename VT, int LPC, int VEC>
__global__ void __launch_bounds__(256) scs_task_kernel(const int *__restrict__ chunk_ptr,
                                                       const int *__restrict__ chunk_len,
                                                       const int *__restrict__ task_chunk,
                                                       const int *__restrict__ task_j0,
                                                       const int *__restrict__ task_slot, int64_t n_tasks,
                                                       const int *__restrict__ col, const VT *__restrict__ val,
                                                       const VT *__restrict__ x, VT *__restrict__ y,
                                                       VT *__restrict__ partial, const int *__restrict__ row_len) {
    constexpr int C = LPC * VEC;
    constexpr int CPI = 32 / LPC;  // chunk columns per warp instruction
    const int lane = threadIdx.x & 31;
    const int64_t t = (int64_t)blockIdx.x * 8 + (threadIdx.x >> 5);
    if (t >= n_tasks) return;
    const int c = task_chunk[t];
    const int jt = task_j0[t];
    const int slot = task_slot[t];
    const int64_t cs = chunk_ptr[c];
    const int jl = min(chunk_len[c], jt + kScsTaskCols);
    const int sub = lane % LPC;
    VT acc[VEC];
#pragma unroll
    for (int i = 0; i < VEC; ++i) acc[i] = VT(0);
    // Entries past a row's last stored entry are the layout's padding
    // (column 0, value 0): their products 0 * x[0] add nothing when x[0] is
    // finite, so the lane neither loads them nor gathers for them -- the
    // sectors of a column that hold only padding are not fetched.  With a
    // non-finite x[0] every stored entry is used, as the reference does.
    int rl[VEC], rlmax = 0x7fffffff;
#pragma unroll
    for (int i = 0; i < VEC; ++i) rl[i] = 0x7fffffff;
    if (row_len && isfinite(__ldg(x))) {
        rlmax = 0;
#pragma unroll
        for (int i = 0; i < VEC; ++i) {
            rl[i] = row_len[(int64_t)c * C + sub * VEC + i];
            rlmax = max(rlmax, rl[i]);
        }
    }
    int j = jt + lane / LPC;
    auto step = [&](int jj) {
        if (jj >= rlmax) return;
        const int64_t idx = cs + (int64_t)jj * C + sub * VEC;
        VT v[VEC];
        load_vals<VT, VEC>(val + idx, v);
        int cc[VEC];
        load_cols<VEC>(col + idx, cc);
#pragma unroll
        for (int i = 0; i < VEC; ++i)
            if (jj < rl[i]) acc[i] += v[i] * __ldcg(x + cc[i]);
    };
    for (; j + 3 * CPI < jl; j += 4 * CPI) {
        // four columns' loads first, then their products in column order
        const int64_t i0 = cs + (int64_t)j * C + sub * VEC;
        VT v[4][VEC];
        int cc[4][VEC];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int64_t idx = i0 + (int64_t)u * CPI * C;
            if (j + u * CPI < rlmax) {
                load_vals<VT, VEC>(val + idx, v[u]);
                load_cols<VEC>(col + idx, cc[u]);
            } else {
#pragma unroll
                for (int i = 0; i < VEC; ++i) {
                    v[u][i] = VT(0);
                    cc[u][i] = 0;
                }
            }
        }
        VT xv[4][VEC];
#pragma unroll
        for (int u = 0; u < 4; ++u)
#pragma unroll
            for (int i = 0; i < VEC; ++i) xv[u][i] = j + u * CPI < rl[i] ? __ldcg(x + cc[u][i]) : VT(0);
#pragma unroll
        for (int u = 0; u < 4; ++u)
#pragma unroll
            for (int i = 0; i < VEC; ++i)
                if (j + u * CPI < rl[i]) acc[i] += v[u][i] * xv[u][i];
    }
    for (; j < jl; j += CPI) step(j);
#pragma unroll
    for (int o = LPC; o < 32; o <<= 1)
#pragma unroll
        for (int i = 0; i < VEC; ++i) acc[i] += __shfl_xor_sync(0xffffffffu, acc[i], o);
    if (lane < LPC) {
        VT *dst = slot < 0 ? y + (int64_t)c * C : partial + (int64_t)slot * C;
        store_vals<VT, VEC>(dst + sub * VEC, acc);
    }
}

// y rows of a split chunk = its tasks' partial sums, added in task order
template <typename VT>
__global__ void scs_fixup_kernel(const int *__restrict__ multi_chunk, const int *__restrict__ multi_first,
                                 const int *__restrict__ multi_count, int64_t n_multi, int C,
                                 const VT *__restrict__ partial, VT *__restrict__ y) {
    const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= n_multi * C) return;
    const int64_t m = g / C;
    const int i = (int)(g % C);
    const int f = multi_first[m], k = multi_count[m];
    VT s = VT(0);
    for (int p = 0; p < k; ++p) s += partial[(int64_t)(f + p) * C + i];
    y[(int64_t)multi_chunk[m] * C + i] = s;
}

// generic: one thread per (padded) row
template <typename VT>
__global__ void scs_thread_kernel(const int *__restrict__ chunk_ptr, const int *__restrict__ chunk_len, int64_t C,
                                  int64_t n_rows_padded, const int *__restrict__ col, const VT *__restrict__ val,
                                  const VT *__restrict__ x, VT *__restrict__ y) {
    const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n_rows_padded) return;
    const int64_t c = r / C, i = r % C;
    const int64_t cs = chunk_ptr[c];
    const int len = chunk_len[c];
    VT acc = VT(0);
    for (int j = 0; j < len; ++j) {
        const int64_t idx = cs + (int64_t)j * C + i;
        acc += ld_stream(val + idx) * ld_keep(x + ld_stream(col + idx));
    }
    y[r] = acc;
}

// ----------------------------------------------------------- conversion ----
__global__ void scs_keys_kernel(const int *__restrict__ row_ptr, int64_t n, int64_t npad,
                                unsigned long long *__restrict__ keys) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= npad) return;
    const unsigned cnt = i < n ? (unsigned)(row_ptr[i + 1] - row_ptr[i]) : 0u;
    // high half orders longer rows first (the reference compares counts only);
    // the low half carries the row through the sort
    keys[i] = ((unsigned long long)(0x7fffffffu - cnt) << 32) | (unsigned long long)i;
}

// One sigma window per single-thread block, ordered exactly as the
// reference's std::sort orders it (scs_window_sort.cuh).  A single thread per
// block keeps the data-dependent loops free of warp divergence; as many
// windows share an SM as its block slots and shared memory allow (7 staged
// windows of 4096 keys).  SMEM: the window is staged in shared memory
// (windows of up to kScsSortSmemKeys keys), else it is sorted in place in `out`.
constexpr int64_t kScsSortSmemKeys = 4096;  // 32 KB of keys per block

template <bool SMEM>
__global__ void __launch_bounds__(1) scs_window_sort_kernel(const unsigned long long *__restrict__ keys,
                                                            unsigned long long *__restrict__ out, int64_t npad,
                                                            int64_t sigma, int *__restrict__ err) {
    extern __shared__ unsigned long long win[];
    const int64_t lo = (int64_t)blockIdx.x * sigma;
    const int64_t len = (lo + sigma < npad ? lo + sigma : npad) - lo;
    unsigned long long *a = SMEM ? win : out + lo;
    for (int64_t i = 0; i < len; ++i) a[i] = keys[lo + i];
    if (!scs_sort::std_sort_order(a, len)) atomicExch(err, 1);
    if (SMEM)
        for (int64_t i = 0; i < len; ++i) out[lo + i] = a[i];
}

// chunk lengths (max row length in the chunk) and perm[old] = new
__global__ void scs_chunks_kernel(const unsigned long long *__restrict__ sorted, int64_t n, int64_t C,
                                  int64_t n_chunks, int *__restrict__ chunk_len, int *__restrict__ perm) {
    const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n_chunks) return;
    unsigned mx = 0;
    for (int64_t i = c * C; i < (c + 1) * C; ++i) {
        const unsigned long long k = sorted[i];
        const unsigned cnt = 0x7fffffffu - (unsigned)(k >> 32);
        const int64_t old = (int64_t)(k & 0xffffffffull);
        if (cnt > mx) mx = cnt;
        if (old < n) perm[old] = (int)i;
    }
    chunk_len[c] = (int)mx;
}

__global__ void scs_chunk_sizes(const int *__restrict__ chunk_len, int64_t n_chunks, int64_t C,
                                long long *__restrict__ sizes) {
    const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c < n_chunks) sizes[c] = (long long)chunk_len[c] * C;
}

__global__ void scs_ptr_kernel(const long long *__restrict__ incl, int64_t n_chunks, int *__restrict__ chunk_ptr) {
    const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c > n_chunks) return;
    chunk_ptr[c] = c == 0 ? 0 : (int)incl[c - 1];
}

// one warp per original row: its entries go to chunk-column j of its new row
template <typename VT>
__global__ void scs_scatter_kernel(const int *__restrict__ row_ptr, const int *__restrict__ col,
                                   const VT *__restrict__ val, int64_t n, int64_t C, const int *__restrict__ perm,
                                   const int *__restrict__ chunk_ptr, int *__restrict__ o_col, VT *__restrict__ o_val) {
    const int64_t r = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (r >= n) return;
    const int64_t nr = perm[r];
    const int64_t base = (int64_t)chunk_ptr[nr / C] + nr % C;
    const int s = row_ptr[r], e = row_ptr[r + 1];
    for (int j = s + lane; j < e; j += 32) {
        const int64_t dst = base + (int64_t)(j - s) * C;
        o_col[dst] = col[j];
        o_val[dst] = val[j];
    }
}

}  // namespace

bool scs_vector_path(int64_t C, int vbytes) {
    const int vec = scs_vec(C, vbytes);
    return C % vec == 0 && C / vec >= 1 && C / vec <= 32 && ((C / vec) & (C / vec - 1)) == 0;
}

namespace {
template <typename VT>
__global__ void scs_row_len_kernel(const int *__restrict__ chunk_ptr, const int *__restrict__ chunk_len,
                                   const int *__restrict__ col, const VT *__restrict__ val, int64_t C,
                                   int64_t n_rows_padded, int *__restrict__ row_len) {
    const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n_rows_padded) return;
    const int64_t c = r / C, l = r % C;
    const int64_t cs = chunk_ptr[c];
    int j = chunk_len[c];
    while (j > 0) {
        const int64_t idx = cs + (int64_t)(j - 1) * C + l;
        if (col[idx] != 0 || val[idx] != VT(0)) break;
        --j;
    }
    row_len[r] = j;
}
}  // namespace

void scs_plan(DevSCS &m, int vbytes, cudaStream_t st) {
    const int64_t nc = m.n_chunks;
    std::vector<int> len(nc > 0 ? nc : 1);
    if (nc) SMAX_CUDA(cudaMemcpyAsync(len.data(), m.chunk_len.p, sizeof(int) * nc, cudaMemcpyDeviceToHost, st));
    SMAX_CUDA(cudaStreamSynchronize(st));
    std::vector<int> tc, tj, ts, mc, mf, mk;
    int slots = 0;
    for (int64_t c = 0; c < nc; ++c) {
        const int parts = len[c] > kScsTaskCols ? (len[c] + kScsTaskCols - 1) / kScsTaskCols : 1;
        if (parts > 1) {
            mc.push_back((int)c);
            mf.push_back(slots);
            mk.push_back(parts);
        }
        for (int p = 0; p < parts; ++p) {
            tc.push_back((int)c);
            tj.push_back(p * kScsTaskCols);
            ts.push_back(parts > 1 ? slots + p : -1);
        }
        if (parts > 1) slots += parts;
    }
    auto up = [&](DevBuf &d, const std::vector<int> &h) {
        d.alloc(sizeof(int) * (h.empty() ? 1 : h.size()));
        if (!h.empty()) SMAX_CUDA(cudaMemcpyAsync(d.p, h.data(), sizeof(int) * h.size(), cudaMemcpyHostToDevice, st));
    };
    up(m.task_chunk, tc);
    up(m.task_j0, tj);
    up(m.task_slot, ts);
    up(m.multi_chunk, mc);
    up(m.multi_first, mf);
    up(m.multi_count, mk);
    m.partial.alloc((size_t)vbytes * m.C * (slots > 0 ? slots : 1));
    m.n_tasks = (int64_t)tc.size();
    m.n_multi = (int64_t)mc.size();
    m.n_slots = slots;
    m.plan_vbytes = vbytes;
    // each padded row's length up to its last stored entry that is not
    // padding (column 0 with value 0)
    m.row_len.alloc(sizeof(int) * (m.n_rows_padded > 0 ? m.n_rows_padded : 1));
    if (m.n_rows_padded > 0) {
        const unsigned g = ceil_div_u(m.n_rows_padded, 256);
        if (vbytes == 8)
            scs_row_len_kernel<double><<<g, 256, 0, st>>>(m.chunk_ptr.as<int>(), m.chunk_len.as<int>(),
                                                            m.col.as<int>(), m.val.as<double>(), m.C,
                                                            m.n_rows_padded, m.row_len.as<int>());
        else
            scs_row_len_kernel<float><<<g, 256, 0, st>>>(m.chunk_ptr.as<int>(), m.chunk_len.as<int>(),
                                                           m.col.as<int>(), m.val.as<float>(), m.C,
                                                           m.n_rows_padded, m.row_len.as<int>());
        SMAX_CUDA(cudaGetLastError());
    }
    SMAX_CUDA(cudaStreamSynchronize(st));
}

namespace {

template <typename VT, int VEC>
void launch_task(int64_t lpc, unsigned grid, const int *cp, const int *cl, const int *tc, const int *tj, const int *ts,
                 int64_t n_tasks, const int *ci, const VT *v, const VT *x, VT *y, VT *part, const int *rl,
                 cudaStream_t st) {
    switch (lpc) {
    case 1: scs_task_kernel<VT, 1, VEC><<<grid, 256, 0, st>>>(cp, cl, tc, tj, ts, n_tasks, ci, v, x, y, part, rl); break;
    case 2: scs_task_kernel<VT, 2, VEC><<<grid, 256, 0, st>>>(cp, cl, tc, tj, ts, n_tasks, ci, v, x, y, part, rl); break;
    case 4: scs_task_kernel<VT, 4, VEC><<<grid, 256, 0, st>>>(cp, cl, tc, tj, ts, n_tasks, ci, v, x, y, part, rl); break;
    case 8: scs_task_kernel<VT, 8, VEC><<<grid, 256, 0, st>>>(cp, cl, tc, tj, ts, n_tasks, ci, v, x, y, part, rl); break;
    case 16:
        scs_task_kernel<VT, 16, VEC><<<grid, 256, 0, st>>>(cp, cl, tc, tj, ts, n_tasks, ci, v, x, y, part, rl);
        break;
    case 32:
        scs_task_kernel<VT, 32, VEC><<<grid, 256, 0, st>>>(cp, cl, tc, tj, ts, n_tasks, ci, v, x, y, part, rl);
        break;
    default: fail(SMAX_ERR_STATE, "unexpected SELL chunk width");
    }
}

template <typename VT, int VEC>
void launch_warp(int64_t lpc, unsigned grid, const int *cp, const int *cl, int64_t n_chunks, const int *ci, const VT *v,
                 const VT *x, VT *y, cudaStream_t st) {
    switch (lpc) {
    case 1: scs_warp_kernel<VT, 1, VEC><<<grid, 256, 0, st>>>(cp, cl, n_chunks, ci, v, x, y); break;
    case 2: scs_warp_kernel<VT, 2, VEC><<<grid, 256, 0, st>>>(cp, cl, n_chunks, ci, v, x, y); break;
    case 4: scs_warp_kernel<VT, 4, VEC><<<grid, 256, 0, st>>>(cp, cl, n_chunks, ci, v, x, y); break;
    case 8: scs_warp_kernel<VT, 8, VEC><<<grid, 256, 0, st>>>(cp, cl, n_chunks, ci, v, x, y); break;
    case 16: scs_warp_kernel<VT, 16, VEC><<<grid, 256, 0, st>>>(cp, cl, n_chunks, ci, v, x, y); break;
    case 32: scs_warp_kernel<VT, 32, VEC><<<grid, 256, 0, st>>>(cp, cl, n_chunks, ci, v, x, y); break;
    default: fail(SMAX_ERR_STATE, "unexpected SELL chunk width");
    }
}

}  // namespace

template <typename VT>
void scs_spmv(const DevSCS &m, const VT *x, VT *y, cudaStream_t st) {
    if (m.n_chunks == 0) return;
    const int vec = scs_vec(m.C, sizeof(VT));
    // y is written with 16-byte stores: an offset given to apply() may unalign it
    const bool y_aligned = (reinterpret_cast<uintptr_t>(y) & 15) == 0;
    if (y_aligned && scs_vector_path(m.C, sizeof(VT)) && m.plan_vbytes == (int)sizeof(VT) && m.n_tasks > 0) {
        const unsigned grid = ceil_div_u(m.n_tasks, 8);
        const int *cp = m.chunk_ptr.as<int>(), *cl = m.chunk_len.as<int>(), *ci = m.col.as<int>();
        const int *tc = m.task_chunk.as<int>(), *tj = m.task_j0.as<int>(), *ts = m.task_slot.as<int>();
        const VT *v = m.val.as<VT>();
        VT *part = m.partial.as<VT>();
        const int *rl = m.row_len.p ? m.row_len.as<int>() : nullptr;
        if (vec == 1) launch_task<VT, 1>(m.C, grid, cp, cl, tc, tj, ts, m.n_tasks, ci, v, x, y, part, rl, st);
        else launch_task<VT, 2>(m.C / 2, grid, cp, cl, tc, tj, ts, m.n_tasks, ci, v, x, y, part, rl, st);
        if (m.n_multi > 0)
            scs_fixup_kernel<VT><<<ceil_div_u(m.n_multi * m.C, 256), 256, 0, st>>>(
                m.multi_chunk.as<int>(), m.multi_first.as<int>(), m.multi_count.as<int>(), m.n_multi, (int)m.C, part,
                y);
    } else if (y_aligned && scs_vector_path(m.C, sizeof(VT))) {
        const unsigned grid = ceil_div_u(m.n_chunks, 8);
        const int *cp = m.chunk_ptr.as<int>(), *cl = m.chunk_len.as<int>(), *ci = m.col.as<int>();
        const VT *v = m.val.as<VT>();
        if (vec == 1) launch_warp<VT, 1>(m.C, grid, cp, cl, m.n_chunks, ci, v, x, y, st);
        else launch_warp<VT, 2>(m.C / 2, grid, cp, cl, m.n_chunks, ci, v, x, y, st);
    } else {
        scs_thread_kernel<VT><<<ceil_div_u(m.n_rows_padded, 256), 256, 0, st>>>(
            m.chunk_ptr.as<int>(), m.chunk_len.as<int>(), m.C, m.n_rows_padded, m.col.as<int>(), m.val.as<VT>(),
            x, y);
    }
    SMAX_CUDA(cudaGetLastError());
}

template void scs_spmv<double>(const DevSCS &, const double *, double *, cudaStream_t);
template void scs_spmv<float>(const DevSCS &, const float *, float *, cudaStream_t);

void crs_to_scs(const DevCRS &a, int vbytes, int64_t C, int64_t sigma, DevSCS &out, DevBuf &perm, cudaStream_t st) {
    if (C <= 0 || sigma <= 0) fail(SMAX_ERR_BAD_ARG, "C and sigma must be positive");
    const int64_t n = a.n_rows;
    const int64_t n_chunks = (n + C - 1) / C;
    const int64_t npad = n_chunks * C;
    out.C = C;
    out.sigma = sigma;
    out.n_rows = n;
    out.n_rows_padded = npad;
    out.n_cols = a.n_cols;
    out.n_chunks = n_chunks;
    out.nnz = a.nnz;
    perm.alloc(sizeof(int) * (n > 0 ? n : 1));
    out.chunk_ptr.alloc(sizeof(int) * (n_chunks + 1));
    out.chunk_len.alloc(sizeof(int) * (n_chunks > 0 ? n_chunks : 1));
    if (npad == 0) {
        SMAX_CUDA(cudaMemsetAsync(out.chunk_ptr.p, 0, sizeof(int), st));
        out.n_elements = 0;
        return;
    }
    DevBuf keys(sizeof(unsigned long long) * npad), sorted(sizeof(unsigned long long) * npad);
    scs_keys_kernel<<<ceil_div_u(npad, 256), 256, 0, st>>>(a.rp(), n, npad, keys.as<unsigned long long>());
    SMAX_CUDA(cudaGetLastError());
    const int64_t n_windows = (npad + sigma - 1) / sigma;
    if (n_windows > 0x7fffffffll) fail(SMAX_ERR_UNSUPPORTED, "too many sigma windows");
    DevBuf sort_err(sizeof(int));
    SMAX_CUDA(cudaMemsetAsync(sort_err.p, 0, sizeof(int), st));
    const int64_t win_keys = sigma < npad ? sigma : npad;
    if (win_keys <= kScsSortSmemKeys) {
        const size_t smem = sizeof(unsigned long long) * (size_t)win_keys;
        SMAX_CUDA(cudaFuncSetAttribute(scs_window_sort_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)smem));
        scs_window_sort_kernel<true><<<(unsigned)n_windows, 1, smem, st>>>(
            keys.as<unsigned long long>(), sorted.as<unsigned long long>(), npad, sigma, sort_err.as<int>());
    } else {
        scs_window_sort_kernel<false><<<(unsigned)n_windows, 1, 0, st>>>(
            keys.as<unsigned long long>(), sorted.as<unsigned long long>(), npad, sigma, sort_err.as<int>());
    }
    SMAX_CUDA(cudaGetLastError());
    scs_chunks_kernel<<<ceil_div_u(n_chunks, 256), 256, 0, st>>>(sorted.as<unsigned long long>(), n, C, n_chunks,
                                                                 out.chunk_len.as<int>(), perm.as<int>());
    SMAX_CUDA(cudaGetLastError());
    DevBuf sizes(sizeof(long long) * n_chunks), incl(sizeof(long long) * n_chunks);
    scs_chunk_sizes<<<ceil_div_u(n_chunks, 256), 256, 0, st>>>(out.chunk_len.as<int>(), n_chunks, C,
                                                               sizes.as<long long>());
    SMAX_CUDA(cudaGetLastError());
    size_t tb2 = 0;
    SMAX_CUDA(cub::DeviceScan::InclusiveSum(nullptr, tb2, sizes.as<long long>(), incl.as<long long>(),
                                            (int)n_chunks, st));
    DevBuf tmp2(tb2);
    SMAX_CUDA(cub::DeviceScan::InclusiveSum(tmp2.p, tb2, sizes.as<long long>(), incl.as<long long>(),
                                            (int)n_chunks, st));
    long long ne = 0;
    int h_sort_err = 0;
    SMAX_CUDA(cudaMemcpyAsync(&ne, incl.as<long long>() + n_chunks - 1, sizeof(long long), cudaMemcpyDeviceToHost,
                              st));
    SMAX_CUDA(cudaMemcpyAsync(&h_sort_err, sort_err.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    SMAX_CUDA(cudaStreamSynchronize(st));
    if (h_sort_err) fail(SMAX_ERR_UNSUPPORTED, "sigma-window sort exceeded its stack");
    if (ne >= (1ll << 31)) fail(SMAX_ERR_UNSUPPORTED, "SELL-C-sigma matrix exceeds int32 indexing");
    out.n_elements = ne;
    scs_ptr_kernel<<<ceil_div_u(n_chunks + 1, 256), 256, 0, st>>>(incl.as<long long>(), n_chunks,
                                                                  out.chunk_ptr.as<int>());
    SMAX_CUDA(cudaGetLastError());
    out.col.alloc(sizeof(int) * (ne > 0 ? ne : 1));
    out.val.alloc((size_t)vbytes * (ne > 0 ? ne : 1));
    SMAX_CUDA(cudaMemsetAsync(out.col.p, 0, sizeof(int) * ne, st));
    SMAX_CUDA(cudaMemsetAsync(out.val.p, 0, (size_t)vbytes * ne, st));
    if (n > 0 && a.nnz > 0) {
        const unsigned grid = ceil_div_u((uint64_t)n * 32, 256);
        if (vbytes == 8)
            scs_scatter_kernel<double><<<grid, 256, 0, st>>>(a.rp(), a.ci(), a.val.as<double>(), n, C, perm.as<int>(),
                                                             out.chunk_ptr.as<int>(), out.col.as<int>(),
                                                             out.val.as<double>());
        else
            scs_scatter_kernel<float><<<grid, 256, 0, st>>>(a.rp(), a.ci(), a.val.as<float>(), n, C, perm.as<int>(),
                                                            out.chunk_ptr.as<int>(), out.col.as<int>(),
                                                            out.val.as<float>());
        SMAX_CUDA(cudaGetLastError());
    }
    SMAX_CUDA(cudaStreamSynchronize(st));
}

}  // namespace smax

namespace smax {
namespace {
// chunk_ptr[0] == 0, chunk_ptr[c+1] - chunk_ptr[c] == chunk_len[c]*C (so every
// chunk start is a multiple of C, which the vector loads rely on),
// chunk_ptr[n_chunks] == n_elements, every column in [0, n_cols).
__global__ void validate_scs_kernel(const int *__restrict__ cp, const int *__restrict__ cl,
                                    const int *__restrict__ col, int64_t n_chunks, int64_t C, int64_t n_elements,
                                    int64_t n_cols, DevStatus *st) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t == 0 && (cp[0] != 0 || cp[n_chunks] != n_elements)) report(st, SMAX_ERR_BAD_ARG, 0);
    for (int64_t c = t; c < n_chunks; c += stride)
        if (cl[c] < 0 || (int64_t)cp[c + 1] - cp[c] != (int64_t)cl[c] * C) report(st, SMAX_ERR_BAD_ARG, c);
    for (int64_t j = t; j < n_elements; j += stride) {
        const int c = col[j];
        if (c < 0 || c >= n_cols) report(st, SMAX_ERR_COL_OOB, j);
    }
}
}  // namespace

void validate_scs(const DevSCS &m, DevStatus *st, cudaStream_t s) {
    validate_scs_kernel<<<4 * sm_count(), 256, 0, s>>>(m.chunk_ptr.as<int>(), m.chunk_len.as<int>(), m.col.as<int>(),
                                                       m.n_chunks, m.C, m.n_elements, m.n_cols, st);
    SMAX_CUDA(cudaGetLastError());
}
}  // namespace smax
