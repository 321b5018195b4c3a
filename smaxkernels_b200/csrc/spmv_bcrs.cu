// spmv_bcrs.cu -- BCRS SpMV and CRS -> BCRS conversion on sm_100a.
//
// Layout (src/common.hpp:90-111, src/utils/convert_formats.hpp:134-247): block
// row r holds blocks row_ptr[r]..row_ptr[r+1]-1; block j is the hpad x wpad
// tile val[j*hpad*wpad ...] stored row-major (ix*wpad+jx) or column-major
// (jx*hpad+ix); x is indexed by col[j]*wpad+jx and y by r*hpad+ix, for
// ix < bh and jx < bw (SPMV::CPU::naive_bcrs_spmv,
// src/kernels/spmv/spmv_cpu/spmv_cpu_bcrs_impl.hpp:19-85).
//
// SpMV, register-blocked block-row stream (block size bs = hpad*wpad divisible
// by VEC = 16/sizeof(VT) and dividing 32*VEC, e.g. 4x4): one warp per block
// row streams that row's blocks as one flat array with 128-bit evict-first
// loads; because the warp advances 32*VEC values per step, every lane always
// sees the same VEC in-block positions, so it keeps VEC register accumulators
// for fixed (ix, jx).  Lanes holding the same positions combine with
// shuffles; the bs partial sums are then folded into the bh outputs through
// a per-warp shared-memory tile (fixed order, deterministic).  Long block
// rows (three or more warp steps on average) use a four-step loop with more
// loads in flight; short ones (under two steps: e.g. a stencil in 4x4 blocks)
// give each block row a group of bs/VEC lanes instead of a warp.  Other block
// shapes: one thread per block row in the reference's loop order.
//
// Conversion: per block row, the sorted distinct block columns of its bh rows
// (segmented radix sort of col/bw over the block row's entries, then a
// uniqueness pass and a scan), then every entry is written into its block at
// the in-block index of the chosen order; blocks are zero-filled first.
#include "spmv_formats.cuh"

#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>
#include <cub/device/device_segmented_radix_sort.cuh>
#include <cub/device/device_select.cuh>

namespace smax {

namespace {

template <typename VT> struct V16;
template <> struct V16<double> { using T = double2; static constexpr int N = 2; };
template <> struct V16<float> { using T = float4; static constexpr int N = 4; };

// Block values: evict-first (streamed once), or with KEEP the default
// policy, so that a matrix whose values fit in L2 stays there across products.
template <typename VT, int VEC, bool KEEP = false>
__device__ __forceinline__ void load16(const VT *p, VT *o) {
    if constexpr (VEC == 2) {
        const double2 *q = reinterpret_cast<const double2 *>(p);
        const double2 v = KEEP ? __ldg(q) : __ldcs(q);
        o[0] = v.x; o[1] = v.y;
    } else {
        const float4 *q = reinterpret_cast<const float4 *>(p);
        const float4 v = KEEP ? __ldg(q) : __ldcs(q);
        o[0] = v.x; o[1] = v.y; o[2] = v.z; o[3] = v.w;
    }
}

constexpr int kMaxBs = 128;  // largest block size of the stream path

// The stream loop of one block row per warp (the kernels below launch it).
template <typename VT, bool UNROLL>
__device__ __forceinline__ void bcrs_stream_rows(const int *__restrict__ row_ptr, const int *__restrict__ col,
                                                 const VT *__restrict__ val, int64_t n_brows, int bh, int bw,
                                                 int hpad, int wpad, int col_major, const VT *__restrict__ x,
                                                 VT *__restrict__ y, const int *__restrict__ order) {
    constexpr int VEC = V16<VT>::N;
    __shared__ VT tile[8][kMaxBs];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int64_t w = (int64_t)blockIdx.x * 8 + warp;
    if (w >= n_brows) return;  // uniform per warp
    const int64_t br = order ? order[w] : w;
    const int bs = hpad * wpad;
    const int o = (lane * VEC) % bs;  // this lane's first in-block position
    int jx[VEC];
    bool ok[VEC];
#pragma unroll
    for (int i = 0; i < VEC; ++i) {
        const int q = o + i;
        const int ix = col_major ? q % hpad : q / wpad;
        jx[i] = col_major ? q / hpad : q % wpad;
        ok[i] = ix < bh && jx[i] < bw;
    }
    VT acc[VEC];
#pragma unroll
    for (int i = 0; i < VEC; ++i) acc[i] = VT(0);
    const int64_t b0 = row_ptr[br], b1 = row_ptr[br + 1];
    const int64_t end = b1 * bs;
    constexpr int64_t STEP = 32 * VEC;
    int64_t f = b0 * bs + lane * VEC;
    // four steps' value and column loads first, then their x gathers, then
    // the products in step order (the same sums as the one-step loop); for
    // short block rows the registers this takes cost more occupancy than the
    // overlap gains, so it is compiled out (UNROLL false)
    // The column indices are loaded one iteration ahead, so an iteration's x
    // gathers wait on no load of their own.
    if constexpr (UNROLL) {
    int cn[4] = {0, 0, 0, 0};
    if (f + 3 * STEP < end)
#pragma unroll
        for (int u = 0; u < 4; ++u) cn[u] = col[(f + u * STEP) / bs];
    for (; f + 3 * STEP < end; f += 4 * STEP) {
        VT v[4][VEC];
        int64_t c[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            load16<VT, VEC>(val + f + u * STEP, v[u]);
            c[u] = (int64_t)cn[u] * wpad;
        }
        const int64_t fn = f + 4 * STEP;
        if (fn + 3 * STEP < end)
#pragma unroll
            for (int u = 0; u < 4; ++u) cn[u] = col[(fn + u * STEP) / bs];
        VT xv[4][VEC];
#pragma unroll
        for (int u = 0; u < 4; ++u)
#pragma unroll
            for (int i = 0; i < VEC; ++i) xv[u][i] = ok[i] ? ld_keep(x + c[u] + jx[i]) : VT(0);
#pragma unroll
        for (int u = 0; u < 4; ++u)
#pragma unroll
            for (int i = 0; i < VEC; ++i)
                if (ok[i]) acc[i] += v[u][i] * xv[u][i];
    }
    }
    for (; f < end; f += STEP) {
        const int64_t c = (int64_t)col[f / bs] * wpad;
        VT v[VEC];
        load16<VT, VEC>(val + f, v);
#pragma unroll
        for (int i = 0; i < VEC; ++i)
            if (ok[i]) acc[i] += v[i] * ld_keep(x + c + jx[i]);
    }
    const int groups = bs / VEC;  // lanes l and l + groups*m hold the same positions
    for (int s = groups; s < 32; s <<= 1)
#pragma unroll
        for (int i = 0; i < VEC; ++i) acc[i] += __shfl_xor_sync(0xffffffffu, acc[i], s);
    if (lane < groups)
#pragma unroll
        for (int i = 0; i < VEC; ++i) tile[warp][o + i] = acc[i];
    __syncwarp();
    for (int ix = lane; ix < bh; ix += 32) {
        VT s = VT(0);
        for (int j = 0; j < bw; ++j) s += tile[warp][col_major ? j * hpad + ix : ix * wpad + j];
        st_stream(y + br * hpad + ix, s);
    }
}

template <typename VT, bool UNROLL>
__global__ void __launch_bounds__(256) bcrs_stream_kernel(const int *__restrict__ row_ptr,
                                                          const int *__restrict__ col, const VT *__restrict__ val,
                                                          int64_t n_brows, int bh, int bw, int hpad, int wpad,
                                                          int col_major, const VT *__restrict__ x,
                                                          VT *__restrict__ y, const int *__restrict__ order) {
    bcrs_stream_rows<VT, UNROLL>(row_ptr, col, val, n_brows, bh, bw, hpad, wpad, col_major, x, y, order);
}

// FP64: at most 48 registers, five CTAs per SM instead of four (the four-step
// loop spills 32 bytes; 2^22 lognormal 4x4: 2.30 -> 2.26 ms; a bound of six
// CTAs spilled 64 bytes and took 2.54 ms).  FP32 keeps the plain kernel: the
// same bound spilled 88 bytes there.
template <bool UNROLL>
__global__ void __launch_bounds__(256, 5) bcrs_stream_kernel_f64(const int *__restrict__ row_ptr,
                                                                 const int *__restrict__ col,
                                                                 const double *__restrict__ val, int64_t n_brows,
                                                                 int bh, int bw, int hpad, int wpad, int col_major,
                                                                 const double *__restrict__ x, double *__restrict__ y,
                                                                 const int *__restrict__ order) {
    bcrs_stream_rows<double, UNROLL>(row_ptr, col, val, n_brows, bh, bw, hpad, wpad, col_major, x, y, order);
}

// Short block rows: a group of G = bs / VEC lanes per block row (8 lanes for
// 4x4 FP64), one block per step, two blocks' loads in flight.  Every lane
// keeps the same VEC in-block positions for the whole row, so the bs sums
// are complete without shuffles and are folded into the bh outputs through
// the group's shared-memory tile (fixed order).
template <typename VT, bool KEEP>
__global__ void __launch_bounds__(256) bcrs_group_kernel(const int *__restrict__ row_ptr,
                                                         const int *__restrict__ col, const VT *__restrict__ val,
                                                         int64_t n_brows, int bh, int bw, int hpad, int wpad,
                                                         int col_major, const VT *__restrict__ x,
                                                         VT *__restrict__ y) {
    constexpr int VEC = V16<VT>::N;
    __shared__ VT tile[256 * VEC];  // 256 / G groups x bs values = 256 * VEC
    const int bs = hpad * wpad;
    const int G = bs / VEC;
    const int g_in_cta = threadIdx.x / G, lg = threadIdx.x % G;
    const int64_t br = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) / G;
    const int o = lg * VEC;
    int jx[VEC];
    bool ok[VEC];
#pragma unroll
    for (int i = 0; i < VEC; ++i) {
        const int q = o + i;
        const int ix = col_major ? q % hpad : q / wpad;
        jx[i] = col_major ? q / hpad : q % wpad;
        ok[i] = ix < bh && jx[i] < bw;
    }
    VT acc[VEC];
#pragma unroll
    for (int i = 0; i < VEC; ++i) acc[i] = VT(0);
    if (br < n_brows) {
        const int b1 = row_ptr[br + 1];
        int j = row_ptr[br];
        for (; j + 1 < b1; j += 2) {
            VT v0[VEC], v1[VEC];
            load16<VT, VEC, KEEP>(val + (int64_t)j * bs + o, v0);
            load16<VT, VEC, KEEP>(val + (int64_t)(j + 1) * bs + o, v1);
            const int64_t c0 = (int64_t)col[j] * wpad, c1 = (int64_t)col[j + 1] * wpad;
            VT x0[VEC], x1[VEC];
#pragma unroll
            for (int i = 0; i < VEC; ++i) {
                x0[i] = ok[i] ? ld_keep(x + c0 + jx[i]) : VT(0);
                x1[i] = ok[i] ? ld_keep(x + c1 + jx[i]) : VT(0);
            }
#pragma unroll
            for (int i = 0; i < VEC; ++i)
                if (ok[i]) {
                    acc[i] += v0[i] * x0[i];
                    acc[i] += v1[i] * x1[i];
                }
        }
        if (j < b1) {
            VT v[VEC];
            load16<VT, VEC, KEEP>(val + (int64_t)j * bs + o, v);
            const int64_t c = (int64_t)col[j] * wpad;
#pragma unroll
            for (int i = 0; i < VEC; ++i)
                if (ok[i]) acc[i] += v[i] * ld_keep(x + c + jx[i]);
        }
    }
    VT *t = tile + g_in_cta * bs;
#pragma unroll
    for (int i = 0; i < VEC; ++i) t[o + i] = acc[i];
    __syncthreads();
    if (br < n_brows)
        for (int ix = lg; ix < bh; ix += G) {
            VT s = VT(0);
            for (int q = 0; q < bw; ++q) s += t[col_major ? q * hpad + ix : ix * wpad + q];
            st_stream(y + br * hpad + ix, s);
        }
}

// generic block shapes: one thread per block row, the reference's loop order
template <typename VT>
__global__ void bcrs_thread_kernel(const int *__restrict__ row_ptr, const int *__restrict__ col,
                                   const VT *__restrict__ val, int64_t n_brows, int bh, int bw, int hpad, int wpad,
                                   int col_major, const VT *__restrict__ x, VT *__restrict__ y) {
    const int64_t br = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (br >= n_brows) return;
    const int64_t bs = (int64_t)hpad * wpad;
    for (int ix = 0; ix < bh; ++ix) {
        VT s = VT(0);
        for (int j = row_ptr[br]; j < row_ptr[br + 1]; ++j) {
            const VT *blk = val + (int64_t)j * bs;
            const VT *xb = x + (int64_t)col[j] * wpad;
            for (int jx = 0; jx < bw; ++jx) s += blk[col_major ? jx * hpad + ix : ix * wpad + jx] * xb[jx];
        }
        y[br * hpad + ix] = s;
    }
}

// ----------------------------------------------------------- conversion ----
__global__ void bcrs_keys(const int *__restrict__ row_ptr, const int *__restrict__ col, int64_t n, int bw,
                          int *__restrict__ keys) {
    const int64_t r = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (r >= n) return;
    for (int j = row_ptr[r] + lane; j < row_ptr[r + 1]; j += 32) keys[j] = col[j] / bw;
}

__global__ void bcrs_seg_offsets(const int *__restrict__ row_ptr, int64_t n_brows, int bh, int *__restrict__ off) {
    const int64_t b = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (b <= n_brows) off[b] = row_ptr[b * bh];
}

// flag[j] = 1 when sorted[j] starts a new distinct block column in its block row
__global__ void bcrs_unique_flags(const int *__restrict__ sorted, const int *__restrict__ off, int64_t n_brows,
                                  int64_t nnz, unsigned char *__restrict__ flag, int *__restrict__ brow_of) {
    const int64_t b = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (b >= n_brows) return;
    for (int64_t j = off[b] + lane; j < off[b + 1]; j += 32) {
        flag[j] = (j == off[b] || sorted[j] != sorted[j - 1]) ? 1 : 0;
        brow_of[j] = (int)b;
    }
}

__global__ void bcrs_count(const int *__restrict__ brow_of_unique, int64_t n_unique, int *__restrict__ counts) {
    const int64_t u = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (u < n_unique) atomicAdd(counts + brow_of_unique[u], 1);
}

__global__ void bcrs_ptr(const int *__restrict__ incl, int64_t n_brows, int *__restrict__ b_row_ptr) {
    const int64_t b = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (b <= n_brows) b_row_ptr[b] = b == 0 ? 0 : incl[b - 1];
}

template <typename VT>
__global__ void bcrs_fill(const int *__restrict__ row_ptr, const int *__restrict__ col, const VT *__restrict__ val,
                          int64_t n, int bh, int bw, int hpad, int wpad, int col_major,
                          const int *__restrict__ b_row_ptr, const int *__restrict__ b_col, VT *__restrict__ b_val) {
    const int64_t r = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (r >= n) return;
    const int64_t br = r / bh;
    const int lr = (int)(r % bh);
    const int64_t bs = (int64_t)hpad * wpad;
    for (int j = row_ptr[r] + lane; j < row_ptr[r + 1]; j += 32) {
        const int bc = col[j] / bw;
        int lo = b_row_ptr[br], hi = b_row_ptr[br + 1];
        while (lo < hi) {
            const int mid = (lo + hi) >> 1;
            if (b_col[mid] < bc) lo = mid + 1; else hi = mid;
        }
        const int in = col_major ? hpad * (col[j] % bw) + lr : wpad * lr + col[j] % bw;
        b_val[(int64_t)lo * bs + in] = val[j];
    }
}

}  // namespace

bool bcrs_stream_path(int64_t hpad, int64_t wpad, int vbytes) {
    const int vec = 16 / vbytes;
    const int64_t bs = hpad * wpad;
    return bs > 0 && bs <= kMaxBs && bs % vec == 0 && (32 * vec) % bs == 0;
}

template <typename VT>
void bcrs_spmv(const DevBCRS &m, const VT *x, VT *y, cudaStream_t st) {
    if (m.n_rows == 0) return;
    const int *order = m.order.p ? m.order.as<int>() : nullptr;
    if (bcrs_stream_path(m.hpad, m.wpad, sizeof(VT))) {
        // mean warp steps per block row: below two a lane group per block row
        // wastes fewer lanes; the four-step loop pays off from about three
        const double steps = (double)m.n_blocks * (double)(m.hpad * m.wpad) /
                             ((double)m.n_rows * 32.0 * (16.0 / sizeof(VT)));
        const int64_t group = m.hpad * m.wpad / (16 / (int64_t)sizeof(VT));
        // values that fit in half of L2 are loaded with the default policy and
        // stay resident across repeated products (4x4 blocks of the 7-point
        // 64^3 Laplacian, 59 MB of values, in a loop of products: see the
        // BCRS notes); larger ones stream evict-first
        const bool keep = (double)m.n_blocks * (double)(m.hpad * m.wpad) * sizeof(VT) <= 0.5 * (double)l2_bytes();
        if (steps < 2.0 && keep)
            bcrs_group_kernel<VT, true><<<ceil_div_u((uint64_t)m.n_rows * group, 256), 256, 0, st>>>(
                m.row_ptr.as<int>(), m.col.as<int>(), m.val.as<VT>(), m.n_rows, (int)m.bh, (int)m.bw, (int)m.hpad,
                (int)m.wpad, m.col_major ? 1 : 0, x, y);
        else if (steps < 2.0)
            bcrs_group_kernel<VT, false><<<ceil_div_u((uint64_t)m.n_rows * group, 256), 256, 0, st>>>(
                m.row_ptr.as<int>(), m.col.as<int>(), m.val.as<VT>(), m.n_rows, (int)m.bh, (int)m.bw, (int)m.hpad,
                (int)m.wpad, m.col_major ? 1 : 0, x, y);
        else if (steps >= 3.0 && sizeof(VT) == 8)
            bcrs_stream_kernel_f64<true><<<ceil_div_u(m.n_rows, 8), 256, 0, st>>>(
                m.row_ptr.as<int>(), m.col.as<int>(), reinterpret_cast<const double *>(m.val.as<VT>()), m.n_rows,
                (int)m.bh, (int)m.bw, (int)m.hpad, (int)m.wpad, m.col_major ? 1 : 0,
                reinterpret_cast<const double *>(x), reinterpret_cast<double *>(y), order);
        else if (steps >= 3.0)
            bcrs_stream_kernel<VT, true><<<ceil_div_u(m.n_rows, 8), 256, 0, st>>>(
                m.row_ptr.as<int>(), m.col.as<int>(), m.val.as<VT>(), m.n_rows, (int)m.bh, (int)m.bw, (int)m.hpad,
                (int)m.wpad, m.col_major ? 1 : 0, x, y, order);
        else
            bcrs_stream_kernel<VT, false><<<ceil_div_u(m.n_rows, 8), 256, 0, st>>>(
                m.row_ptr.as<int>(), m.col.as<int>(), m.val.as<VT>(), m.n_rows, (int)m.bh, (int)m.bw, (int)m.hpad,
                (int)m.wpad, m.col_major ? 1 : 0, x, y, order);
    } else
        bcrs_thread_kernel<VT><<<ceil_div_u(m.n_rows, 128), 128, 0, st>>>(
            m.row_ptr.as<int>(), m.col.as<int>(), m.val.as<VT>(), m.n_rows, (int)m.bh, (int)m.bw, (int)m.hpad,
            (int)m.wpad, m.col_major ? 1 : 0, x, y);
    SMAX_CUDA(cudaGetLastError());
}

namespace {
__global__ void bcrs_row_lengths(const int *__restrict__ row_ptr, int64_t n, int *__restrict__ len,
                                 int *__restrict__ idx) {
    const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n) return;
    len[r] = row_ptr[r + 1] - row_ptr[r];
    idx[r] = (int)r;
}
}  // namespace

void bcrs_plan(DevBCRS &m, cudaStream_t st) {
    m.order.release();
    if (m.n_rows < 2) return;
    const int64_t n = m.n_rows;
    DevBuf len(sizeof(int) * n), idx(sizeof(int) * n), len_sorted(sizeof(int) * n);
    m.order.alloc(sizeof(int) * n);
    bcrs_row_lengths<<<ceil_div_u(n, 256), 256, 0, st>>>(m.row_ptr.as<int>(), n, len.as<int>(), idx.as<int>());
    SMAX_CUDA(cudaGetLastError());
    size_t tb = 0;
    SMAX_CUDA(cub::DeviceRadixSort::SortPairsDescending(nullptr, tb, len.as<int>(), len_sorted.as<int>(),
                                                        idx.as<int>(), m.order.as<int>(), (int)n, 0, 32, st));
    DevBuf tmp(tb ? tb : 1);
    SMAX_CUDA(cub::DeviceRadixSort::SortPairsDescending(tmp.p, tb, len.as<int>(), len_sorted.as<int>(),
                                                        idx.as<int>(), m.order.as<int>(), (int)n, 0, 32, st));
    SMAX_CUDA(cudaStreamSynchronize(st));
}

template void bcrs_spmv<double>(const DevBCRS &, const double *, double *, cudaStream_t);
template void bcrs_spmv<float>(const DevBCRS &, const float *, float *, cudaStream_t);

void crs_to_bcrs(const DevCRS &a, int vbytes, int64_t bh, int64_t bw, int64_t hpad, int64_t wpad, bool col_major,
                 DevBCRS &out, cudaStream_t st, int64_t max_blocks) {
    // the reference throws for these (src/utils/convert_formats.hpp:143-160); it
    // tests the height padding twice, this platform tests both paddings
    if (bh <= 0 || bw <= 0 || a.n_rows % bh) fail(SMAX_ERR_BAD_ARG, "Target block height does not divide number of input rows");
    if (a.n_cols % bw) fail(SMAX_ERR_BAD_ARG, "Target block width does not divide number of input columns");
    if (hpad < bh) fail(SMAX_ERR_BAD_ARG, "Height padding has to be at least target block height");
    if (wpad < bw) fail(SMAX_ERR_BAD_ARG, "Width padding has to be at least target block width");
    const int64_t n = a.n_rows, nnz = a.nnz, nb = n / bh;
    out.n_rows = nb;
    out.n_cols = a.n_cols / bw;
    out.bh = bh; out.bw = bw; out.hpad = hpad; out.wpad = wpad;
    out.col_major = col_major;
    out.row_ptr.alloc(sizeof(int) * (nb + 1));
    if (nnz == 0) {
        SMAX_CUDA(cudaMemsetAsync(out.row_ptr.p, 0, sizeof(int) * (nb + 1), st));
        out.n_blocks = 0;
        SMAX_CUDA(cudaStreamSynchronize(st));
        return;
    }
    DevBuf keys(sizeof(int) * nnz), sorted(sizeof(int) * nnz), off(sizeof(int) * (nb + 1));
    bcrs_keys<<<ceil_div_u((uint64_t)n * 32, 256), 256, 0, st>>>(a.rp(), a.ci(), n, (int)bw, keys.as<int>());
    bcrs_seg_offsets<<<ceil_div_u(nb + 1, 256), 256, 0, st>>>(a.rp(), nb, (int)bh, off.as<int>());
    SMAX_CUDA(cudaGetLastError());
    size_t tb = 0;
    SMAX_CUDA(cub::DeviceSegmentedRadixSort::SortKeys(nullptr, tb, keys.as<int>(), sorted.as<int>(), (int)nnz,
                                                      (int)nb, off.as<int>(), off.as<int>() + 1, 0, 32, st));
    DevBuf tmp(tb);
    SMAX_CUDA(cub::DeviceSegmentedRadixSort::SortKeys(tmp.p, tb, keys.as<int>(), sorted.as<int>(), (int)nnz,
                                                      (int)nb, off.as<int>(), off.as<int>() + 1, 0, 32, st));
    DevBuf flag(nnz), brow(sizeof(int) * nnz), ucol(sizeof(int) * nnz), ubrow(sizeof(int) * nnz), nsel(sizeof(int) * 2);
    bcrs_unique_flags<<<ceil_div_u((uint64_t)nb * 32, 256), 256, 0, st>>>(sorted.as<int>(), off.as<int>(), nb, nnz,
                                                                          flag.as<unsigned char>(), brow.as<int>());
    SMAX_CUDA(cudaGetLastError());
    size_t tb2 = 0;
    SMAX_CUDA(cub::DeviceSelect::Flagged(nullptr, tb2, sorted.as<int>(), flag.as<unsigned char>(), ucol.as<int>(),
                                         nsel.as<int>(), (int)nnz, st));
    DevBuf tmp2(tb2);
    SMAX_CUDA(cub::DeviceSelect::Flagged(tmp2.p, tb2, sorted.as<int>(), flag.as<unsigned char>(), ucol.as<int>(),
                                         nsel.as<int>(), (int)nnz, st));
    SMAX_CUDA(cub::DeviceSelect::Flagged(tmp2.p, tb2, brow.as<int>(), flag.as<unsigned char>(), ubrow.as<int>(),
                                         nsel.as<int>() + 1, (int)nnz, st));
    int nu = 0;
    SMAX_CUDA(cudaMemcpyAsync(&nu, nsel.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    SMAX_CUDA(cudaStreamSynchronize(st));
    out.n_blocks = nu;
    if (max_blocks >= 0 && nu > max_blocks) {
        // more blocks than the caller accepts: report the count, build nothing
        out.col.release();
        out.val.release();
        return;
    }
    DevBuf counts(sizeof(int) * nb), incl(sizeof(int) * nb);
    SMAX_CUDA(cudaMemsetAsync(counts.p, 0, sizeof(int) * nb, st));
    bcrs_count<<<ceil_div_u(nu, 256), 256, 0, st>>>(ubrow.as<int>(), nu, counts.as<int>());
    SMAX_CUDA(cudaGetLastError());
    size_t tb3 = 0;
    SMAX_CUDA(cub::DeviceScan::InclusiveSum(nullptr, tb3, counts.as<int>(), incl.as<int>(), (int)nb, st));
    DevBuf tmp3(tb3);
    SMAX_CUDA(cub::DeviceScan::InclusiveSum(tmp3.p, tb3, counts.as<int>(), incl.as<int>(), (int)nb, st));
    bcrs_ptr<<<ceil_div_u(nb + 1, 256), 256, 0, st>>>(incl.as<int>(), nb, out.row_ptr.as<int>());
    SMAX_CUDA(cudaGetLastError());
    out.col.alloc(sizeof(int) * nu);
    SMAX_CUDA(cudaMemcpyAsync(out.col.p, ucol.p, sizeof(int) * nu, cudaMemcpyDeviceToDevice, st));
    const int64_t bs = hpad * wpad;
    out.val.alloc((size_t)vbytes * nu * bs);
    SMAX_CUDA(cudaMemsetAsync(out.val.p, 0, (size_t)vbytes * nu * bs, st));
    const unsigned grid = ceil_div_u((uint64_t)n * 32, 256);
    if (vbytes == 8)
        bcrs_fill<double><<<grid, 256, 0, st>>>(a.rp(), a.ci(), a.val.as<double>(), n, (int)bh, (int)bw, (int)hpad,
                                                (int)wpad, col_major, out.row_ptr.as<int>(), out.col.as<int>(),
                                                out.val.as<double>());
    else
        bcrs_fill<float><<<grid, 256, 0, st>>>(a.rp(), a.ci(), a.val.as<float>(), n, (int)bh, (int)bw, (int)hpad,
                                               (int)wpad, col_major, out.row_ptr.as<int>(), out.col.as<int>(),
                                               out.val.as<float>());
    SMAX_CUDA(cudaGetLastError());
    SMAX_CUDA(cudaStreamSynchronize(st));
}

}  // namespace smax

namespace smax {
namespace {
__global__ void validate_bcrs_kernel(const int *__restrict__ rp, const int *__restrict__ col, int64_t n,
                                     int64_t n_blocks, int64_t n_cols, DevStatus *st) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t == 0 && (rp[0] != 0 || rp[n] != n_blocks)) report(st, SMAX_ERR_BAD_ARG, 0);
    for (int64_t r = t; r < n; r += stride)
        if (rp[r + 1] < rp[r]) report(st, SMAX_ERR_BAD_ARG, r);
    for (int64_t j = t; j < n_blocks; j += stride) {
        const int c = col[j];
        if (c < 0 || c >= n_cols) report(st, SMAX_ERR_COL_OOB, j);
    }
}
}  // namespace

void validate_bcrs(const DevBCRS &m, DevStatus *st, cudaStream_t s) {
    validate_bcrs_kernel<<<4 * sm_count(), 256, 0, s>>>(m.row_ptr.as<int>(), m.col.as<int>(), m.n_rows, m.n_blocks,
                                                        m.n_cols, st);
    SMAX_CUDA(cudaGetLastError());
}
}  // namespace smax
