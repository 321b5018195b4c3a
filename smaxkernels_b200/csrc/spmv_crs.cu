// spmv_crs.cu -- CRS SpMV y = A*x for sm_100a.
//
// Reference semantics: SPMV::CPU::naive_crs_spmv
// (src/kernels/spmv/spmv_cpu/spmv_cpu_crs_impl.hpp:9-38): y[i] = sum_j val[j]*x[col[j]]
// over row i.  The reference CUDA kernel (src/kernels/spmv/spmv_cuda/
// spmv_cuda_crs_impl.cu:5-22) runs one thread per row, so a warp's loads of
// val/col touch 32 unrelated rows; it is replaced here by a row-tile design.
//
// Design (nnz-balanced row tiles, one CTA per tile):
//   * At plan time the rows are cut into tiles.  A tile starts at row r when r
//     is the first row, when r or r-1 is "long" (more than `cap` entries), when
//     row_ptr[r] falls into a different cap-sized bucket of the nnz range than
//     row_ptr[r-1], or when r is a multiple of kRowsMax.  A short-row tile thus
//     holds < 2*cap entries and <= kRowsMax rows; a long row is a tile alone.
//     The cut is a pure function of row_ptr and is computed on the GPU.
//   * Short-row tile: the CTA streams the tile's contiguous val/col range with
//     coalesced, evict-first loads, gathers x (kept in L2), stages the products
//     in shared memory, then reduces each row with a power-of-two group of
//     lanes sized from the tile's row count and writes y.
//   * Long-row tile: the whole CTA strides the row and block-reduces.
// HBM traffic is the algorithmic minimum: each val/col/row_ptr element and each
// y element once; x through L2.
#include "spmv_crs.cuh"

#include <cub/device/device_select.cuh>
#include <thrust/iterator/counting_iterator.h>

namespace smax {

namespace {

constexpr int kBlock = 256;       // threads per tile CTA
constexpr int kRowsMax = kBlock;  // rows per short-row tile

__global__ void tile_flags_kernel(const int *__restrict__ row_ptr, int64_t n, int cap,
                                  unsigned char *__restrict__ flags) {
    int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n) return;
    unsigned char f;
    int s = row_ptr[r], e = row_ptr[r + 1];
    if (r == 0) {
        f = 1;
    } else {
        int ps = row_ptr[r - 1];
        bool long_r = (e - s) > cap;
        bool long_p = (s - ps) > cap;
        bool bucket = (s / cap) != (ps / cap);
        f = (long_r || long_p || bucket || (r % kRowsMax) == 0) ? 1 : 0;
    }
    flags[r] = f;
}

__global__ void set_last_kernel(int *tiles, const int *n_sel, int value) { tiles[*n_sel] = value; }

// Sum over the G lanes of an aligned G-lane segment of a warp.
template <int G, typename VT> __device__ __forceinline__ VT group_sum(VT v) {
#pragma unroll
    for (int o = G / 2; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

template <typename VT> __device__ __forceinline__ VT dyn_group_sum(VT v, int G) {
    for (int o = G >> 1; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

template <typename VT, int CAP>
__global__ void __launch_bounds__(kBlock) crs_tile_kernel(const int *__restrict__ tiles,
                                                          const int *__restrict__ row_ptr,
                                                          const int *__restrict__ col,
                                                          const VT *__restrict__ val,
                                                          const VT *__restrict__ x,
                                                          VT *__restrict__ y) {
    constexpr int PER = (2 * CAP) / kBlock;  // staged entries per thread
    __shared__ VT prod[2 * CAP];
    __shared__ int srp[kRowsMax + 1];
    __shared__ VT red[kBlock / 32];

    const int tid = threadIdx.x;
    const int r0 = tiles[blockIdx.x];
    const int r1 = tiles[blockIdx.x + 1];
    const int nr = r1 - r0;

    if (nr == 1) {
        const int s = row_ptr[r0], e = row_ptr[r0 + 1];
        if (e - s > CAP) {
            // ---- long row: whole CTA, direct from global --------------------
            VT acc = VT(0);
            int j = s + tid;
            for (; j + 3 * kBlock < e; j += 4 * kBlock) {
                int c0 = ld_stream(col + j), c1 = ld_stream(col + j + kBlock);
                int c2 = ld_stream(col + j + 2 * kBlock), c3 = ld_stream(col + j + 3 * kBlock);
                VT v0 = ld_stream(val + j), v1 = ld_stream(val + j + kBlock);
                VT v2 = ld_stream(val + j + 2 * kBlock), v3 = ld_stream(val + j + 3 * kBlock);
                acc += v0 * ld_keep(x + c0);
                acc += v1 * ld_keep(x + c1);
                acc += v2 * ld_keep(x + c2);
                acc += v3 * ld_keep(x + c3);
            }
            for (; j < e; j += kBlock) acc += ld_stream(val + j) * ld_keep(x + ld_stream(col + j));
            acc = group_sum<32>(acc);
            if ((tid & 31) == 0) red[tid >> 5] = acc;
            __syncthreads();
            if (tid < 32) {
                VT v = tid < kBlock / 32 ? red[tid] : VT(0);
                v = group_sum<32>(v);
                if (tid == 0) st_stream(y + r0, v);
            }
            return;
        }
    }

    // ---- short-row tile ----------------------------------------------------
    for (int i = tid; i <= nr; i += kBlock) srp[i] = row_ptr[r0 + i];
    __syncthreads();
    const int j0 = srp[0];
    const int m = srp[nr] - j0;  // < 2*CAP by construction of the tiles

    int cbuf[PER];
    VT vbuf[PER];
#pragma unroll
    for (int k = 0; k < PER; ++k) {
        const int e = tid + k * kBlock;
        if (e < m) {
            cbuf[k] = ld_stream(col + j0 + e);
            vbuf[k] = ld_stream(val + j0 + e);
        }
    }
#pragma unroll
    for (int k = 0; k < PER; ++k) {
        const int e = tid + k * kBlock;
        if (e < m) prod[e] = vbuf[k] * ld_keep(x + cbuf[k]);
    }
    __syncthreads();

    // lanes per row: the largest power of two with nr*G <= kBlock, at most 32
    int G = 32;
    while (G > 1 && nr * G > kBlock) G >>= 1;
    const int lane = tid & (G - 1);
    const int grp = tid / G;
    const int ngrp = kBlock / G;
    // every lane of a warp runs the same number of loop trips so the shuffles
    // of dyn_group_sum always see the full warp
    const int trips = (nr + ngrp - 1) / ngrp;
    for (int t = 0; t < trips; ++t) {
        const int row = grp + t * ngrp;
        VT s = VT(0);
        if (row < nr) {
            const int a = srp[row] - j0, b = srp[row + 1] - j0;
            for (int e = a + lane; e < b; e += G) s += prod[e];
        }
        s = dyn_group_sum(s, G);
        if (lane == 0 && row < nr) st_stream(y + r0 + row, s);
    }
}

}  // namespace

void CrsTilePlan::build(const int *d_row_ptr, int64_t n, int cap_, cudaStream_t st) {
    cap = cap_;
    n_rows = n;
    n_tiles = 0;
    if (n <= 0) return;
    DevBuf flags(n);
    tiles.alloc(sizeof(int) * (n + 1));
    DevBuf nsel(sizeof(int));
    tile_flags_kernel<<<ceil_div_u(n, 256), 256, 0, st>>>(d_row_ptr, n, cap, flags.as<unsigned char>());
    SMAX_CUDA(cudaGetLastError());
    thrust::counting_iterator<int> it(0);
    size_t tb = 0;
    SMAX_CUDA(cub::DeviceSelect::Flagged(nullptr, tb, it, flags.as<unsigned char>(), tiles.as<int>(),
                                         nsel.as<int>(), (int)n, st));
    DevBuf tmp(tb);
    SMAX_CUDA(cub::DeviceSelect::Flagged(tmp.p, tb, it, flags.as<unsigned char>(), tiles.as<int>(),
                                         nsel.as<int>(), (int)n, st));
    set_last_kernel<<<1, 1, 0, st>>>(tiles.as<int>(), nsel.as<int>(), (int)n);
    SMAX_CUDA(cudaGetLastError());
    int h = 0;
    SMAX_CUDA(cudaMemcpyAsync(&h, nsel.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    SMAX_CUDA(cudaStreamSynchronize(st));
    n_tiles = h;
}

template <typename VT>
void crs_spmv(const CrsTilePlan &plan, const int *row_ptr, const int *col, const VT *val, const VT *x,
              VT *y, cudaStream_t st) {
    if (plan.n_tiles == 0) return;
    constexpr int CAP = sizeof(VT) == 8 ? 1024 : 2048;
    if (plan.cap != CAP) fail(SMAX_ERR_STATE, "CRS tile plan built for a different tile capacity");
    crs_tile_kernel<VT, CAP><<<plan.n_tiles, kBlock, 0, st>>>(plan.tiles.as<int>(), row_ptr, col, val, x, y);
    SMAX_CUDA(cudaGetLastError());
}

template void crs_spmv<double>(const CrsTilePlan &, const int *, const int *, const double *, const double *,
                               double *, cudaStream_t);
template void crs_spmv<float>(const CrsTilePlan &, const int *, const int *, const float *, const float *,
                              float *, cudaStream_t);

int crs_default_cap(int vbits) { return vbits == 64 ? 1024 : 2048; }

}  // namespace smax
