// adjoint.cu -- reverse-mode derivatives of SpMV and SpTRSV.
//
// The reference has no derivatives.  The definitions follow from y = A x and
// L x = b with a loss gradient g = dLoss/dy (or dLoss/dx):
//   SpMV:   dx = A^T g,          dval[k] = g[row(k)] * x[col(k)]
//   SpTRSV: L^T lambda = g,  db = lambda,  dval[k] = -lambda[row(k)] * x[col(k)]
// A^T is a transposed CRS copy built once on the GPU by a stable radix sort of
// the entries by column, so dx = A^T g is an ordinary (deterministic)
// warp-stream SpMV instead of a scatter with atomics.  For L^T the rows of the
// transpose are ordered so the diagonal is the last entry of each row (the
// layout of the triangular kernels); the adjoint solve then runs on the
// forward solve's level sets swept in the opposite direction.
#include "adjoint.cuh"

#include <cub/device/device_radix_sort.cuh>

namespace smax {

namespace {

__global__ void row_of_kernel(const int *__restrict__ rp, int64_t n, int *__restrict__ row_of) {
    const int lane = threadIdx.x & 31;
    const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t r = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; r < n; r += nw) {
        const int e = rp[r + 1];
        for (int j = rp[r] + lane; j < e; j += 32) row_of[j] = (int)r;
    }
}

__global__ void transpose_keys(const int *__restrict__ col, int64_t nnz, bool desc, int *__restrict__ kin,
                               int *__restrict__ vin) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nnz; i += stride) {
        const int64_t src = desc ? nnz - 1 - i : i;
        kin[i] = col[src];
        vin[i] = (int)src;
    }
}

// rp[c] = first e with sorted_col[e] >= c, for c in [0, m]
__global__ void transpose_row_ptr(const int *__restrict__ sorted_col, int64_t nnz, int64_t m, int *__restrict__ rp) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e <= nnz; e += stride) {
        const int64_t prev = e > 0 ? sorted_col[e - 1] : -1;
        const int64_t cur = e < nnz ? sorted_col[e] : m;
        for (int64_t c = prev + 1; c <= cur; ++c) rp[c] = (int)e;
    }
}

template <typename W>
__global__ void transpose_fill(const int *__restrict__ map, const int *__restrict__ row_of, const W *__restrict__ val,
                               int64_t nnz, int *__restrict__ tcol, W *__restrict__ tval) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < nnz; e += stride) {
        const int k = map[e];
        if (tcol) tcol[e] = row_of[k];
        tval[e] = val[k];
    }
}

template <typename VT>
__global__ void sddmm_outer_kernel(const int *__restrict__ row_of, const int *__restrict__ col, int64_t nnz, VT s,
                                   const VT *__restrict__ g, const VT *__restrict__ x, VT *__restrict__ dval) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < nnz; k += stride)
        dval[k] = s * ld_keep(g + row_of[k]) * ld_keep(x + col[k]);
}

__global__ void diag_last_kernel(const int *__restrict__ rp, const int *__restrict__ col, int64_t n,
                                 DevStatus *status) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < n; r += stride) {
        const int e = rp[r + 1] - 1;
        if (e < rp[r] || col[e] != (int)r) report(status, SMAX_ERR_NO_DIAG, r);
    }
}

unsigned grid_for(int64_t work, int threads) {
    const int64_t cap = (int64_t)sm_count() * 8;
    int64_t g = (work + threads - 1) / threads;
    if (g > cap) g = cap;
    return (unsigned)(g < 1 ? 1 : g);
}

int key_bits(int64_t m) {
    int b = 1;
    while (b < 31 && (int64_t(1) << b) < m) ++b;
    return b;
}

void gather_values(const DevCRS &a, int vbytes, DevTranspose &t, bool with_cols, cudaStream_t st) {
    const int64_t nnz = a.nnz;
    if (nnz == 0) return;
    const unsigned g = grid_for(nnz, 256);
    int *tcol = with_cols ? t.at.col.as<int>() : nullptr;
    if (vbytes == 8)
        transpose_fill<unsigned long long><<<g, 256, 0, st>>>(t.map.as<int>(), t.row_of.as<int>(),
                                                              a.val.as<unsigned long long>(), nnz, tcol,
                                                              t.at.val.as<unsigned long long>());
    else
        transpose_fill<unsigned><<<g, 256, 0, st>>>(t.map.as<int>(), t.row_of.as<int>(), a.val.as<unsigned>(), nnz,
                                                    tcol, t.at.val.as<unsigned>());
    SMAX_CUDA(cudaGetLastError());
}

}  // namespace

void crs_row_of(const DevCRS &a, DevBuf &row_of, cudaStream_t st) {
    row_of.alloc(sizeof(int) * (a.nnz > 0 ? a.nnz : 1));
    if (a.nnz == 0 || a.n_rows == 0) return;
    row_of_kernel<<<grid_for(a.n_rows * 32, 256), 256, 0, st>>>(a.rp(), a.n_rows, row_of.as<int>());
    SMAX_CUDA(cudaGetLastError());
}

void build_transpose(const DevCRS &a, int vbytes, bool desc, bool with_plan, DevTranspose &t, cudaStream_t st) {
    const int64_t n = a.n_rows, m = a.n_cols, nnz = a.nnz;
    crs_row_of(a, t.row_of, st);
    const size_t ib = sizeof(int) * (nnz > 0 ? nnz : 1);
    t.map.alloc(ib);
    DevBuf kin(ib), vin(ib), kout(ib);
    if (nnz > 0) {
        transpose_keys<<<grid_for(nnz, 256), 256, 0, st>>>(a.ci(), nnz, desc, kin.as<int>(), vin.as<int>());
        SMAX_CUDA(cudaGetLastError());
        size_t tb = 0;
        SMAX_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tb, kin.as<int>(), kout.as<int>(), vin.as<int>(),
                                                  t.map.as<int>(), (int)nnz, 0, key_bits(m), st));
        DevBuf tmp(tb);
        SMAX_CUDA(cub::DeviceRadixSort::SortPairs(tmp.p, tb, kin.as<int>(), kout.as<int>(), vin.as<int>(),
                                                  t.map.as<int>(), (int)nnz, 0, key_bits(m), st));
    }
    DevCRS &at = t.at;
    at.n_rows = m;
    at.n_cols = n;
    at.nnz = nnz;
    const int64_t pad = crs_stream_pad();
    const int64_t cap = (nnz + pad - 1) / pad * pad;
    at.row_ptr.alloc(sizeof(int) * (m + 1));
    at.col.alloc(sizeof(int) * (cap > 0 ? cap : 1));
    at.val.alloc((size_t)vbytes * (cap > 0 ? cap : 1));
    if (cap > nnz) {
        SMAX_CUDA(cudaMemsetAsync(at.col.as<int>() + nnz, 0, sizeof(int) * (cap - nnz), st));
        SMAX_CUDA(cudaMemsetAsync(static_cast<char *>(at.val.p) + (size_t)vbytes * nnz, 0,
                                  (size_t)vbytes * (cap - nnz), st));
    }
    transpose_row_ptr<<<grid_for(nnz + 1, 256), 256, 0, st>>>(kout.as<int>(), nnz, m, at.row_ptr.as<int>());
    SMAX_CUDA(cudaGetLastError());
    gather_values(a, vbytes, t, true, st);
    t.plan = CrsStreamPlan();
    if (with_plan) t.plan.build(at.rp(), m, nnz, vbytes, st);
    t.has_plan = with_plan;
    t.descending = desc;
    t.built = true;
    // the temporaries are freed when this returns; the stream must be done with them
    SMAX_CUDA(cudaStreamSynchronize(st));
}

void refresh_transpose_values(const DevCRS &a, int vbytes, DevTranspose &t, cudaStream_t st) {
    if (t.built) gather_values(a, vbytes, t, false, st);
}

template <typename VT>
void sddmm_outer(const DevCRS &a, const int *row_of, VT s, const VT *g, const VT *x, VT *dval, cudaStream_t st) {
    if (a.nnz == 0) return;
    sddmm_outer_kernel<VT><<<grid_for(a.nnz, 256), 256, 0, st>>>(row_of, a.ci(), a.nnz, s, g, x, dval);
    SMAX_CUDA(cudaGetLastError());
}

void check_diag_last(const DevCRS &a, DevStatus *status, cudaStream_t st) {
    if (a.n_rows == 0) return;
    diag_last_kernel<<<grid_for(a.n_rows, 256), 256, 0, st>>>(a.rp(), a.ci(), a.n_rows, status);
    SMAX_CUDA(cudaGetLastError());
}

template void sddmm_outer<double>(const DevCRS &, const int *, double, const double *, const double *, double *,
                                  cudaStream_t);
template void sddmm_outer<float>(const DevCRS &, const int *, float, const float *, const float *, float *,
                                 cudaStream_t);

}  // namespace smax
