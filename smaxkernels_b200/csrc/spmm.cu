// spmm.cu -- CRS SpMM Y = A X against a block of k dense vectors, sm_100a.
//
// Reference semantics: SPMM::CPU::naive_crs_spmm_row_maj / _col_maj
// (src/kernels/spmm/spmm_cpu/spmm_cpu_crs_impl.hpp:9-89).  Row-major blocks
// (X[col*k+v], Y[row*k+v]) are the layout the platform is built for: a row of
// X is k contiguous values, so one group of G lanes owns one row of A and
// reads/writes whole rows of X/Y with 128-bit loads and stores.  The group
// loads G (col, val) pairs of its row at once (coalesced) and broadcasts them
// with shuffles; each lane accumulates NV vectors of VEC = 16/sizeof(VT)
// values.  X rows are gathered through L2 (neighbouring rows of a stencil
// matrix reuse them); A is streamed once with evict-first loads.
// Column-major blocks are k independent SpMVs on the columns and reuse the
// CRS SpMV kernel (abi.cu).
#include "spmv_formats.cuh"

namespace smax {

namespace {

template <typename VT> struct V16;
template <> struct V16<double> { using T = double2; static constexpr int N = 2; };
template <> struct V16<float> { using T = float4; static constexpr int N = 4; };

// One row of Y from its group of G lanes (lane g of the group, gmask the
// group's lanes): NV vectors of VEC values per lane, k == G * NV * VEC (VEC
// == 1 is the scalar path for k not divisible by the vector width).
template <typename VT, int G, int NV, int VEC>
__device__ __forceinline__ void spmm_row(int64_t row, int g, unsigned gmask, const int *__restrict__ row_ptr,
                                         const int *__restrict__ col, const VT *__restrict__ val, int64_t k,
                                         const VT *__restrict__ X, VT *__restrict__ Y) {
    VT acc[NV][VEC];
#pragma unroll
    for (int m = 0; m < NV; ++m)
#pragma unroll
        for (int i = 0; i < VEC; ++i) acc[m][i] = VT(0);
    const int s = row_ptr[row], e = row_ptr[row + 1];
    // FP32: the group's next G (col, val) pairs are loaded while the current
    // ones are used (k = 16 / 64 on the 27-point stencil: 7 % / 4 % faster);
    // FP64: the extra registers cost more occupancy than the overlap gains
    constexpr bool kAhead = sizeof(VT) == 4;
    int nc = 0;
    VT nv = VT(0);
    if (kAhead && s + g < e) {
        nc = ld_stream(col + s + g);
        nv = ld_stream(val + s + g);
    }
    for (int j0 = s; j0 < e; j0 += G) {
        const int jj = j0 + g;
        int myc;
        VT myv;
        if constexpr (kAhead) {
            myc = nc;
            myv = nv;
            nc = jj + G < e ? ld_stream(col + jj + G) : 0;
            nv = jj + G < e ? ld_stream(val + jj + G) : VT(0);
        } else {
            myc = jj < e ? ld_stream(col + jj) : 0;
            myv = jj < e ? ld_stream(val + jj) : VT(0);
        }
        const int cnt = min(G, e - j0);
        // unrolled so the X-row loads of consecutive entries overlap; holding
        // more rows in registers lowered occupancy and was measured slower
#pragma unroll 4
        for (int t = 0; t < cnt; ++t) {
            const int c = __shfl_sync(gmask, myc, t, G);
            const VT v = __shfl_sync(gmask, myv, t, G);
            const VT *xr = X + (int64_t)c * k;
#pragma unroll
            for (int m = 0; m < NV; ++m) {
                const int off = (m * G + g) * VEC;
                if constexpr (VEC == 2) {
                    const double2 xv = __ldg(reinterpret_cast<const double2 *>(xr + off));
                    acc[m][0] += v * xv.x;
                    acc[m][1] += v * xv.y;
                } else if constexpr (VEC == 4) {
                    const float4 xv = __ldg(reinterpret_cast<const float4 *>(xr + off));
                    acc[m][0] += v * xv.x;
                    acc[m][1] += v * xv.y;
                    acc[m][2] += v * xv.z;
                    acc[m][3] += v * xv.w;
                } else {
                    acc[m][0] += v * __ldg(xr + off);
                }
            }
        }
    }
    VT *yr = Y + row * k;
#pragma unroll
    for (int m = 0; m < NV; ++m) {
        const int off = (m * G + g) * VEC;
        if constexpr (VEC == 2) {
            __stcs(reinterpret_cast<double2 *>(yr + off), make_double2(acc[m][0], acc[m][1]));
        } else if constexpr (VEC == 4) {
            __stcs(reinterpret_cast<float4 *>(yr + off), make_float4(acc[m][0], acc[m][1], acc[m][2], acc[m][3]));
        } else {
            __stcs(yr + off, acc[m][0]);
        }
    }
}

template <int G> __device__ __forceinline__ unsigned group_mask(int lane) {
    return (G == 32) ? 0xffffffffu : (((1u << G) - 1u) << (lane - lane % G));
}

// a grid of all rows, one group of G lanes per row
template <typename VT, int G, int NV, int VEC>
__global__ void __launch_bounds__(256) spmm_row_major_kernel(const int *__restrict__ row_ptr,
                                                             const int *__restrict__ col,
                                                             const VT *__restrict__ val, int64_t n_rows, int64_t k,
                                                             const VT *__restrict__ X, VT *__restrict__ Y) {
    const int lane = threadIdx.x & 31;
    const int64_t row = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) / G;
    if (row >= n_rows) return;  // whole groups leave together
    spmm_row<VT, G, NV, VEC>(row, lane % G, group_mask<G>(lane), row_ptr, col, val, k, X, Y);
}

// CTA b walks rows ranges[b] .. ranges[b+1] in order, kWalkThreads / G rows
// at a time
constexpr int kWalkThreads = 1024;
template <typename VT, int G, int NV, int VEC>
__global__ void __launch_bounds__(kWalkThreads, 1)
    spmm_walk_kernel(const int *__restrict__ row_ptr, const int *__restrict__ col, const VT *__restrict__ val,
                     const int64_t *__restrict__ ranges, int64_t k, const VT *__restrict__ X, VT *__restrict__ Y) {
    const int lane = threadIdx.x & 31;
    const int64_t r0 = ranges[blockIdx.x], r1 = ranges[blockIdx.x + 1];
    for (int64_t row = r0 + threadIdx.x / G; row < r1; row += kWalkThreads / G)
        spmm_row<VT, G, NV, VEC>(row, lane % G, group_mask<G>(lane), row_ptr, col, val, k, X, Y);
}

// ranges[b] = first row r with row_ptr[r] + r >= b * (nnz + n) / grid
// (nonzeros and rows balanced: a row costs its entries plus its Y write)
__global__ void walk_ranges_kernel(const int *__restrict__ row_ptr, int64_t n, int grid, int64_t *__restrict__ ranges) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b > grid) return;
    const int64_t total = (int64_t)row_ptr[n] + n;
    const int64_t target = total * b / grid;
    int64_t lo = 0, hi = n;
    while (lo < hi) {
        const int64_t mid = (lo + hi) >> 1;
        if ((int64_t)row_ptr[mid] + mid < target) lo = mid + 1;
        else hi = mid;
    }
    ranges[b] = b == grid ? n : lo;
}

template <typename VT, int G, int NV, int VEC>
void launch_rm(const DevCRS &a, int64_t k, const VT *X, VT *Y, cudaStream_t st, const SpmmPlan *walk) {
    if (walk) {
        static bool carve[64] = {};
        int dev = 0;
        cudaGetDevice(&dev);
        if (dev >= 0 && dev < 64 && !carve[dev]) {
            // no shared memory: the whole unified L1 holds X rows
            SMAX_CUDA(cudaFuncSetAttribute(spmm_walk_kernel<VT, G, NV, VEC>,
                                           cudaFuncAttributePreferredSharedMemoryCarveout, 0));
            carve[dev] = true;
        }
        spmm_walk_kernel<VT, G, NV, VEC><<<walk->grid, kWalkThreads, 0, st>>>(
            a.rp(), a.ci(), a.val.template as<VT>(), walk->ranges.as<int64_t>(), k, X, Y);
        return;
    }
    const uint64_t threads = (uint64_t)a.n_rows * G;
    spmm_row_major_kernel<VT, G, NV, VEC><<<ceil_div_u(threads, 256), 256, 0, st>>>(a.rp(), a.ci(),
                                                                                    a.val.template as<VT>(),
                                                                                    a.n_rows, k, X, Y);
}

const SpmmPlan *walk_plan(const DevCRS &a, SpmmPlan *plan, cudaStream_t st) {
    if (!plan) return nullptr;
    if (plan->key != a.row_ptr.p || plan->n != a.n_rows || plan->nnz != a.nnz) {
        plan->grid = sm_count();
        plan->ranges.ensure(sizeof(int64_t) * (plan->grid + 1));
        walk_ranges_kernel<<<ceil_div_u((uint64_t)plan->grid + 1, 256), 256, 0, st>>>(a.rp(), a.n_rows, plan->grid,
                                                                                      plan->ranges.as<int64_t>());
        SMAX_CUDA(cudaGetLastError());
        plan->key = a.row_ptr.p;
        plan->n = a.n_rows;
        plan->nnz = a.nnz;
    }
    return plan;
}

// scalar fallback for any k: one warp per row, lanes over the k columns
template <typename VT>
__global__ void spmm_row_major_generic(const int *__restrict__ row_ptr, const int *__restrict__ col,
                                       const VT *__restrict__ val, int64_t n_rows, int64_t k,
                                       const VT *__restrict__ X, VT *__restrict__ Y) {
    const int64_t row = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (row >= n_rows) return;
    const int s = row_ptr[row], e = row_ptr[row + 1];
    for (int64_t v = lane; v < k; v += 32) {
        VT acc = VT(0);
        for (int j = s; j < e; ++j) acc += val[j] * X[(int64_t)col[j] * k + v];
        Y[row * k + v] = acc;
    }
}

}  // namespace

template <typename VT>
void crs_spmm_row_major(const DevCRS &a, int64_t k, const VT *X, VT *Y, cudaStream_t st, SpmmPlan *plan,
                        int variant) {
    if (a.n_rows == 0 || k == 0) return;
    const SpmmPlan *w = variant == 2 ? walk_plan(a, plan, st) : nullptr;
    constexpr int VEC = V16<VT>::N;
    // vector path when k is a multiple of VEC: k/VEC vectors spread over G lanes
    // (and X, Y 16-byte aligned: offsets given to apply() may shift them)
    const bool aligned = ((reinterpret_cast<uintptr_t>(X) | reinterpret_cast<uintptr_t>(Y)) & 15) == 0;
    const int64_t nvec = (aligned && k % VEC == 0) ? k / VEC : 0;
    bool done = true;
    switch (nvec) {
    case 1: launch_rm<VT, 1, 1, VEC>(a, k, X, Y, st, w); break;
    case 2: launch_rm<VT, 2, 1, VEC>(a, k, X, Y, st, w); break;
    case 4: launch_rm<VT, 4, 1, VEC>(a, k, X, Y, st, w); break;
    case 8: launch_rm<VT, 8, 1, VEC>(a, k, X, Y, st, w); break;
    // 16 and 32 vectors: 8 lanes per row with 2 / 4 vectors each (k = 64 on
    // the 27-point stencil: FP32 0.99 -> 0.84 ms, FP64 2.05 -> 1.58 ms against
    // one vector per lane); 64 vectors: 16 lanes with 4 each (k = 128 FP64
    // 2.91 -> 2.85 ms, k = 256 FP32 2.84 -> 2.73 ms); more vectors per lane
    // cost occupancy
    case 16: launch_rm<VT, 8, 2, VEC>(a, k, X, Y, st, w); break;
    case 32: launch_rm<VT, 8, 4, VEC>(a, k, X, Y, st, w); break;
    case 64: launch_rm<VT, 16, 4, VEC>(a, k, X, Y, st, w); break;
    case 128: launch_rm<VT, 32, 4, VEC>(a, k, X, Y, st, w); break;
    default: done = false;
    }
    if (!done) {
        // k not a power-of-two number of vectors: small k -> scalar lanes per
        // element, otherwise one warp per row
        if (k == 1) launch_rm<VT, 1, 1, 1>(a, k, X, Y, st, w);
        else if (k == 2) launch_rm<VT, 2, 1, 1>(a, k, X, Y, st, w);
        else if (k == 4) launch_rm<VT, 4, 1, 1>(a, k, X, Y, st, w);
        else if (k == 8) launch_rm<VT, 8, 1, 1>(a, k, X, Y, st, w);
        else if (k == 16) launch_rm<VT, 16, 1, 1>(a, k, X, Y, st, w);
        else
            spmm_row_major_generic<VT><<<ceil_div_u((uint64_t)a.n_rows * 32, 256), 256, 0, st>>>(
                a.rp(), a.ci(), a.val.template as<VT>(), a.n_rows, k, X, Y);
    }
    SMAX_CUDA(cudaGetLastError());
}

template void crs_spmm_row_major<double>(const DevCRS &, int64_t, const double *, double *, cudaStream_t, SpmmPlan *,
                                         int);
template void crs_spmm_row_major<float>(const DevCRS &, int64_t, const float *, float *, cudaStream_t, SpmmPlan *,
                                        int);

}  // namespace smax
