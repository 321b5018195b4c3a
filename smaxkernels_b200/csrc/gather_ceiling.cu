// gather_ceiling.cu -- measurement kernel: the cost of the CRS SpMV's memory
// traffic without its row bookkeeping.
//
// The warp-stream CRS SpMV (spmv_crs_stream.cu) reads val and col as a
// stream and gathers x[col[e]] for every entry.  With uniformly random
// columns those gathers are one independent 32-byte sector each, and on
// sm_100a their cost is set by how many separate requests the SM can issue,
// not by bytes.  This kernel does exactly that traffic -- the same 512-entry
// warp slices, the same 16-byte streaming loads of 4 consecutive entries per
// lane, one gather per entry -- and sums val*x per slice, so its time is the
// floor any kernel with this access pattern can reach on the same arrays:
//   mode 0  gathers: lanes [0, tma_lanes) fetch their four x values with one
//           TMA tile::gather4 (four 32-byte rows into shared memory), the
//           other lanes with ordinary L2 loads (ld.global.cg);
//   mode 1  stream only: val and col are read, x is not touched.
// Warps are persistent and keep `depth` chunks of 128 entries in flight
// (ring of shared-memory slots and registers).  Nothing here is on a product
// path; smax_measure_gather() is called by the benchmark.
#include <algorithm>
#include <cstring>

#include "tma.cuh"

namespace smax {
namespace {

constexpr int kSlice = 512;   // entries per warp slice (as the CRS stream kernel)
constexpr int kChunk = 128;   // entries per chunk (32 lanes x 4)
constexpr int kWarps = 8;     // warps per CTA
constexpr int kSlotBytes = 128;  // one gather4: four 32-byte rows
constexpr int kBarBytes = 1024;  // mbarrier area at the start of shared memory

template <typename VT> struct Vec4;
template <> struct Vec4<double> {
    double v[4];
    __device__ __forceinline__ void load(const double *p) {
        double2 a = __ldcs(reinterpret_cast<const double2 *>(p));
        double2 b = __ldcs(reinterpret_cast<const double2 *>(p + 2));
        v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y;
    }
};
template <> struct Vec4<float> {
    float v[4];
    __device__ __forceinline__ void load(const float *p) {
        float4 a = __ldcs(reinterpret_cast<const float4 *>(p));
        v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w;
    }
};

template <typename VT, int D>
__global__ void __launch_bounds__(kWarps * 32)
    gather_probe_kernel(const int *__restrict__ col, const VT *__restrict__ val, const VT *__restrict__ x,
                        int64_t n_slices, int tma_lanes, int mode, const __grid_constant__ CUtensorMap map,
                        int64_t x_rows, VT *__restrict__ out, int *__restrict__ err, long long spin_limit) {
    constexpr int RW = 32 / sizeof(VT);  // elements per gathered row
    constexpr int SH = RW == 4 ? 2 : 3;  // log2(RW)
    extern __shared__ __align__(128) unsigned char smem[];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const int64_t gw = (int64_t)blockIdx.x * kWarps + wib;
    const int64_t tw = (int64_t)gridDim.x * kWarps;
    uint64_t *bars = reinterpret_cast<uint64_t *>(smem) + wib * D;
    unsigned char *slots = smem + kBarBytes + (size_t)wib * D * 32 * kSlotBytes;
    const bool use_tma = mode == 0 && tma_lanes > 0;
    const bool my_tma = use_tma && lane < tma_lanes;
    if (use_tma) {
        if (lane == 0) {
#pragma unroll
            for (int s = 0; s < D; ++s) mbar_init(bars + s, 1);
            mbar_fence_init();
        }
        __syncwarp();
    }
    const int64_t my_slices = gw < n_slices ? (n_slices - gw + tw - 1) / tw : 0;
    const int64_t nj = my_slices * (kSlice / kChunk);

    int4 c[D];
    Vec4<VT> v[D];
    auto issue = [&](int64_t j, int s) {
        const int64_t t = gw + (j >> 2) * tw;
        const int64_t e = t * kSlice + (j & 3) * kChunk + lane * 4;
        c[s] = __ldcs(reinterpret_cast<const int4 *>(col + e));
        v[s].load(val + e);
        if (use_tma) {
            if (lane == 0) mbar_arrive_expect_tx(bars + s, (uint32_t)tma_lanes * kSlotBytes);
            __syncwarp();
            if (my_tma) {
                int r0 = c[s].x >> SH, r1 = c[s].y >> SH, r2 = c[s].z >> SH, r3 = c[s].w >> SH;
                r0 = r0 < x_rows ? r0 : 0; r1 = r1 < x_rows ? r1 : 0;
                r2 = r2 < x_rows ? r2 : 0; r3 = r3 < x_rows ? r3 : 0;
                tma_gather4(slots + ((size_t)s * 32 + lane) * kSlotBytes, &map, r0, r1, r2, r3, bars + s);
            }
        }
    };
    VT acc = VT(0);
    auto consume = [&](int64_t j, int s) {
        const int cc[4] = {c[s].x, c[s].y, c[s].z, c[s].w};
        if (mode == 1) {
#pragma unroll
            for (int i = 0; i < 4; ++i) acc += v[s].v[i] * (VT)cc[i];
        } else {
            if (use_tma) {
                if (!mbar_wait_bounded(bars + s, (uint32_t)((j / D) & 1), spin_limit)) {
                    atomicExch(err, 1);
                    (void)mbar_wait_bounded(bars + s, (uint32_t)((j / D) & 1), spin_limit);
                }
            }
            const VT *slot = reinterpret_cast<const VT *>(slots + ((size_t)s * 32 + lane) * kSlotBytes);
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                const int r = cc[i] >> SH;
                const VT xv = (my_tma && r < x_rows) ? slot[i * RW + (cc[i] & (RW - 1))] : __ldcg(x + cc[i]);
                acc += v[s].v[i] * xv;
            }
            if (my_tma) fence_proxy_async_smem();  // this lane's reads of its slot, before the slot's next copy
        }
        if ((j & 3) == 3) {  // end of a slice: one sum per slice, whatever the grid
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
            if (lane == 0) out[gw + (j >> 2) * tw] = acc;
            acc = VT(0);
        }
    };

#pragma unroll
    for (int s = 0; s < D; ++s)
        if (s < nj) issue(s, s);
    for (int64_t j0 = 0; j0 < nj; j0 += D) {
#pragma unroll
        for (int s = 0; s < D; ++s) {
            const int64_t j = j0 + s;
            if (j < nj) {
                consume(j, s);
                if (j + D < nj) issue(j + D, s);
            }
        }
    }
}

template <typename VT, int D>
void launch_probe(int mode, int tma_lanes, int64_t n_slices, const int *col, const VT *val, const VT *x,
                  int64_t n_cols, VT *out, int *err, cudaStream_t st) {
    CUtensorMap map;
    memset(&map, 0, sizeof(map));
    const bool tma = mode == 0 && tma_lanes > 0;
    if (tma && !make_gather_map(&map, x, n_cols, sizeof(VT)))
        fail(SMAX_ERR_UNSUPPORTED, "x cannot be described by a TMA gather map (alignment or size)");
    const int64_t x_rows = gather_rows(n_cols, sizeof(VT));
    const size_t smem = tma ? kBarBytes + (size_t)kWarps * D * 32 * kSlotBytes : kBarBytes;
    auto kern = gather_probe_kernel<VT, D>;
    SMAX_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int per_sm = 0;
    SMAX_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kWarps * 32, smem));
    if (per_sm < 1) fail(SMAX_ERR_UNSUPPORTED, "probe kernel does not fit on an SM");
    const int64_t want = (n_slices + kWarps - 1) / kWarps;
    const unsigned grid = (unsigned)std::min<int64_t>(want, (int64_t)sm_count() * per_sm);
    kern<<<grid, kWarps * 32, smem, st>>>(col, val, x, n_slices, tma_lanes, mode, map, x_rows, out, err,
                                          1ll << 20);
    SMAX_CUDA(cudaGetLastError());
}

template <typename VT>
void probe_t(int mode, int tma_lanes, int depth, int64_t n_slices, const void *col, const void *val,
             const void *x, int64_t n_cols, void *out, int *err, cudaStream_t st) {
    const int *c = static_cast<const int *>(col);
    const VT *v = static_cast<const VT *>(val);
    const VT *xx = static_cast<const VT *>(x);
    VT *o = static_cast<VT *>(out);
    switch (depth) {
        case 1: launch_probe<VT, 1>(mode, tma_lanes, n_slices, c, v, xx, n_cols, o, err, st); break;
        case 2: launch_probe<VT, 2>(mode, tma_lanes, n_slices, c, v, xx, n_cols, o, err, st); break;
        case 4: launch_probe<VT, 4>(mode, tma_lanes, n_slices, c, v, xx, n_cols, o, err, st); break;
        default: fail(SMAX_ERR_BAD_ARG, "depth must be 1, 2 or 4");
    }
}

}  // namespace
}  // namespace smax

using namespace smax;

extern "C" smax_status smax_measure_gather(int float_type, int mode, int tma_lanes, int depth, uint64_t n_slices,
                                           const void *d_col, const void *d_val, const void *d_x, uint64_t n_cols,
                                           void *d_out, void *d_err, void *stream) {
    return guarded([&] {
        if (float_type != SMAX_FLOAT32 && float_type != SMAX_FLOAT64)
            fail(SMAX_ERR_UNSUPPORTED_TYPE, "value type must be float32 or float64");
        if (mode != 0 && mode != 1) fail(SMAX_ERR_BAD_ARG, "mode must be 0 (gathers) or 1 (stream only)");
        if (tma_lanes < 0 || tma_lanes > 32) fail(SMAX_ERR_BAD_ARG, "tma_lanes must be in [0, 32]");
        if (n_cols < 1 || n_cols >= (1ull << 31)) fail(SMAX_ERR_BAD_ARG, "n_cols out of range");
        if (!d_col || !d_val || !d_x || !d_out || !d_err) fail(SMAX_ERR_BAD_ARG, "null device pointer");
        if (((uintptr_t)d_col & 15u) || ((uintptr_t)d_val & 15u))
            fail(SMAX_ERR_BAD_ARG, "col and val must be 16-byte aligned");
        if (n_slices == 0) return;
        cudaStream_t st = static_cast<cudaStream_t>(stream);
        if (float_type == SMAX_FLOAT64)
            probe_t<double>(mode, tma_lanes, depth, (int64_t)n_slices, d_col, d_val, d_x, (int64_t)n_cols, d_out,
                            static_cast<int *>(d_err), st);
        else
            probe_t<float>(mode, tma_lanes, depth, (int64_t)n_slices, d_col, d_val, d_x, (int64_t)n_cols, d_out,
                           static_cast<int *>(d_err), st);
    });
}
