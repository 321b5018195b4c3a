// spmv_noalloc.cu -- CRS SpMV for callers that cannot allocate device memory.
//
// Who needs it: code that may not call cudaMalloc -- an application whose
// memory pool already owns the whole GPU, a plugin whose host forbids device
// allocations, or a latency-critical loop that must not enter the allocator.
// smax_spmv_crs_noalloc() runs the warp-stream CRS SpMV (the algorithm of
// spmv_crs_stream.cu) on arrays the caller already has in device memory and
// keeps everything else it needs -- the row-end bit mask, the slice table, the
// slice carries, the list of non-empty rows and a status word -- in one
// file-scope __device__ array of fixed size.  It calls no cudaMalloc, no
// cudaFree and no allocating library routine.
//
// Properties of the fixed scratch area:
//   * every GPU that loads the library holds it (SMAX_NOALLOC_SCRATCH_BYTES)
//     until the process exits;
//   * all calls share it and it keeps the last call's contents; what must
//     start at zero (the bit mask, the status word) is cleared by each call;
//   * calls that overlap on the GPU (two streams, or two host threads) race
//     on it -- order them on one stream or serialise them;
//   * the first call on a device does the set-up: it looks up the array's
//     device address (cudaGetSymbolAddress) with that device current; make
//     that first call before any stream capture.
// Limits: n_rows <= SMAX_NOALLOC_MAX_ROWS, nnz <= SMAX_NOALLOC_MAX_NNZ; larger
// problems are rejected with SMAX_ERR_BAD_ARG before any work is queued.
#include <mutex>

#include "common.cuh"

namespace smax {
namespace {

constexpr int64_t kMaxRows = SMAX_NOALLOC_MAX_ROWS;
constexpr int64_t kMaxNnz = SMAX_NOALLOC_MAX_NNZ;
constexpr int kW = 512;                         // entries per warp slice
constexpr int64_t kMaxTasks = kMaxNnz / kW + 1;
constexpr int kRowsPerBlock = 1024;             // rows per block of the row-list scan
constexpr int64_t kMaxBlocks = (kMaxRows + kRowsPerBlock - 1) / kRowsPerBlock;

constexpr size_t align256(size_t b) { return (b + 255) / 256 * 256; }
// byte offsets of the regions of the scratch array
constexpr size_t kOffStatus = 0;                                                 // DevStatus + n_nonempty
constexpr size_t kOffEndbits = 256;
constexpr size_t kOffTaskRank = kOffEndbits + align256(sizeof(uint32_t) * (kMaxTasks * kW / 32 + 1));
constexpr size_t kOffCarryVal = kOffTaskRank + align256(sizeof(int) * kMaxTasks);
constexpr size_t kOffCarryRank = kOffCarryVal + align256(sizeof(double) * kMaxTasks);
constexpr size_t kOffRowList = kOffCarryRank + align256(sizeof(int) * kMaxTasks);
constexpr size_t kOffBlockCnt = kOffRowList + align256(sizeof(int) * kMaxRows);
constexpr size_t kScratchBytes = kOffBlockCnt + align256(sizeof(int) * (kMaxBlocks + 1));
static_assert(kScratchBytes <= SMAX_NOALLOC_SCRATCH_BYTES, "scratch layout exceeds the stated size");

// The scratch area.  Host code must not use this name as an address: it is a
// host-side stand-in; the device address comes from cudaGetSymbolAddress.
static __device__ __align__(256) unsigned char g_noalloc_scratch[SMAX_NOALLOC_SCRATCH_BYTES];

struct Scratch {
    DevStatus *status;
    int *n_nonempty;
    uint32_t *endbits;
    int *task_rank;
    void *carry_val;
    int *carry_rank;
    int *row_list;
    int *block_cnt;
};

Scratch carve(unsigned char *base) {
    Scratch s;
    s.status = reinterpret_cast<DevStatus *>(base + kOffStatus);
    s.n_nonempty = reinterpret_cast<int *>(base + kOffStatus + sizeof(DevStatus));
    s.endbits = reinterpret_cast<uint32_t *>(base + kOffEndbits);
    s.task_rank = reinterpret_cast<int *>(base + kOffTaskRank);
    s.carry_val = base + kOffCarryVal;
    s.carry_rank = reinterpret_cast<int *>(base + kOffCarryRank);
    s.row_list = reinterpret_cast<int *>(base + kOffRowList);
    s.block_cnt = reinterpret_cast<int *>(base + kOffBlockCnt);
    return s;
}

// ---------------------------------------------------------------- set-up --
// Device address of the scratch array, looked up once per device with that
// device current.
constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
unsigned char *g_scratch_ptr[kMaxDevices] = {nullptr};

unsigned char *scratch_for_current_device() {
    int dev = 0;
    SMAX_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) fail(SMAX_ERR_UNSUPPORTED, "device ordinal out of range");
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (!g_scratch_ptr[dev]) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || p == nullptr) {
            (void)cudaGetLastError();
            fail(SMAX_ERR_CUDA, std::string("cudaGetSymbolAddress of the no-alloc scratch failed: ") +
                                    cudaGetErrorString(e));
        }
        g_scratch_ptr[dev] = static_cast<unsigned char *>(p);
    }
    return g_scratch_ptr[dev];
}

// ---------------------------------------------------------------- kernels --
// Validation (row_ptr monotone, ends at nnz; columns in range), row-end bits,
// y = 0 for rows without entries, and per-block counts of non-empty rows.
__global__ void na_prepare(const int *__restrict__ row_ptr, const int *__restrict__ col, int64_t n, int64_t nnz,
                           int64_t n_cols, Scratch s, void *y, int vbytes) {
    __shared__ int warp_cnt[kRowsPerBlock / 32];
    const int64_t r = (int64_t)blockIdx.x * kRowsPerBlock + threadIdx.x;
    if (blockIdx.x == 0 && threadIdx.x == 0 && (row_ptr[0] != 0 || row_ptr[n] != nnz))
        report(s.status, SMAX_ERR_BAD_ARG, 0);
    int nonempty = 0;
    if (r < n) {
        const int a = row_ptr[r], b = row_ptr[r + 1];
        // any bound outside [0, nnz] or a decreasing pair is an error; the
        // row-end bit is set only for 0 <= a < b <= nnz, so a malformed
        // row_ptr never writes outside the bit mask
        if (b < a || a < 0 || (int64_t)b > nnz) report(s.status, SMAX_ERR_BAD_ARG, r);
        if (a >= 0 && b > a && (int64_t)b <= nnz) {
            nonempty = 1;
            atomicOr(s.endbits + ((b - 1) >> 5), 1u << ((b - 1) & 31));
        } else if (b == a) {
            if (vbytes == 8) static_cast<double *>(y)[r] = 0.0;
            else static_cast<float *>(y)[r] = 0.f;
        }
    }
    const unsigned bal = __ballot_sync(0xffffffffu, nonempty);
    if ((threadIdx.x & 31) == 0) warp_cnt[threadIdx.x >> 5] = __popc(bal);
    __syncthreads();
    if (threadIdx.x == 0) {
        int t = 0;
        for (int w = 0; w < kRowsPerBlock / 32; ++w) t += warp_cnt[w];
        s.block_cnt[blockIdx.x] = t;
    }
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < nnz; j += stride) {
        const int c = col[j];
        if (c < 0 || c >= n_cols) report(s.status, SMAX_ERR_COL_OOB, j);
    }
}

// Exclusive scan of the per-block counts (one CTA; at most kMaxBlocks values).
__global__ void na_scan_blocks(Scratch s, int n_blocks) {
    __shared__ int buf[kMaxBlocks + 1];
    for (int i = threadIdx.x; i < n_blocks; i += blockDim.x) buf[i] = s.block_cnt[i];
    __syncthreads();
    if (threadIdx.x == 0) {
        int run = 0;
        for (int i = 0; i < n_blocks; ++i) {
            const int c = buf[i];
            buf[i] = run;
            run += c;
        }
        *s.n_nonempty = run;
    }
    __syncthreads();
    for (int i = threadIdx.x; i < n_blocks; i += blockDim.x) s.block_cnt[i] = buf[i];
}

// row_list[k] = index of the k-th non-empty row.
__global__ void na_row_list(const int *__restrict__ row_ptr, int64_t n, Scratch s) {
    __shared__ int warp_off[kRowsPerBlock / 32];
    if (s.status->code != 0) return;
    const int64_t r = (int64_t)blockIdx.x * kRowsPerBlock + threadIdx.x;
    const int nonempty = (r < n && row_ptr[r + 1] > row_ptr[r]) ? 1 : 0;
    const unsigned bal = __ballot_sync(0xffffffffu, nonempty);
    const int lane = threadIdx.x & 31;
    if (lane == 0) warp_off[threadIdx.x >> 5] = __popc(bal);
    __syncthreads();
    if (threadIdx.x == 0) {
        int run = 0;
        for (int w = 0; w < kRowsPerBlock / 32; ++w) {
            const int c = warp_off[w];
            warp_off[w] = run;
            run += c;
        }
    }
    __syncthreads();
    if (nonempty) {
        const int pos = s.block_cnt[blockIdx.x] + warp_off[threadIdx.x >> 5] + __popc(bal & ((1u << lane) - 1u));
        s.row_list[pos] = (int)r;
    }
}

// Rank (among non-empty rows) of the row holding entry t*W.
__global__ void na_task_rank(const int *__restrict__ row_ptr, int64_t n, int64_t n_tasks, Scratch s) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n_tasks || s.status->code != 0) return;
    const int64_t e = t * kW;
    int64_t lo = 0, hi = n;
    while (lo < hi) {
        const int64_t mid = (lo + hi) >> 1;
        if ((int64_t)row_ptr[mid] <= e) lo = mid + 1; else hi = mid;
    }
    const int64_t r = lo - 1;
    int64_t a = 0, b = *s.n_nonempty;
    while (a < b) {
        const int64_t m = (a + b) >> 1;
        if (s.row_list[m] < r) a = m + 1; else b = m;
    }
    s.task_rank[t] = (int)a;
}

// Warp-stream SpMV over unpadded caller arrays: entry e is read only if e < nnz.
template <typename VT>
__global__ void __launch_bounds__(256) na_stream(const int *__restrict__ col, const VT *__restrict__ val,
                                                 int64_t nnz, int64_t n_tasks, const VT *__restrict__ x,
                                                 VT *__restrict__ y, Scratch s) {
    constexpr int U = 4;
    constexpr int CH = 32 * U;
    constexpr int NC = kW / CH;
    const int lane = threadIdx.x & 31;
    const int64_t t = (int64_t)blockIdx.x * 8 + (threadIdx.x >> 5);
    if (t >= n_tasks || s.status->code != 0) return;  // uniform per warp
    const int n_nonempty = *s.n_nonempty;
    VT *carry_val = static_cast<VT *>(s.carry_val);
    int q = s.task_rank[t];
    VT carry = VT(0);
    int64_t e0 = t * kW + lane * U;
    for (int k = 0; k < NC; ++k, e0 += CH) {
        const unsigned nib = (s.endbits[e0 >> 5] >> (unsigned)(e0 & 31)) & 0xFu;
        VT p[U];
#pragma unroll
        for (int i = 0; i < U; ++i) {
            const int64_t e = e0 + i;
            p[i] = e < nnz ? __ldcs(val + e) * __ldg(x + __ldcs(col + e)) : VT(0);
        }
        const int nend = __popc(nib);
        int incl = nend;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int v = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += v;
        }
        const int excl = incl - nend;
        const int total_ends = __shfl_sync(0xffffffffu, incl, 31);
        VT run = VT(0), head = VT(0);
        int ri = 0;
#pragma unroll
        for (int i = 0; i < U; ++i) {
            run += p[i];
            if ((nib >> i) & 1u) {
                if (ri == 0) head = run;
                else y[s.row_list[q + excl + ri]] = run;
                run = VT(0);
                ++ri;
            }
        }
        VT sv = run;
        int sf = nend > 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const VT vu = __shfl_up_sync(0xffffffffu, sv, o);
            const int fu = __shfl_up_sync(0xffffffffu, sf, o);
            if (lane >= o) {
                if (!sf) sv += vu;
                sf |= fu;
            }
        }
        VT ev = __shfl_up_sync(0xffffffffu, sv, 1);
        int ef = __shfl_up_sync(0xffffffffu, sf, 1);
        if (lane == 0) { ev = VT(0); ef = 0; }
        if (nend) y[s.row_list[q + excl]] = (ef ? ev : carry + ev) + head;
        const VT v31 = __shfl_sync(0xffffffffu, sv, 31);
        const int f31 = __shfl_sync(0xffffffffu, sf, 31);
        carry = f31 ? v31 : carry + v31;
        q += total_ends;
    }
    if (lane == 0) {
        carry_val[t] = carry;
        s.carry_rank[t] = q < n_nonempty ? q : -1;
    }
}

template <typename VT>
__global__ void na_fixup(int64_t n_tasks, VT *__restrict__ y, Scratch s) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n_tasks || s.status->code != 0) return;
    const VT *carry_val = static_cast<const VT *>(s.carry_val);
    const int q = s.carry_rank[t];
    if (q < 0 || (t > 0 && s.carry_rank[t - 1] == q)) return;
    VT acc = VT(0);
    for (int64_t u = t; u < n_tasks && s.carry_rank[u] == q; ++u) acc += carry_val[u];
    y[s.row_list[q]] += acc;
}

}  // namespace
}  // namespace smax

using namespace smax;

extern "C" smax_status smax_spmv_crs_noalloc(int float_type, uint64_t n_rows, uint64_t n_cols, uint64_t nnz,
                                             const void *d_row_ptr, const void *d_col, const void *d_val,
                                             const void *d_x, void *d_y, void *stream) {
    return guarded([&] {
        // size and argument checks come before any CUDA call
        if (float_type != SMAX_FLOAT32 && float_type != SMAX_FLOAT64)
            fail(SMAX_ERR_UNSUPPORTED_TYPE, "value type must be float32 or float64");
        if (n_rows > (uint64_t)kMaxRows || nnz > (uint64_t)kMaxNnz)
            fail(SMAX_ERR_BAD_ARG, "smax_spmv_crs_noalloc: n_rows must be <= " + std::to_string(kMaxRows) +
                                       " and nnz <= " + std::to_string(kMaxNnz) + " (fixed scratch size)");
        if (n_cols >= (1ull << 31)) fail(SMAX_ERR_BAD_ARG, "n_cols exceeds the int32 index range");
        if (!d_row_ptr || (nnz && (!d_col || !d_val || !d_x)) || (n_rows && !d_y))
            fail(SMAX_ERR_BAD_ARG, "null device pointer");
        if (n_rows == 0) return;
        cudaStream_t st = static_cast<cudaStream_t>(stream);
        Scratch s = carve(scratch_for_current_device());
        const int vbytes = float_type == SMAX_FLOAT64 ? 8 : 4;
        const int64_t n = (int64_t)n_rows, z = (int64_t)nnz;
        const int64_t n_tasks = (z + kW - 1) / kW;
        const int n_blocks = (int)((n + kRowsPerBlock - 1) / kRowsPerBlock);
        const int *rp = static_cast<const int *>(d_row_ptr);
        const int *ci = static_cast<const int *>(d_col);

        // clear what must start at zero: the status word and the row-end bits
        SMAX_CUDA(cudaMemsetAsync(s.status, 0, sizeof(DevStatus) + sizeof(int), st));
        SMAX_CUDA(cudaMemsetAsync(s.endbits, 0, sizeof(uint32_t) * ((n_tasks * kW) / 32 + 1), st));
        na_prepare<<<n_blocks, kRowsPerBlock, 0, st>>>(rp, ci, n, z, (int64_t)n_cols, s, d_y, vbytes);
        SMAX_CUDA(cudaGetLastError());
        na_scan_blocks<<<1, 256, 0, st>>>(s, n_blocks);
        SMAX_CUDA(cudaGetLastError());
        na_row_list<<<n_blocks, kRowsPerBlock, 0, st>>>(rp, n, s);
        SMAX_CUDA(cudaGetLastError());
        if (n_tasks > 0) {
            na_task_rank<<<ceil_div_u(n_tasks, 256), 256, 0, st>>>(rp, n, n_tasks, s);
            SMAX_CUDA(cudaGetLastError());
            const unsigned grid = ceil_div_u(n_tasks, 8);
            if (vbytes == 8) {
                na_stream<double><<<grid, 256, 0, st>>>(ci, static_cast<const double *>(d_val), z, n_tasks,
                                                        static_cast<const double *>(d_x),
                                                        static_cast<double *>(d_y), s);
                SMAX_CUDA(cudaGetLastError());
                na_fixup<double><<<ceil_div_u(n_tasks, 256), 256, 0, st>>>(n_tasks, static_cast<double *>(d_y), s);
            } else {
                na_stream<float><<<grid, 256, 0, st>>>(ci, static_cast<const float *>(d_val), z, n_tasks,
                                                       static_cast<const float *>(d_x),
                                                       static_cast<float *>(d_y), s);
                SMAX_CUDA(cudaGetLastError());
                na_fixup<float><<<ceil_div_u(n_tasks, 256), 256, 0, st>>>(n_tasks, static_cast<float *>(d_y), s);
            }
            SMAX_CUDA(cudaGetLastError());
        }
        DevStatus h{};
        SMAX_CUDA(cudaMemcpyAsync(&h, s.status, sizeof(DevStatus), cudaMemcpyDeviceToHost, st));
        SMAX_CUDA(cudaStreamSynchronize(st));
        if (h.code != 0)
            fail(h.code, "malformed CRS matrix (code " + std::to_string(h.code) + " at index " +
                             std::to_string(h.index) + ")");
    });
}
