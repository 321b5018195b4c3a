// runtime.cu -- shared host-side runtime of the platform: error capture, device
// queries, CUDA-event stopwatches, uploads and the validation passes that run
// once per registered matrix before any kernel trusts it.
#include <atomic>
#include <chrono>

#include "kernel_obj.cuh"

namespace smax {

namespace {
thread_local std::string g_last_error;
}  // namespace

void set_last_error(const std::string &m) { g_last_error = m; }
const char *last_error() { return g_last_error.c_str(); }

namespace {
std::atomic<long long> g_alloc_count{0};    // device allocations attempted since load
std::atomic<long long> g_alloc_fail_at{0};  // armed: g_alloc_count value that fails; 0 = off
}  // namespace

bool device_alloc_should_fail() {
    const long long k = ++g_alloc_count;
    long long at = g_alloc_fail_at.load();
    return at != 0 && k == at && g_alloc_fail_at.compare_exchange_strong(at, 0);
}

void arm_device_alloc_failure(long long n) { g_alloc_fail_at = n > 0 ? g_alloc_count.load() + n : 0; }
long long device_alloc_count() { return g_alloc_count.load(); }

double wall_s() {
    using clk = std::chrono::steady_clock;
    return std::chrono::duration<double>(clk::now().time_since_epoch()).count();
}

int sm_count() {
    static int cached[64] = {0};
    int dev = 0;
    SMAX_CUDA(cudaGetDevice(&dev));
    if (dev < 64 && cached[dev]) return cached[dev];
    int n = 0;
    SMAX_CUDA(cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev));
    if (dev < 64) cached[dev] = n;
    return n;
}

int64_t l2_bytes() {
    static int cached[64] = {0};
    int dev = 0;
    SMAX_CUDA(cudaGetDevice(&dev));
    if (dev < 64 && cached[dev]) return cached[dev];
    int n = 0;
    SMAX_CUDA(cudaDeviceGetAttribute(&n, cudaDevAttrL2CacheSize, dev));
    if (dev < 64) cached[dev] = n;
    return n;
}

namespace {
// One pass over an uploaded CRS matrix: row_ptr[0] == 0, row_ptr[n] == nnz,
// row_ptr non-decreasing, every column in [0, n_cols).  Hot kernels trust the
// matrix afterwards, so malformed input becomes an error status here instead
// of an out-of-bounds access later.
__global__ void validate_crs_kernel(const int *__restrict__ row_ptr, const int *__restrict__ col, int64_t n,
                                    int64_t nnz, int64_t n_cols, DevStatus *st) {
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t == 0 && (row_ptr[0] != 0 || row_ptr[n] != nnz)) report(st, SMAX_ERR_BAD_ARG, 0);
    for (int64_t r = t; r < n; r += stride)
        if (row_ptr[r + 1] < row_ptr[r]) report(st, SMAX_ERR_BAD_ARG, r);
    for (int64_t j = t; j < nnz; j += stride) {
        int c = col[j];
        if (c < 0 || c >= n_cols) report(st, SMAX_ERR_COL_OOB, j);
    }
}
}  // namespace

void validate_crs(const DevCRS &m, DevStatus *st, cudaStream_t s) {
    int blocks = 4 * sm_count();
    validate_crs_kernel<<<blocks, 256, 0, s>>>(m.rp(), m.ci(), m.n_rows, m.nnz, m.n_cols, st);
    SMAX_CUDA(cudaGetLastError());
}

void upload_crs(DevCRS &d, const RegCRS &r, int vbytes, cudaStream_t st, int64_t pad) {
    d.n_rows = (int64_t)r.n_rows;
    d.n_cols = (int64_t)r.n_cols;
    d.nnz = (int64_t)r.nnz;
    if (r.n_rows >= (1ull << 31) || r.nnz + (uint64_t)pad >= (1ull << 31) || r.n_cols >= (1ull << 31))
        fail(SMAX_ERR_UNSUPPORTED, "int32 indices cannot address this matrix");
    // one spare slice: a row block's last slice may start mid-array and read up
    // to one slice past its end (the pipelined SpMV), always inside the buffer
    const int64_t cap = pad > 1 ? (d.nnz + pad - 1) / pad * pad + pad : d.nnz;
    d.row_ptr.alloc(sizeof(int) * (r.n_rows + 1));
    d.col.alloc(sizeof(int) * cap);
    d.val.alloc((size_t)vbytes * cap);
    if (cap > d.nnz) {
        SMAX_CUDA(cudaMemsetAsync(d.col.as<int>() + d.nnz, 0, sizeof(int) * (cap - d.nnz), st));
        SMAX_CUDA(cudaMemsetAsync(static_cast<char *>(d.val.p) + (size_t)vbytes * d.nnz, 0,
                                  (size_t)vbytes * (cap - d.nnz), st));
    }
    // the registered arrays may be host or device memory: the copy direction
    // follows from the addresses (unified addressing)
    SMAX_CUDA(cudaMemcpyAsync(d.row_ptr.p, r.row_ptr, sizeof(int) * (r.n_rows + 1), cudaMemcpyDefault, st));
    if (r.nnz) {
        SMAX_CUDA(cudaMemcpyAsync(d.col.p, r.col, sizeof(int) * r.nnz, cudaMemcpyDefault, st));
        // a pattern-only upload (val == nullptr) leaves the values unset
        if (r.val) SMAX_CUDA(cudaMemcpyAsync(d.val.p, r.val, (size_t)vbytes * r.nnz, cudaMemcpyDefault, st));
    }
}

std::pair<cudaEvent_t, cudaEvent_t> PendingEvents::acquire() {
    std::pair<cudaEvent_t, cudaEvent_t> p;
    if (!spare.empty()) {
        p = spare.back();
        spare.pop_back();
    } else {
        SMAX_CUDA(cudaEventCreate(&p.first));
        SMAX_CUDA(cudaEventCreate(&p.second));
    }
    live.push_back(p);
    return p;
}

double PendingEvents::trim(size_t keep) {
    if (live.size() <= 2 * keep) return 0.0;
    // the oldest intervals finished long ago in any pipelined loop
    const size_t n = live.size() - keep;
    double s = 0.0;
    for (size_t i = 0; i < n; ++i) {
        auto &p = live[i];
        SMAX_CUDA(cudaEventSynchronize(p.second));
        float ms = 0.f;
        SMAX_CUDA(cudaEventElapsedTime(&ms, p.first, p.second));
        s += ms * 1e-3;
        spare.push_back(p);
    }
    live.erase(live.begin(), live.begin() + (ptrdiff_t)n);
    return s;
}

double PendingEvents::drain() {
    double s = 0.0;
    for (auto &p : live) {
        SMAX_CUDA(cudaEventSynchronize(p.second));
        float ms = 0.f;
        SMAX_CUDA(cudaEventElapsedTime(&ms, p.first, p.second));
        s += ms * 1e-3;
        spare.push_back(p);
    }
    live.clear();
    return s;
}

void PendingEvents::drop(std::pair<cudaEvent_t, cudaEvent_t> p) {
    for (size_t i = live.size(); i-- > 0;)
        if (live[i] == p) {
            live.erase(live.begin() + (ptrdiff_t)i);
            spare.push_back(p);
            return;
        }
}

PendingEvents::~PendingEvents() {
    for (auto &p : live) { cudaEventDestroy(p.first); cudaEventDestroy(p.second); }
    for (auto &p : spare) { cudaEventDestroy(p.first); cudaEventDestroy(p.second); }
}

}  // namespace smax
