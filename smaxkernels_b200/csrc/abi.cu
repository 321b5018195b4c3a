// abi.cu -- exported C functions of include/smax_b200.h: contexts, kernel
// objects, registration and the initialize / apply / finalize cycle.
#include <chrono>
#include <cstring>

#include "kernel_obj.cuh"

namespace smax {

namespace {
thread_local std::string g_last_error;

double wall_s() {
    using clk = std::chrono::steady_clock;
    return std::chrono::duration<double>(clk::now().time_since_epoch()).count();
}
}  // namespace

void set_last_error(const std::string &m) { g_last_error = m; }
const char *last_error() { return g_last_error.c_str(); }

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

void DevCRS::upload(const RegCRS &r, int vbytes, cudaStream_t st, int64_t pad) {
    n_rows = (int64_t)r.n_rows;
    n_cols = (int64_t)r.n_cols;
    nnz = (int64_t)r.nnz;
    if (r.n_rows >= (1ull << 31) || r.nnz + (uint64_t)pad >= (1ull << 31))
        fail(SMAX_ERR_UNSUPPORTED, "int32 indices cannot address this matrix");
    const int64_t cap = pad > 1 ? (nnz + pad - 1) / pad * pad : nnz;
    row_ptr.alloc(sizeof(int) * (r.n_rows + 1));
    col.alloc(sizeof(int) * cap);
    val.alloc((size_t)vbytes * cap);
    if (cap > nnz) {
        SMAX_CUDA(cudaMemsetAsync(col.as<int>() + nnz, 0, sizeof(int) * (cap - nnz), st));
        SMAX_CUDA(cudaMemsetAsync(static_cast<char *>(val.p) + (size_t)vbytes * nnz, 0,
                                  (size_t)vbytes * (cap - nnz), st));
    }
    SMAX_CUDA(cudaMemcpyAsync(row_ptr.p, r.row_ptr, sizeof(int) * (r.n_rows + 1), cudaMemcpyHostToDevice, st));
    if (r.nnz) {
        SMAX_CUDA(cudaMemcpyAsync(col.p, r.col, sizeof(int) * r.nnz, cudaMemcpyHostToDevice, st));
        SMAX_CUDA(cudaMemcpyAsync(val.p, r.val, (size_t)vbytes * r.nnz, cudaMemcpyHostToDevice, st));
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

PendingEvents::~PendingEvents() {
    for (auto &p : live) { cudaEventDestroy(p.first); cudaEventDestroy(p.second); }
    for (auto &p : spare) { cudaEventDestroy(p.first); cudaEventDestroy(p.second); }
}

}  // namespace smax

smax_kernel_s::~smax_kernel_s() {
    if (stream) cudaStreamSynchronize(stream);
    if (own_stream) cudaStreamDestroy(own_stream);
}

using namespace smax;

namespace {

void require(bool c, int code, const char *msg) {
    if (!c) fail(code, msg);
}

void read_status(smax_kernel_s *k);

smax_kernel_s *K(smax_kernel k) {
    require(k != nullptr, SMAX_ERR_BAD_ARG, "null kernel handle");
    return k;
}

void read_status(smax_kernel_s *k) {
    if (!k->status.p) return;
    DevStatus st{};
    SMAX_CUDA(cudaMemcpyAsync(&st, k->status.p, sizeof(st), cudaMemcpyDeviceToHost, k->stream));
    SMAX_CUDA(cudaStreamSynchronize(k->stream));
    if (st.code != 0) {
        SMAX_CUDA(cudaMemsetAsync(k->status.p, 0, sizeof(DevStatus), k->stream));
        fail(st.code, "device reported error " + std::to_string(st.code) + " at index " +
                          std::to_string(st.index));
    }
}

// ------------------------------------------------------------------ SpMV --
void spmv_initialize(smax_kernel_s *k) {
    require(k->A.set, SMAX_ERR_STATE, "register_A before initialize");
    require(!k->f_scs && !k->f_bcrs, SMAX_ERR_UNSUPPORTED, "SCS/BCRS SpMV not available in this build");
    if (k->a_dirty) {
        k->dA.upload(k->A, k->vbytes, k->stream, crs_stream_pad());
        validate_crs(k->dA, k->status.as<DevStatus>(), k->stream);
        read_status(k);
        k->crs_plan = CrsTilePlan();
        k->crs_stream = CrsStreamPlan();
        if (k->spmv_variant == 2)
            k->crs_plan.build(k->dA.rp(), k->dA.n_rows, crs_default_cap(k->vbytes * 8), k->stream);
        else
            k->crs_stream.build(k->dA.rp(), k->dA.n_rows, k->dA.nnz, k->vbytes, k->stream);
        k->a_dirty = false;
    }
}

void spmv_apply(smax_kernel_s *k, const void *x, void *y) {
    if (k->spmv_variant != 2) {
        if (k->vbytes == 8)
            crs_spmv_stream<double>(k->crs_stream, k->dA.ci(), k->dA.val.as<double>(),
                                    static_cast<const double *>(x), static_cast<double *>(y), k->stream);
        else
            crs_spmv_stream<float>(k->crs_stream, k->dA.ci(), k->dA.val.as<float>(),
                                   static_cast<const float *>(x), static_cast<float *>(y), k->stream);
        return;
    }
    if (k->vbytes == 8)
        crs_spmv<double>(k->crs_plan, k->dA.rp(), k->dA.ci(), k->dA.val.as<double>(),
                         static_cast<const double *>(x), static_cast<double *>(y), k->stream);
    else
        crs_spmv<float>(k->crs_plan, k->dA.rp(), k->dA.ci(), k->dA.val.as<float>(),
                        static_cast<const float *>(x), static_cast<float *>(y), k->stream);
}

// Device addresses of B and C (+ element offsets).
const void *dev_b(smax_kernel_s *k, uint64_t off) {
    const char *base = k->f_device ? static_cast<const char *>(k->B.val) : static_cast<const char *>(k->dB.p);
    return base + off * k->vbytes;
}
void *dev_c(smax_kernel_s *k, uint64_t off) {
    char *base = k->f_device ? static_cast<char *>(k->C.val) : static_cast<char *>(k->dC.p);
    return base + off * k->vbytes;
}

void do_initialize(smax_kernel_s *k) {
    double t0 = wall_s();
    require(k->B.set && k->C.set, SMAX_ERR_STATE, "register_B and register_C before initialize");
    switch (k->ktype) {
    case SMAX_KERNEL_SPMV: spmv_initialize(k); break;
    default: fail(SMAX_ERR_UNSUPPORTED, "kernel type not available in this build");
    }
    if (!k->f_device) {
        size_t bb = (size_t)k->B.elems() * k->vbytes, cb = (size_t)k->C.elems() * k->vbytes;
        k->dB.ensure(bb);
        k->dC.ensure(cb);
        if (bb) SMAX_CUDA(cudaMemcpyAsync(k->dB.p, k->B.val, bb, cudaMemcpyHostToDevice, k->stream));
    }
    SMAX_CUDA(cudaStreamSynchronize(k->stream));
    k->timers["initialize"] += wall_s() - t0;
}

// Operand extents the kernel reads (B) and writes (C), in elements.
void check_extents(smax_kernel_s *k, uint64_t b_off, uint64_t c_off) {
    uint64_t need_b = 0, need_c = 0;
    switch (k->ktype) {
    case SMAX_KERNEL_SPMV: need_b = k->A.n_cols; need_c = k->A.n_rows; break;
    default: break;
    }
    require(b_off + need_b <= k->B.elems(), SMAX_ERR_BAD_ARG, "B (with offset) is smaller than the operator needs");
    require(c_off + need_c <= k->C.elems(), SMAX_ERR_BAD_ARG, "C (with offset) is smaller than the operator needs");
}

void do_apply(smax_kernel_s *k, uint64_t b_off, uint64_t c_off) {
    require(!k->a_dirty, SMAX_ERR_STATE, "initialize before apply");
    check_extents(k, b_off, c_off);
    auto ev = k->apply_events.acquire();
    SMAX_CUDA(cudaEventRecord(ev.first, k->stream));
    switch (k->ktype) {
    case SMAX_KERNEL_SPMV: spmv_apply(k, dev_b(k, b_off), dev_c(k, c_off)); break;
    default: fail(SMAX_ERR_UNSUPPORTED, "kernel type not available in this build");
    }
    SMAX_CUDA(cudaEventRecord(ev.second, k->stream));
}

void do_finalize(smax_kernel_s *k) {
    double t0 = wall_s();
    if (!k->f_device) {
        size_t cb = (size_t)k->C.elems() * k->vbytes;
        if (cb) SMAX_CUDA(cudaMemcpyAsync(k->C.val, k->dC.p, cb, cudaMemcpyDeviceToHost, k->stream));
    }
    SMAX_CUDA(cudaStreamSynchronize(k->stream));
    read_status(k);
    k->timers["apply"] += k->apply_events.drain();
    k->timers["finalize"] += wall_s() - t0;
}

}  // namespace

extern "C" {

int smax_abi_version(void) { return SMAX_B200_ABI_VERSION; }

const char *smax_last_error(void) { return smax::last_error(); }

smax_status smax_ctx_create(smax_ctx *out) {
    return guarded([&] {
        require(out != nullptr, SMAX_ERR_BAD_ARG, "null output");
        *out = new smax_ctx_s();
    });
}

smax_status smax_ctx_destroy(smax_ctx ctx) {
    return guarded([&] { delete ctx; });
}

int smax_ctx_get_n_levels(smax_ctx ctx) { return ctx ? ctx->n_levels : 0; }

int smax_ctx_get_level_ptr_at(smax_ctx ctx, int idx) {
    if (!ctx || idx < 0 || idx >= (int)ctx->lvl_ptr.size()) return -1;
    return ctx->lvl_ptr[idx];
}

smax_status smax_kernel_create(smax_kernel *out, smax_ctx ctx, int kernel_type, int int_type, int float_type) {
    return guarded([&] {
        require(out != nullptr, SMAX_ERR_BAD_ARG, "null output");
        require(kernel_type >= SMAX_KERNEL_SPMV && kernel_type <= SMAX_KERNEL_SPTRSM, SMAX_ERR_BAD_ARG,
                "unknown kernel type");
        require(int_type == SMAX_INT32, SMAX_ERR_UNSUPPORTED_TYPE, "only int32 indices are supported");
        require(float_type == SMAX_FLOAT32 || float_type == SMAX_FLOAT64, SMAX_ERR_UNSUPPORTED_TYPE,
                "value type must be float32 or float64");
        auto *k = new smax_kernel_s();
        k->ctx = ctx;
        k->ktype = kernel_type;
        k->itype = int_type;
        k->ftype = float_type;
        k->vbytes = float_type == SMAX_FLOAT64 ? 8 : 4;
        cudaError_t e = cudaStreamCreateWithFlags(&k->own_stream, cudaStreamNonBlocking);
        if (e != cudaSuccess) {
            k->own_stream = nullptr;
            delete k;
            cuda_check(e, "cudaStreamCreateWithFlags");
        }
        k->stream = k->own_stream;
        k->status.alloc(sizeof(DevStatus));
        SMAX_CUDA(cudaMemsetAsync(k->status.p, 0, sizeof(DevStatus), k->stream));
        *out = k;
    });
}

smax_status smax_kernel_destroy(smax_kernel k) {
    return guarded([&] { delete k; });
}

smax_status smax_kernel_set_flag(smax_kernel k, int flag, int value) {
    return guarded([&] {
        smax_kernel_s *kk = K(k);
        bool v = value != 0;
        switch (flag) {
        case SMAX_FLAG_MAT_PERM: kk->f_perm = v; break;
        case SMAX_FLAG_MAT_UPPER_TRIANG: kk->f_upper = v; break;
        case SMAX_FLAG_MAT_LOWER_TRIANG: kk->f_lower = v; break;
        case SMAX_FLAG_VEC_ROW_MAJOR: kk->f_row_major = v; break;
        case SMAX_FLAG_MAT_SCS: kk->f_scs = v; break;
        case SMAX_FLAG_MAT_BCRS: kk->f_bcrs = v; break;
        case SMAX_FLAG_BLOCK_COLUMN_MAJOR: kk->f_block_col_major = v; break;
        case SMAX_FLAG_KERNEL_IMPL: kk->impl = value; break;
        case SMAX_FLAG_DEVICE_POINTERS: kk->f_device = v; break;
        case SMAX_FLAG_A_DIRTY: kk->a_dirty = kk->a_dirty || v; break;
        case SMAX_FLAG_SPMV_VARIANT:
            require(value >= 0 && value <= 2, SMAX_ERR_BAD_ARG, "SpMV variant must be 0, 1 or 2");
            if (value != kk->spmv_variant) kk->a_dirty = true;  // plans differ per variant
            kk->spmv_variant = value;
            break;
        default: fail(SMAX_ERR_BAD_ARG, "unknown flag");
        }
    });
}

smax_status smax_kernel_register_A_crs(smax_kernel k, uint64_t n_rows, uint64_t n_cols, uint64_t nnz, void *col,
                                       void *row_ptr, void *val) {
    return guarded([&] {
        smax_kernel_s *kk = K(k);
        require(row_ptr != nullptr, SMAX_ERR_BAD_ARG, "null row_ptr");
        require(nnz == 0 || (col && val), SMAX_ERR_BAD_ARG, "null col/val");
        kk->A = RegCRS{true, n_rows, n_cols, nnz, col, row_ptr, val};
        kk->a_dirty = true;
    });
}

smax_status smax_kernel_register_dense(smax_kernel k, int slot, uint64_t n_rows, uint64_t n_cols, void *val) {
    return guarded([&] {
        smax_kernel_s *kk = K(k);
        require(slot == 1 || slot == 2, SMAX_ERR_BAD_ARG, "slot must be 1 (B) or 2 (C)");
        require(val != nullptr || n_rows == 0, SMAX_ERR_BAD_ARG, "null dense operand");
        RegDense d{true, n_rows, n_cols, val};
        if (slot == 1) kk->B = d; else kk->C = d;
    });
}

smax_status smax_kernel_initialize(smax_kernel k, uint64_t, uint64_t, uint64_t) {
    return guarded([&] { do_initialize(K(k)); });
}

smax_status smax_kernel_apply(smax_kernel k, uint64_t, uint64_t B_offset, uint64_t C_offset) {
    return guarded([&] { do_apply(K(k), B_offset, C_offset); });
}

smax_status smax_kernel_finalize(smax_kernel k, uint64_t, uint64_t, uint64_t) {
    return guarded([&] { do_finalize(K(k)); });
}

smax_status smax_kernel_run(smax_kernel k, uint64_t A_offset, uint64_t B_offset, uint64_t C_offset) {
    (void)A_offset;
    return guarded([&] {
        smax_kernel_s *kk = K(k);
        do_initialize(kk);
        do_apply(kk, B_offset, C_offset);
        do_finalize(kk);
    });
}

smax_status smax_kernel_sync(smax_kernel k) {
    return guarded([&] {
        smax_kernel_s *kk = K(k);
        SMAX_CUDA(cudaStreamSynchronize(kk->stream));
        read_status(kk);
        kk->timers["apply"] += kk->apply_events.drain();
    });
}

smax_status smax_kernel_get_timer(smax_kernel k, const char *name, double *seconds) {
    return guarded([&] {
        smax_kernel_s *kk = K(k);
        require(name && seconds, SMAX_ERR_BAD_ARG, "null argument");
        if (!kk->apply_events.live.empty()) kk->timers["apply"] += kk->apply_events.drain();
        auto it = kk->timers.find(name);
        *seconds = it == kk->timers.end() ? 0.0 : it->second;
    });
}

void *smax_kernel_stream(smax_kernel k) { return k ? (void *)k->stream : nullptr; }

smax_status smax_kernel_set_stream(smax_kernel k, void *stream) {
    return guarded([&] {
        smax_kernel_s *kk = K(k);
        cudaStream_t next = stream ? static_cast<cudaStream_t>(stream) : kk->own_stream;
        if (next != kk->stream) {
            // work queued so far stays ordered before work on the new stream
            SMAX_CUDA(cudaStreamSynchronize(kk->stream));
            kk->stream = next;
        }
    });
}

}  // extern "C"
