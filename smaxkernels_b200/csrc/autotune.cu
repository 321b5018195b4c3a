// autotune.cu -- smax_kernel_autotune and smax_utils_tune_spmv_format.
//
// No counterpart in the reference, where the user picks the format and the
// kernel.  Both tuners time candidates with CUDA events on the stream the
// work runs on (two warm-up calls, then the mean of five) and keep the
// fastest.  Kernel-level choices are cached for the life of the process per
// matrix, keyed by kernel type, value type, layout flags, sizes and an FNV-1a
// hash of row_ptr plus 4096 evenly spaced column indices.
#include <cstring>
#include <functional>
#include <map>
#include <mutex>
#include <tuple>
#include <vector>

#include "abi_internal.cuh"

using namespace smax;

namespace {

using Key = std::tuple<int, int, int, int, int, int, int, uint64_t, uint64_t, uint64_t, uint64_t, uint64_t>;

std::mutex g_mu;
std::map<Key, smax_tuning> g_cache;

constexpr int kWarm = 2, kReps = 5;

uint64_t fnv1a(uint64_t h, const void *p, size_t n) {
    const unsigned char *b = static_cast<const unsigned char *>(p);
    for (size_t i = 0; i < n; ++i) {
        h ^= b[i];
        h *= 1099511628211ull;
    }
    return h;
}

uint64_t pattern_hash(const RegCRS &A) {
    uint64_t h = 1469598103934665603ull;
    if (A.row_ptr) h = fnv1a(h, A.row_ptr, sizeof(int) * (A.n_rows + 1));
    if (A.col && A.nnz) {
        const int *c = static_cast<const int *>(A.col);
        for (uint64_t i = 0; i < 4096; ++i) {
            const uint64_t j = (A.nnz - 1) * i / 4095;
            h = fnv1a(h, c + j, sizeof(int));
        }
    }
    return h;
}

Key key_of(const smax_kernel_s *k) {
    return Key{k->ktype, k->vbytes, (int)k->f_scs, (int)k->f_bcrs, (int)k->f_perm, (int)k->f_upper,
               (int)k->f_row_major + 2 * (k->refine_steps > 0), k->A.n_rows, k->A.n_cols, k->A.nnz,
               k->B.n_cols, pattern_hash(k->A)};
}

// mean seconds of one call after kWarm warm-up calls
double time_calls(cudaStream_t st, const std::function<void()> &f) {
    for (int i = 0; i < kWarm; ++i) f();
    SMAX_CUDA(cudaStreamSynchronize(st));
    cudaEvent_t a, b;
    SMAX_CUDA(cudaEventCreate(&a));
    SMAX_CUDA(cudaEventCreate(&b));
    struct Free {
        cudaEvent_t a, b;
        ~Free() {
            cudaEventDestroy(a);
            cudaEventDestroy(b);
        }
    } fr{a, b};
    SMAX_CUDA(cudaEventRecord(a, st));
    for (int i = 0; i < kReps; ++i) f();
    SMAX_CUDA(cudaEventRecord(b, st));
    SMAX_CUDA(cudaEventSynchronize(b));
    float ms = 0.f;
    SMAX_CUDA(cudaEventElapsedTime(&ms, a, b));
    return ms * 1e-3 / kReps;
}

double time_apply(smax_kernel_s *k) {
    const double t = time_calls(k->stream, [&] { apply_core(k, 0, 0); });
    read_status(k);
    return t;
}

void tune_kernel(smax_kernel_s *k, smax_tuning &r) {
    r.spmv_variant = k->spmv_variant;
    r.solve_mode = k->solve_mode;
    r.level_merge = k->level_merge;
    r.sweep_cluster = k->sweep_cluster;
    double best = 1e300;
    if (k->ktype == SMAX_KERNEL_SPMV && !k->f_scs && !k->f_bcrs) {
        build_crs_plans(k);
        for (int v : {1, 2}) {
            k->spmv_variant = v;
            const double t = time_apply(k);
            ++r.n_candidates;
            if (t < best) { best = t; r.spmv_variant = v; }
        }
        k->spmv_variant = r.spmv_variant;
    } else if (k->ktype == SMAX_KERNEL_SPMM && k->f_row_major) {
        // row-major SpMM: all-rows grid (1) or per-SM row walks (2)
        for (int v : {1, 2}) {
            k->spmv_variant = v;
            const double t = time_apply(k);
            ++r.n_candidates;
            if (t < best) { best = t; r.spmv_variant = v; }
        }
        k->spmv_variant = r.spmv_variant;
    } else if (is_tri(k)) {
        struct Cand { int mode, merge; bool cluster; };
        std::vector<Cand> cands;
        for (int m : {0, 1024, 4096, 16384, 65536}) cands.push_back({SMAX_SOLVE_GRAPH, m, false});
        const bool one_rhs = k->ktype == SMAX_KERNEL_SPTRSV || (k->B.n_cols <= 1);
        if (k->ktype == SMAX_KERNEL_SPTRSV) {
            cands.push_back({SMAX_SOLVE_GRAPH, 4096, true});
            cands.push_back({SMAX_SOLVE_GRAPH, 16384, true});
        }
        if (k->ktype == SMAX_KERNEL_SPTRSV && one_rhs && k->refine_steps == 0) {
            cands.push_back({SMAX_SOLVE_PERSISTENT, 0, false});
            cands.push_back({SMAX_SOLVE_SYNCFREE, 0, false});
        }
        if (k->ktype == SMAX_KERNEL_SPTRSM) cands.push_back({SMAX_SOLVE_SYNCFREE, 0, false});
        for (const Cand &c : cands) {
            k->solve_mode = c.mode;
            k->level_merge = c.merge;
            k->sweep_cluster = c.cluster;
            double t;
            try {
                t = time_apply(k);
            } catch (const Error &e) {
                // a persistent or sync-free solve whose wait timed out is not a candidate
                if (e.code != SMAX_ERR_TIMEOUT) throw;
                continue;
            }
            ++r.n_candidates;
            if (t < best) { best = t; r.solve_mode = c.mode; r.level_merge = c.merge; r.sweep_cluster = c.cluster; }
        }
        k->solve_mode = r.solve_mode;
        k->level_merge = r.level_merge;
        k->sweep_cluster = r.sweep_cluster != 0;
    } else {
        best = time_apply(k);
        r.n_candidates = 1;
    }
    r.seconds = best;
}

void apply_choice(smax_kernel_s *k, const smax_tuning &t) {
    if (k->ktype == SMAX_KERNEL_SPMV && !k->f_scs && !k->f_bcrs) {
        if (t.spmv_variant != k->spmv_variant) build_crs_plans(k);
        k->spmv_variant = t.spmv_variant;
    } else if (k->ktype == SMAX_KERNEL_SPMM && k->f_row_major) {
        k->spmv_variant = t.spmv_variant;
    } else if (is_tri(k)) {
        k->solve_mode = t.solve_mode;
        k->level_merge = t.level_merge;
        k->sweep_cluster = t.sweep_cluster != 0;
    }
}

__global__ void fill_kernel(double *x, int64_t n) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
        x[i] = 1.0 / (double)(1 + (i & 1023));
}
__global__ void fill_kernel(float *x, int64_t n) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
        x[i] = 1.0f / (float)(1 + (i & 1023));
}

struct OwnStream {
    cudaStream_t s = nullptr;
    OwnStream() { cuda_check(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking), "cudaStreamCreateWithFlags"); }
    ~OwnStream() {
        cudaStreamSynchronize(s);
        cudaStreamDestroy(s);
    }
};

template <typename VT>
void tune_format(const RegCRS &r, smax_format_choice &out) {
    const int vbytes = sizeof(VT);
    OwnStream os;
    cudaStream_t st = os.s;
    DevCRS a;
    upload_crs(a, r, vbytes, st, crs_stream_pad());
    DevBuf status(sizeof(DevStatus));
    SMAX_CUDA(cudaMemsetAsync(status.p, 0, sizeof(DevStatus), st));
    validate_crs(a, status.as<DevStatus>(), st);
    DevStatus hs{};
    SMAX_CUDA(cudaMemcpyAsync(&hs, status.p, sizeof(hs), cudaMemcpyDeviceToHost, st));
    SMAX_CUDA(cudaStreamSynchronize(st));
    if (hs.code) fail(hs.code, "invalid CRS matrix at index " + std::to_string(hs.index));

    const int64_t n = a.n_rows, m = a.n_cols, nnz = a.nnz;
    DevBuf x(sizeof(VT) * (m > 0 ? m : 1)), y(sizeof(VT) * (n + 64));
    fill_kernel<<<256, 256, 0, st>>>(x.as<VT>(), m);
    SMAX_CUDA(cudaGetLastError());
    const VT *xp = x.as<VT>();
    VT *yp = y.as<VT>();
    double best = 1e300;
    auto consider = [&](double t, int fmt, int var, int C, int sg, int bh) {
        ++out.n_candidates;
        if (fmt == 0 && t < out.crs_seconds) out.crs_seconds = t;
        if (t < best) {
            best = t;
            out.format = fmt;
            out.spmv_variant = var;
            out.C = C;
            out.sigma = sg;
            out.b_height = out.b_width = bh;
        }
    };
    out.crs_seconds = 1e300;
    {
        CrsStreamPlan p;
        p.build(a.rp(), n, nnz, vbytes, st);
        consider(time_calls(st, [&] { crs_spmv_stream<VT>(p, a.ci(), a.val.as<VT>(), xp, yp, st); }), 0, 1, 0, 0, 0);
    }
    {
        CrsTilePlan p;
        p.build(a.rp(), n, crs_default_cap(vbytes * 8), st);
        consider(time_calls(st, [&] { crs_spmv<VT>(p, a.rp(), a.ci(), a.val.as<VT>(), xp, yp, st); }), 0, 2, 0, 0,
                 0);
    }
    for (int C : {8, 16, 32, 64}) {
        std::vector<int> sigmas{1, 8 * C, 1024};
        for (size_t i = 0; i < sigmas.size(); ++i) {
            const int sg = sigmas[i];
            bool dup = false;
            for (size_t j = 0; j < i; ++j) dup = dup || sigmas[j] == sg;
            if (dup) continue;
            DevSCS s;
            DevBuf perm;
            crs_to_scs(a, vbytes, C, sg, s, perm, st);
            scs_plan(s, vbytes, st);
            if (s.n_rows_padded > n + 64) {
                // one more padded chunk than y holds: grow y
                y.alloc(sizeof(VT) * s.n_rows_padded);
                yp = y.as<VT>();
            }
            consider(time_calls(st, [&] { scs_spmv<VT>(s, xp, yp, st); }), 1, 0, C, sg, 0);
        }
    }
    for (int b : {2, 4}) {
        if (n == 0 || n % b || m % b) continue;
        DevBCRS bm;
        crs_to_bcrs(a, vbytes, b, b, b, b, false, bm, st, 2 * nnz / (b * b));
        if (!bm.val.p) continue;  // fill above twice the nonzeros
        consider(time_calls(st, [&] { bcrs_spmv<VT>(bm, xp, yp, st); }), 2, 0, 0, 0, b);
    }
    out.seconds = best;
}

}  // namespace

extern "C" {

smax_status smax_kernel_autotune(smax_kernel k, smax_tuning *out) {
    return guarded([&] {
        smax_kernel_s *kk = K(k);
        require(kk->ktype != SMAX_KERNEL_SPGEMM, SMAX_ERR_UNSUPPORTED, "SpGEMM has no launch variants to tune");
        require(!kk->a_dirty, SMAX_ERR_STATE, "initialize before autotune");
        smax_tuning r{};
        const Key key = key_of(kk);
        bool hit = false;
        {
            std::lock_guard<std::mutex> lk(g_mu);
            auto it = g_cache.find(key);
            if (it != g_cache.end()) {
                r = it->second;
                hit = true;
            }
        }
        if (hit) {
            apply_choice(kk, r);
            r.from_cache = 1;
            r.n_candidates = 0;
        } else {
            if (is_tri(kk)) tri_plan(kk);
            tune_kernel(kk, r);
            r.from_cache = 0;
            std::lock_guard<std::mutex> lk(g_mu);
            g_cache[key] = r;
        }
        if (out) *out = r;
    });
}

smax_status smax_utils_tune_spmv_format(int float_type, uint64_t n_rows, uint64_t n_cols, uint64_t nnz,
                                        const void *row_ptr, const void *col, const void *val,
                                        smax_format_choice *out) {
    return guarded([&] {
        require(float_type == SMAX_FLOAT32 || float_type == SMAX_FLOAT64, SMAX_ERR_UNSUPPORTED_TYPE,
                "value type must be float32 or float64");
        require(row_ptr != nullptr && (nnz == 0 || (col && val)), SMAX_ERR_BAD_ARG, "null CRS array");
        require(out != nullptr, SMAX_ERR_BAD_ARG, "null output");
        RegCRS r{true, n_rows, n_cols, nnz, const_cast<void *>(col), const_cast<void *>(row_ptr),
                 const_cast<void *>(val)};
        smax_format_choice c{};
        if (float_type == SMAX_FLOAT64) tune_format<double>(r, c);
        else tune_format<float>(r, c);
        *out = c;
    });
}

}  // extern "C"
