// refine.cu -- FP32 triangular solve with FP64 iterative refinement.
//
// No counterpart in the reference (which solves in the registered precision
// only).  For a float64 SpTRSV kernel with SMAX_FLAG_REFINE = s:
//   x   = (double) solve32(L32, (float) b)
//   s times:  r = b - L x           (FP64 values and arithmetic, one pass)
//             d = solve32(L32, (float) r)
//             x = x + (double) d
// L32 and D32 are float copies of the device matrix (made once per value
// upload).  The FP32 solves run on the same level schedule as the FP64 solve.
// Each correction multiplies the error by about u32 * cond(L), so for the
// well-conditioned triangles of the solve configurations two corrections
// reach the FP64 result to ~1e-15.  With SMAX_FLAG_REFINE_TOL = t the host
// stops after the first correction with max|d| <= 10^-t max|x|; otherwise the
// whole sequence is one CUDA graph (captured on first use) and never syncs.
#include <cmath>
#include <cstring>

#include "abi_internal.cuh"

namespace smax {

namespace {

unsigned grid_of(int64_t n) {
    const int64_t cap = (int64_t)sm_count() * 8;
    int64_t g = (n + 255) / 256;
    return (unsigned)(g < 1 ? 1 : (g > cap ? cap : g));
}

__global__ void cast_to_float(const double *__restrict__ a, int64_t n, float *__restrict__ b) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) b[i] = (float)a[i];
}

__global__ void cast_diag(const double *__restrict__ D, int64_t n, float *__restrict__ D32, DevStatus *st) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const float d = (float)D[i];
        if (d == 0.f || !isfinite(d)) report(st, SMAX_ERR_ZERO_DIAG, i);
        D32[i] = d;
    }
}

// r = (float)(b - A x), the full row including the diagonal
__global__ void residual_kernel(const int *__restrict__ rp, const int *__restrict__ ci,
                                const double *__restrict__ val, const double *__restrict__ b,
                                const double *__restrict__ x, int64_t n, float *__restrict__ r) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        double s = b[i];
        const int e = rp[i + 1];
        for (int j = rp[i]; j < e; ++j) s -= val[j] * x[ci[j]];
        r[i] = (float)s;
    }
}

// max of non-negative doubles through their (order-preserving) bit patterns
__device__ __forceinline__ void block_max2(double a, double b, unsigned long long *stats) {
    for (int o = 16; o > 0; o >>= 1) {
        a = fmax(a, __shfl_xor_sync(0xffffffffu, a, o));
        b = fmax(b, __shfl_xor_sync(0xffffffffu, b, o));
    }
    if ((threadIdx.x & 31) == 0) {
        if (a > 0) atomicMax(stats, (unsigned long long)__double_as_longlong(a));
        if (b > 0) atomicMax(stats + 1, (unsigned long long)__double_as_longlong(b));
    }
}

// x = (double) x32 (first = true) or x += (double) d32; stats = max|d|, max|x|
__global__ void update_x(const float *__restrict__ d32, int64_t n, bool first, double *__restrict__ x,
                         unsigned long long *stats) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    double md = 0.0, mx = 0.0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const double d = (double)d32[i];
        const double v = first ? d : x[i] + d;
        x[i] = v;
        md = fmax(md, fabs(d));
        mx = fmax(mx, fabs(v));
    }
    block_max2(md, mx, stats);
}

void ensure_copies(smax_kernel_s *k) {
    RefineState &R = k->refine;
    if (R.vals_version == k->vals_version) return;
    const int64_t n = k->dA.n_rows, nnz = k->dA.nnz;
    cudaStream_t st = k->stream;
    R.val32.ensure(sizeof(float) * (nnz > 0 ? nnz : 1));
    R.D32.ensure(sizeof(float) * (n > 0 ? n : 1));
    R.b32.ensure(sizeof(float) * (n > 0 ? n : 1));
    R.x32.ensure(sizeof(float) * (n > 0 ? n : 1));
    R.r32.ensure(sizeof(float) * (n > 0 ? n : 1));
    R.stats.ensure(2 * sizeof(unsigned long long));
    if (nnz) cast_to_float<<<grid_of(nnz), 256, 0, st>>>(k->dA.val.as<double>(), nnz, R.val32.as<float>());
    if (n) cast_diag<<<grid_of(n), 256, 0, st>>>(k->D.as<double>(), n, R.D32.as<float>(), dstatus(k));
    SMAX_CUDA(cudaGetLastError());
    read_status(k);
    R.vals_version = k->vals_version;
}

double bits_to_double(unsigned long long u) {
    double d;
    std::memcpy(&d, &u, sizeof d);
    return d;
}

double read_rel(smax_kernel_s *k, cudaStream_t st) {
    unsigned long long h[2] = {0, 0};
    SMAX_CUDA(cudaMemcpyAsync(h, k->refine.stats.p, sizeof(h), cudaMemcpyDeviceToHost, st));
    SMAX_CUDA(cudaStreamSynchronize(st));
    const double md = bits_to_double(h[0]), mx = bits_to_double(h[1]);
    return mx > 0 ? md / mx : (md > 0 ? INFINITY : 0.0);
}

// The initial FP32 solve (when `initial`) and `steps` corrections.
void sequence(smax_kernel_s *k, const double *B, double *X, bool initial, int steps, cudaStream_t st) {
    RefineState &R = k->refine;
    const int64_t n = k->dA.n_rows;
    const int merge = tri_merge_rows(k);
    const int *rp = k->dA.rp(), *ci = k->dA.ci();
    const float *v32 = R.val32.as<float>(), *D32 = R.D32.as<float>();
    float *b32 = R.b32.as<float>(), *x32 = R.x32.as<float>(), *r32 = R.r32.as<float>();
    auto *stats = R.stats.as<unsigned long long>();
    if (initial) {
        cast_to_float<<<grid_of(n), 256, 0, st>>>(B, n, b32);
        tri_solve_raw<float>(k->tri, rp, ci, v32, D32, b32, x32, 1, true, n, merge, k->vals_version, st);
        SMAX_CUDA(cudaMemsetAsync(stats, 0, 2 * sizeof(unsigned long long), st));
        update_x<<<grid_of(n), 256, 0, st>>>(x32, n, true, X, stats);
    }
    for (int s = 0; s < steps; ++s) {
        residual_kernel<<<grid_of(n), 256, 0, st>>>(rp, ci, k->dA.val.as<double>(), B, X, n, r32);
        tri_solve_raw<float>(k->tri, rp, ci, v32, D32, r32, x32, 1, true, n, merge, k->vals_version, st);
        SMAX_CUDA(cudaMemsetAsync(stats, 0, 2 * sizeof(unsigned long long), st));
        update_x<<<grid_of(n), 256, 0, st>>>(x32, n, false, X, stats);
    }
    SMAX_CUDA(cudaGetLastError());
}

}  // namespace

void refine_solve(smax_kernel_s *k, const double *B, double *X) {
    RefineState &R = k->refine;
    const int64_t n = k->dA.n_rows;
    if (n == 0) return;
    ensure_copies(k);
    const int merge = tri_merge_rows(k);
    const int steps = k->refine_steps;
    k->tri.ensure_pack(k->dA.rp(), k->dA.ci(), R.val32.p, R.D32.p, sizeof(float), merge, k->vals_version, k->stream);
    k->tri.prepare(1, merge, k->stream);
    if (k->refine_tol > 0) {
        // host-checked: stop at the first correction below the tolerance
        const double tol = std::pow(10.0, -(double)k->refine_tol);
        sequence(k, B, X, true, 0, k->stream);
        R.steps_done = 0;
        R.last_rel = 0.0;
        for (int s = 0; s < steps; ++s) {
            sequence(k, B, X, false, 1, k->stream);
            R.steps_done = s + 1;
            R.last_rel = read_rel(k, k->stream);
            if (R.last_rel <= tol) break;
        }
        return;
    }
    if (k->solve_mode != SMAX_SOLVE_AUTO && k->solve_mode != SMAX_SOLVE_GRAPH) {
        sequence(k, B, X, true, steps, k->stream);
        R.steps_done = steps;
        R.last_rel = -1.0;  // read lazily by get_refine_stats
        return;
    }
    const bool fenced = !is_capturable(k->stream);
    cudaStream_t st = fenced ? R.aux.enter(k->stream) : k->stream;
    const void *key0 = B, *key1 = X;
    const bool stale = !R.graph || R.gkey[0] != key0 || R.gkey[1] != key1 || R.g_steps != steps ||
                       R.g_merge != merge || R.g_serial != k->tri_plan_serial || R.g_aver != k->a_version ||
                       R.g_pack != k->tri.pack.psrc.p;
    if (stale) {
        R.release_graph();
        SMAX_CUDA(cudaStreamSynchronize(st));
        cudaGraph_t g = nullptr;
        SMAX_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
        try {
            sequence(k, B, X, true, steps, st);
        } catch (...) {
            cudaStreamEndCapture(st, &g);
            if (g) cudaGraphDestroy(g);
            if (fenced) R.aux.leave(k->stream);
            throw;
        }
        SMAX_CUDA(cudaStreamEndCapture(st, &g));
        cudaGraphExec_t ge = nullptr;
        cudaError_t e = cudaGraphInstantiate(&ge, g, 0);
        cudaGraphDestroy(g);
        cuda_check(e, "cudaGraphInstantiate");
        R.graph = ge;
        R.gkey[0] = key0;
        R.gkey[1] = key1;
        R.g_steps = steps;
        R.g_merge = merge;
        R.g_serial = k->tri_plan_serial;
        R.g_aver = k->a_version;
        R.g_pack = k->tri.pack.psrc.p;
    }
    SMAX_CUDA(cudaGraphLaunch(R.graph, st));
    if (fenced) R.aux.leave(k->stream);
    R.steps_done = steps;
    R.last_rel = -1.0;
}

}  // namespace smax

extern "C" smax_status smax_kernel_get_refine_stats(smax_kernel k, int *steps, double *last_rel_correction) {
    using namespace smax;
    return guarded([&] {
        smax_kernel_s *kk = K(k);
        RefineState &R = kk->refine;
        if (R.last_rel < 0.0) R.last_rel = R.steps_done > 0 ? read_rel(kk, kk->stream) : 0.0;
        if (steps) *steps = R.steps_done;
        if (last_rel_correction) *last_rel_correction = R.last_rel;
    });
}
