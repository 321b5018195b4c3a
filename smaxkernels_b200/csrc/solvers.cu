// solvers.cu -- the reference's iterative-solver applications on
// device-resident operators (smax_solver_*, include/smax_b200.h).
//
//   Jacobi        examples/applications/jacobi/jacobi.cpp:14-130,
//                 jacobi/utils.hpp:7-50
//   Gauss-Seidel  examples/applications/gauss_seidel/gauss_seidel.cpp:13-111,
//                 D+L / U split of examples/examples_common.hpp:283-398
//
// The applications call run() on SpMV and SpTRSV kernels once per iteration
// and do the vector arithmetic (normalize_x, subtract_vectors,
// infty_vec_norm) on the host.  Here the operators stay on the device and an
// iteration is one or two launches:
//  * Jacobi: a row-group kernel computes s = (A x_old)_r and, for the same row,
//    normalize_x's update x_new_r = (b_r - (s - D_r x_old_r)) / D_r.  Which of
//    the two buffers is x_old follows from the iteration count kept on the
//    device, so a block of iterations is one replayable launch sequence.
//  * Gauss-Seidel: a row-group kernel forms tmp = b - U x, then the platform's
//    level-scheduled SpTRSV (an internal kernel object on D+L, merged single-
//    CTA runs on its level pack) solves (D+L) x = tmp.
//  * The residual max_r |b_r - (A x)_r| is a row-group kernel with a block
//    maximum and one atomicMax on the bit pattern (non-negative doubles order
//    like their bits); a one-thread kernel records it, advances the iteration
//    count and decides whether the loop goes on.
// Systems of at most kSmallRows rows skip all of this: one CTA runs the whole
// loop in one launch (small_jacobi, small_gauss_seidel).
// A row group is G lanes (1, 2, ..., 32) that stride over the row's entries
// and add their partial sums with shuffles inside the group's lane mask.  G
// is chosen per matrix when the solver is created: the residual kernel (the
// same row loop) is timed for every G on the matrix itself and the fastest
// kept; matrices below 2^20 entries take the smallest power of two >= half
// the mean row length.
#include <cub/device/device_scan.cuh>

#include <cmath>
#include <cstring>
#include <type_traits>
#include <vector>

#include "abi_internal.cuh"

namespace smax {

namespace {

constexpr int kRowThreads = 256;
constexpr int64_t kMaxHistory = 1 << 20;  // residuals recorded per solve, at most

struct SolverState {
    unsigned long long norm_bits;  // running maximum of the residual being measured
    double norm;                   // the last residual measured
    int n_iters;                   // iterations completed
    int n_checks;                  // residuals recorded
    int active;                    // the loop goes on
    int pad;
};

unsigned row_grid(int64_t n, int G) {
    const int64_t cap = (int64_t)sm_count() * 8;
    int64_t g = (n * G + kRowThreads - 1) / kRowThreads;
    return (unsigned)(g < 1 ? 1 : (g > cap ? cap : g));
}

int group_guess(const DevCRS &m) {
    const double mean = m.n_rows ? (double)m.nnz / (double)m.n_rows : 1.0;
    int g = 1;
    while (g < 32 && 2 * g < mean) g <<= 1;
    return g;
}

template <int G> __device__ __forceinline__ unsigned group_mask() {
    if constexpr (G == 32) return 0xffffffffu;
    else return ((1u << G) - 1u) << ((threadIdx.x & 31) & ~(G - 1));
}

// (A x)_r by the G lanes of a group; every lane returns the full sum
template <typename VT, int G>
__device__ __forceinline__ VT row_dot(const int *__restrict__ rp, const int *__restrict__ ci,
                                      const VT *__restrict__ val, const VT *__restrict__ x, int64_t r, int lane,
                                      unsigned mask) {
    VT s = VT(0);
    const int e = rp[r + 1];
#pragma unroll 4
    for (int j = rp[r] + lane; j < e; j += G) s += val[j] * __ldg(x + ci[j]);
#pragma unroll
    for (int o = G / 2; o > 0; o >>= 1) s += __shfl_xor_sync(mask, s, o);
    return s;
}

// Jacobi iteration number st->n_iters + j + 1: odd iterations read x0 and
// write x1, even ones the reverse (the applications' pointer swap)
template <typename VT, int G>
__global__ void __launch_bounds__(kRowThreads)
    jacobi_kernel(const int *__restrict__ rp, const int *__restrict__ ci, const VT *__restrict__ val,
                  const VT *__restrict__ D, const VT *__restrict__ b, VT *x0, VT *x1,
                  const SolverState *__restrict__ st, int j, int64_t n) {
    const long long k = (long long)st->n_iters + j + 1;
    const VT *xo = (k & 1) ? x0 : x1;
    VT *xn = (k & 1) ? x1 : x0;
    const int lane = threadIdx.x & (G - 1);
    const unsigned mask = group_mask<G>();
    const int64_t stride = (int64_t)gridDim.x * (kRowThreads / G);
    for (int64_t r = ((int64_t)blockIdx.x * kRowThreads + threadIdx.x) / G; r < n; r += stride) {
        const VT s = row_dot<VT, G>(rp, ci, val, xo, r, lane, mask);
        if (lane == 0) {
            const VT d = D[r];
            const VT diag_contrib = d * xo[r];
            const VT offdiag_sum = s - diag_contrib;
            xn[r] = (b[r] - offdiag_sum) / d;
        }
    }
}

// tmp = b - U x (gauss_seidel.cpp:25-34: tmp <- Ux, then subtract_vectors)
template <typename VT, int G>
__global__ void __launch_bounds__(kRowThreads)
    rhs_kernel(const int *__restrict__ rp, const int *__restrict__ ci, const VT *__restrict__ val,
               const VT *__restrict__ x, const VT *__restrict__ b, VT *__restrict__ tmp, int64_t n) {
    const int lane = threadIdx.x & (G - 1);
    const unsigned mask = group_mask<G>();
    const int64_t stride = (int64_t)gridDim.x * (kRowThreads / G);
    for (int64_t r = ((int64_t)blockIdx.x * kRowThreads + threadIdx.x) / G; r < n; r += stride) {
        const VT s = row_dot<VT, G>(rp, ci, val, x, r, lane, mask);
        if (lane == 0) tmp[r] = b[r] - s;
    }
}

// st->norm_bits = max(st->norm_bits, max_r |b_r - (A x)_r|); NaNs never win
// (infty_vec_norm compares with >, applications_common.hpp:122-133)
template <typename VT, int G>
__global__ void __launch_bounds__(kRowThreads)
    residual_kernel(const int *__restrict__ rp, const int *__restrict__ ci, const VT *__restrict__ val,
                    const VT *__restrict__ x, const VT *__restrict__ b, int64_t n, SolverState *st) {
    const int lane = threadIdx.x & (G - 1);
    const unsigned mask = group_mask<G>();
    const int64_t stride = (int64_t)gridDim.x * (kRowThreads / G);
    double mx = 0.0;
    for (int64_t r = ((int64_t)blockIdx.x * kRowThreads + threadIdx.x) / G; r < n; r += stride) {
        const VT s = row_dot<VT, G>(rp, ci, val, x, r, lane, mask);
        if (lane == 0) {
            const double a = fabs((double)(b[r] - s));
            if (a > mx) mx = a;
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const double v = __shfl_xor_sync(0xffffffffu, mx, o);
        if (v > mx) mx = v;
    }
    __shared__ double warp_max[kRowThreads / 32];
    if ((threadIdx.x & 31) == 0) warp_max[threadIdx.x >> 5] = mx;
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < kRowThreads / 32; ++w)
            if (warp_max[w] > mx) mx = warp_max[w];
        if (mx > 0.0) atomicMax(&st->norm_bits, (unsigned long long)__double_as_longlong(mx));
    }
}

__global__ void reset_kernel(SolverState *st) {
    st->norm_bits = 0ull;
    st->norm = 0.0;
    st->n_iters = 0;
    st->n_checks = 0;
    st->active = 0;
}

// Records the residual just measured, adds the iterations of the block and
// decides whether the loop goes on; with set_handle it also sets the while
// node's condition (the loop of the DEVICE_LOOP driver ends within
// iter_limit / iters_in_block repetitions: n_iters only grows).
__global__ void decide_kernel(SolverState *st, double *hist, int hist_cap, double tol, int iters_in_block,
                              int iter_limit, cudaGraphConditionalHandle h, int set_handle) {
    const double norm = __longlong_as_double((long long)st->norm_bits);
    st->norm_bits = 0ull;
    st->norm = norm;
    if (st->n_checks < hist_cap) hist[st->n_checks] = norm;
    st->n_checks += 1;
    st->n_iters += iters_in_block;
    const int go = (norm > tol) && (st->n_iters < iter_limit);
    st->active = go;
    if (set_handle) cudaGraphSetConditional(h, go ? 1u : 0u);
}

// The diagonal of every row moved to its end (the last match when a row holds
// several), D = its value; a row without one, or with |a_ii| < 1e-16, is an
// error, as in peel_diag_crs (jacobi/utils.hpp:7-36).
template <typename VT>
__global__ void jacobi_diag_kernel(const int *__restrict__ rp, int *__restrict__ ci, VT *__restrict__ val, int64_t n,
                                   VT *__restrict__ D, DevStatus *status) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < n; r += stride) {
        const int s = rp[r], e = rp[r + 1] - 1;
        int dj = -1;
        for (int j = s; j <= e; ++j)
            if (ci[j] == (int)r) dj = j;
        if (dj < 0) {
            report(status, SMAX_ERR_NO_DIAG, r);
            continue;
        }
        const VT d = val[dj];
        if (fabs((double)d) < 1e-16) report(status, SMAX_ERR_ZERO_DIAG, r);
        D[r] = d;
        if (dj != e) {
            const int tc = ci[dj];
            ci[dj] = ci[e];
            ci[e] = tc;
            val[dj] = val[e];
            val[e] = d;
        }
    }
}

// entries with col <= row (D+L) and col > row (U) per row
__global__ void split_count_kernel(const int *__restrict__ rp, const int *__restrict__ ci, int64_t n,
                                   int *__restrict__ nl, int *__restrict__ nu) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < n; r += stride) {
        int l = 0;
        const int e = rp[r + 1];
        for (int j = rp[r]; j < e; ++j) l += ci[j] <= (int)r;
        nl[r] = l;
        nu[r] = (e - rp[r]) - l;
    }
}

// the split in each row's own entry order (extract_D_L_U keeps it)
template <typename VT>
__global__ void split_fill_kernel(const int *__restrict__ rp, const int *__restrict__ ci, const VT *__restrict__ val,
                                  int64_t n, const int *__restrict__ lrp, int *__restrict__ lci,
                                  VT *__restrict__ lval, const int *__restrict__ urp, int *__restrict__ uci,
                                  VT *__restrict__ uval) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < n; r += stride) {
        int pl = lrp[r], pu = urp[r];
        const int e = rp[r + 1];
        for (int j = rp[r]; j < e; ++j) {
            const int c = ci[j];
            if (c <= (int)r) {
                lci[pl] = c;
                lval[pl++] = val[j];
            } else {
                uci[pu] = c;
                uval[pu++] = val[j];
            }
        }
    }
}

// ---- small systems: the whole loop in one CTA -----------------------------
// Up to kSmallRows rows the loop runs in one launch of one CTA, exactly the
// applications' loop (the check every check_length iterations, the stop test
// before every iteration, iterations past the last full block unchecked),
// with x, b and D in shared memory and __syncthreads between the steps.  The
// loop ends after at most max_iters iterations.
constexpr int kSmallRows = 4096;
constexpr int kSmallThreads = 1024;
constexpr int kSmallStageBytes = 200 * 1024;  // dynamic shared memory of the one-CTA loop, at most

// block-wide maximum of non-negative doubles (NaNs never win); every thread
// returns it
__device__ double block_max(double v, double *red) {
    for (int o = 16; o > 0; o >>= 1) {
        const double w = __shfl_xor_sync(0xffffffffu, v, o);
        if (w > v) v = w;
    }
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        double m = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w)
            if (red[w] > m) m = red[w];
        red[32] = m;
    }
    __syncthreads();
    const double m = red[32];
    __syncthreads();
    return m;
}

// max_r |b_r - (A x)_r| with one thread per row, rows summed in entry order
template <typename VT>
__device__ double small_residual(const int *__restrict__ rp, const int *__restrict__ ci, const VT *__restrict__ val,
                                 const VT *x, const VT *b, int n, double *red) {
    double mx = 0.0;
    for (int r = threadIdx.x; r < n; r += blockDim.x) {
        VT s = VT(0);
        const int e = rp[r + 1];
#pragma unroll 4
        for (int j = rp[r]; j < e; ++j) s += val[j] * x[ci[j]];
        const double a = fabs((double)(b[r] - s));
        if (a > mx) mx = a;
    }
    return block_max(mx, red);
}

__device__ void small_record(SolverState *st, double *hist, int hist_cap, int &checks, double norm) {
    if (threadIdx.x == 0 && checks < hist_cap) hist[checks] = norm;
    ++checks;
}

template <typename VT>
__global__ void __launch_bounds__(kSmallThreads)
    small_jacobi(const int *__restrict__ rp, const int *__restrict__ ci, const VT *__restrict__ val,
                 const VT *__restrict__ Dg, const VT *__restrict__ bg, VT *x0g, VT *x1g, int n, double tol,
                 int max_iters, int cl, double *hist, int hist_cap, SolverState *st) {
    extern __shared__ __align__(16) unsigned char sm_raw[];
    __shared__ double red[33];
    VT *x0 = reinterpret_cast<VT *>(sm_raw), *x1 = x0 + n, *b = x1 + n, *D = b + n;
    for (int r = threadIdx.x; r < n; r += blockDim.x) {
        x0[r] = x0g[r];
        x1[r] = x1g[r];
        b[r] = bg[r];
        D[r] = Dg[r];
    }
    __syncthreads();
    int checks = 0, it = 0;
    double norm = small_residual<VT>(rp, ci, val, x1, b, n, red);  // x1: the first x_new buffer
    small_record(st, hist, hist_cap, checks, norm);
    while (norm > tol && it < max_iters) {
        const bool odd = ((it + 1) & 1) != 0;
        const VT *xo = odd ? x0 : x1;
        VT *xn = odd ? x1 : x0;
        for (int r = threadIdx.x; r < n; r += blockDim.x) {
            VT s = VT(0);
            const int e = rp[r + 1];
#pragma unroll 4
            for (int j = rp[r]; j < e; ++j) s += val[j] * xo[ci[j]];
            const VT diag_contrib = D[r] * xo[r];
            const VT offdiag_sum = s - diag_contrib;
            xn[r] = (b[r] - offdiag_sum) / D[r];
        }
        __syncthreads();
        ++it;
        if (it % cl == 0) {
            norm = small_residual<VT>(rp, ci, val, x1, b, n, red);
            small_record(st, hist, hist_cap, checks, norm);
        }
    }
    for (int r = threadIdx.x; r < n; r += blockDim.x) {
        x0g[r] = x0[r];
        x1g[r] = x1[r];
    }
    if (threadIdx.x == 0) {
        st->norm_bits = 0ull;
        st->norm = norm;
        st->n_iters = it;
        st->n_checks = checks;
        st->active = 0;
    }
}

// (D+L) has its diagonal as the last entry of every row (the SpTRSV kernel's
// peeled copy) and is solved level by level over `order`
// A thread's first row of level l of the Gauss-Seidel sweep (r = -1: none):
// its row index, entry range and first two entries (diagonal last, so e is
// the diagonal's slot), right-hand side and 1/D.
template <typename VT> struct GsRow {
    int r, j, e, c0, c1;
    VT v0, v1, t, d;
};

template <typename VT>
__device__ __forceinline__ GsRow<VT> gs_row(int l, int n_levels, const int *lvl_ptr, const int *order,
                                            const int *lrp, const int *lci, const VT *lval, const VT *tmp,
                                            const VT *D) {
    GsRow<VT> g{-1, 0, 0, 0, 0, VT(0), VT(0), VT(0), VT(0)};
    if (l >= n_levels) return g;
    const int i = lvl_ptr[l] + (int)threadIdx.x;
    if (i >= lvl_ptr[l + 1]) return g;
    g.r = order[i];
    g.j = lrp[g.r];
    g.e = lrp[g.r + 1] - 1;
    if (g.j < g.e) {
        g.c0 = lci[g.j];
        g.v0 = lval[g.j];
    }
    if (g.j + 1 < g.e) {
        g.c1 = lci[g.j + 1];
        g.v1 = lval[g.j + 1];
    }
    g.t = tmp[g.r];
    g.d = D[g.r];
    return g;
}

template <typename VT>
__global__ void __launch_bounds__(kSmallThreads)
    small_gauss_seidel(const int *__restrict__ arp, const int *__restrict__ aci, const VT *__restrict__ aval,
                       const int *__restrict__ urp, const int *__restrict__ uci, const VT *__restrict__ uval,
                       const int *__restrict__ lrp, const int *__restrict__ lci, const VT *__restrict__ lval,
                       const VT *__restrict__ Dg, const int *__restrict__ order_g, const int *__restrict__ lvl_g,
                       int n_levels, const VT *__restrict__ bg, VT *xg, int n, double tol, int max_iters, int cl,
                       double *hist, int hist_cap, SolverState *st, int stage) {
    extern __shared__ __align__(16) unsigned char sm_raw[];
    __shared__ double red[33];
    VT *x = reinterpret_cast<VT *>(sm_raw), *tmp = x + n, *b = tmp + n, *D = b + n;
    for (int r = threadIdx.x; r < n; r += blockDim.x) {
        x[r] = xg[r];
        b[r] = bg[r];
        D[r] = VT(1) / Dg[r];  // the sweep multiplies by 1/D, as the level-pack SpTRSV does
    }
    // with stage, the level sweep's arrays follow the vectors in shared memory:
    // its chain of dependent loads per level then never leaves the SM
    const int *order = order_g, *lvl_ptr = lvl_g, *lrp_s = lrp, *lci_s = lci;
    const VT *lval_s = lval;
    if (stage) {
        const int nl = lrp[n];
        VT *sv = D + n;
        int *si = reinterpret_cast<int *>(sv + nl);
        int *so = si, *sp = so + n, *sl = sp + n + 1, *sc = sl + n_levels + 1;
        for (int j = threadIdx.x; j < nl; j += blockDim.x) {
            sv[j] = lval[j];
            sc[j] = lci[j];
        }
        for (int r = threadIdx.x; r < n; r += blockDim.x) so[r] = order_g[r];
        for (int r = threadIdx.x; r <= n; r += blockDim.x) sp[r] = lrp[r];
        for (int l = threadIdx.x; l <= n_levels; l += blockDim.x) sl[l] = lvl_g[l];
        order = so;
        lvl_ptr = sl;
        lrp_s = sp;
        lci_s = sc;
        lval_s = sv;
    }
    __syncthreads();
    int checks = 0, it = 0;
    double norm = small_residual<VT>(arp, aci, aval, x, b, n, red);
    small_record(st, hist, hist_cap, checks, norm);
    while (norm > tol && it < max_iters) {
        for (int r = threadIdx.x; r < n; r += blockDim.x) {
            VT s = VT(0);
            const int e = urp[r + 1];
#pragma unroll 4
            for (int j = urp[r]; j < e; ++j) s += uval[j] * x[uci[j]];
            tmp[r] = b[r] - s;
        }
        __syncthreads();
        // Each thread's first row of the next level -- its row index, its
        // first two entries, its right-hand side and 1/D -- is loaded while
        // the current level is solved, so a level's chain is only the reads
        // of x, the products and the store.  Further rows of a level wider
        // than the CTA are read in place.
        GsRow<VT> cur = gs_row<VT>(0, n_levels, lvl_ptr, order, lrp_s, lci_s, lval_s, tmp, D);
        for (int l = 0; l < n_levels; ++l) {
            const GsRow<VT> nxt = gs_row<VT>(l + 1, n_levels, lvl_ptr, order, lrp_s, lci_s, lval_s, tmp, D);
            if (cur.r >= 0) {
                VT s = VT(0);
                if (cur.j < cur.e) s += cur.v0 * x[cur.c0];
                if (cur.j + 1 < cur.e) s += cur.v1 * x[cur.c1];
#pragma unroll 4
                for (int j = cur.j + 2; j < cur.e; ++j) s += lval_s[j] * x[lci_s[j]];
                x[cur.r] = (cur.t - s) * cur.d;
            }
            for (int i = lvl_ptr[l] + threadIdx.x + blockDim.x; i < lvl_ptr[l + 1]; i += blockDim.x) {
                const int r = order[i];
                VT s = VT(0);
                const int e = lrp_s[r + 1] - 1;
#pragma unroll 4
                for (int j = lrp_s[r]; j < e; ++j) s += lval_s[j] * x[lci_s[j]];
                x[r] = (tmp[r] - s) * D[r];
            }
            __syncthreads();
            cur = nxt;
        }
        ++it;
        if (it % cl == 0) {
            norm = small_residual<VT>(arp, aci, aval, x, b, n, red);
            small_record(st, hist, hist_cap, checks, norm);
        }
    }
    for (int r = threadIdx.x; r < n; r += blockDim.x) xg[r] = x[r];
    if (threadIdx.x == 0) {
        st->norm_bits = 0ull;
        st->norm = norm;
        st->n_iters = it;
        st->n_checks = checks;
        st->active = 0;
    }
}

unsigned flat_grid(int64_t n) {
    const int64_t cap = (int64_t)sm_count() * 8;
    int64_t g = (n + 255) / 256;
    return (unsigned)(g < 1 ? 1 : (g > cap ? cap : g));
}

// row_ptr (n + 1 entries) = exclusive prefix sum of counts[n]
void counts_to_row_ptr(const int *counts, int64_t n, int *row_ptr, cudaStream_t st) {
    SMAX_CUDA(cudaMemsetAsync(row_ptr, 0, sizeof(int), st));
    if (n == 0) return;
    size_t tb = 0;
    SMAX_CUDA(cub::DeviceScan::InclusiveSum(nullptr, tb, counts, row_ptr + 1, (int)n, st));
    DevBuf tmp(tb);
    SMAX_CUDA(cub::DeviceScan::InclusiveSum(tmp.p, tb, counts, row_ptr + 1, (int)n, st));
    SMAX_CUDA(cudaStreamSynchronize(st));
}

void check_status(DevBuf &status, cudaStream_t st, const char *what) {
    DevStatus h{};
    SMAX_CUDA(cudaMemcpyAsync(&h, status.p, sizeof(h), cudaMemcpyDeviceToHost, st));
    SMAX_CUDA(cudaStreamSynchronize(st));
    if (h.code) fail(h.code, std::string(what) + " (code " + std::to_string(h.code) + " at row " +
                                 std::to_string(h.index) + ")");
}

void abi_check(smax_status s) {
    if (s != SMAX_OK) fail(s, last_error());
}

template <typename F> void with_group(int G, F &&f) {
    switch (G) {
    case 1: f(std::integral_constant<int, 1>{}); break;
    case 2: f(std::integral_constant<int, 2>{}); break;
    case 4: f(std::integral_constant<int, 4>{}); break;
    case 8: f(std::integral_constant<int, 8>{}); break;
    case 16: f(std::integral_constant<int, 16>{}); break;
    default: f(std::integral_constant<int, 32>{}); break;
    }
}

}  // namespace

}  // namespace smax

using namespace smax;

struct smax_solver_s {
    int kind = 0, vbytes = 8;
    int64_t n = 0;
    cudaStream_t own = nullptr;
    DevCRS A;  // Jacobi: diagonal last in each row; Gauss-Seidel: as given
    DevCRS U;  // Gauss-Seidel: the entries above the diagonal
    int gA = 1, gU = 1;
    DevBuf D;                // Jacobi: the diagonal
    DevBuf x0, x1, b, tmp;  // iterate buffers, right-hand side, Gauss-Seidel's rhs of the solve
    DevBuf state, hist;
    int hist_cap = 0;
    DevBuf small_lvl;  // Gauss-Seidel, small systems: the D+L level pointer on the device
    SolverState *h_state = nullptr;  // pinned copy of the state
    smax_kernel tri = nullptr;       // Gauss-Seidel: SpTRSV on D+L
    // cached graphs and what they were built for
    cudaGraphExec_t g_loop = nullptr, g_pro = nullptr, g_block = nullptr;
    double g_tol = -1.0;
    int g_limit = -1, g_cl = -1;
    void *g_hist = nullptr;
    int last_checks = 0;

    ~smax_solver_s() {
        if (own) cudaStreamSynchronize(own);
        release_graphs();
        if (tri) smax_kernel_destroy(tri);
        if (h_state) cudaFreeHost(h_state);
        if (own) cudaStreamDestroy(own);
    }
    void release_graphs() {
        if (g_loop) cudaGraphExecDestroy(g_loop);
        if (g_pro) cudaGraphExecDestroy(g_pro);
        if (g_block) cudaGraphExecDestroy(g_block);
        g_loop = g_pro = g_block = nullptr;
        g_tol = -1.0;
        g_limit = g_cl = -1;
        g_hist = nullptr;
    }
    SolverState *dstate() const { return state.as<SolverState>(); }

    // ---- the launches shared by every driver
    template <typename VT> void iterate(int j, cudaStream_t st) {
        const int64_t nn = n;
        if (kind == SMAX_SOLVER_JACOBI) {
            with_group(gA, [&](auto g) {
                constexpr int G = decltype(g)::value;
                jacobi_kernel<VT, G><<<row_grid(nn, G), kRowThreads, 0, st>>>(
                    A.rp(), A.ci(), A.val.as<VT>(), D.as<VT>(), b.as<VT>(), x0.as<VT>(), x1.as<VT>(), dstate(), j,
                    nn);
            });
        } else {
            with_group(gU, [&](auto g) {
                constexpr int G = decltype(g)::value;
                rhs_kernel<VT, G><<<row_grid(nn, G), kRowThreads, 0, st>>>(U.rp(), U.ci(), U.val.as<VT>(),
                                                                           x0.as<VT>(), b.as<VT>(), tmp.as<VT>(), nn);
            });
            SMAX_CUDA(cudaGetLastError());
            smax_kernel_s *t = K(tri);
            t->stream = st;
            apply_core(t, 0, 0);
        }
        SMAX_CUDA(cudaGetLastError());
    }
    template <typename VT> void residual(cudaStream_t st) {
        // Jacobi measures the first x_new buffer (x1), Gauss-Seidel its x
        const VT *x = kind == SMAX_SOLVER_JACOBI ? x1.as<VT>() : x0.as<VT>();
        const int64_t nn = n;
        with_group(gA, [&](auto g) {
            constexpr int G = decltype(g)::value;
            residual_kernel<VT, G><<<row_grid(nn, G), kRowThreads, 0, st>>>(A.rp(), A.ci(), A.val.as<VT>(), x,
                                                                            b.as<VT>(), nn, dstate());
        });
        SMAX_CUDA(cudaGetLastError());
    }
    void decide(double tol, int iters, int limit, cudaGraphConditionalHandle h, bool set, cudaStream_t st) {
        decide_kernel<<<1, 1, 0, st>>>(dstate(), hist.as<double>(), hist_cap, tol, iters, limit, h, set ? 1 : 0);
        SMAX_CUDA(cudaGetLastError());
    }
    template <typename VT>
    void prologue(double tol, int limit, cudaGraphConditionalHandle h, bool set, cudaStream_t st) {
        reset_kernel<<<1, 1, 0, st>>>(dstate());
        SMAX_CUDA(cudaGetLastError());
        residual<VT>(st);
        decide(tol, 0, limit, h, set, st);
    }
    template <typename VT>
    void block(double tol, int cl, int limit, cudaGraphConditionalHandle h, bool set, cudaStream_t st) {
        for (int j = 0; j < cl; ++j) iterate<VT>(j, st);
        residual<VT>(st);
        decide(tol, cl, limit, h, set, st);
    }

    // the fastest row-group width for the row loop over m (the residual
    // kernel, or with rhs the tmp = b - U x kernel), timed on m itself
    template <typename VT> int tune_group(const DevCRS &m, bool rhs, cudaStream_t st) {
        const int guess = group_guess(m);
        if (m.nnz < (1 << 20)) return guess;
        const int64_t nn = m.n_rows;
        auto launch = [&](int g_) {
            with_group(g_, [&](auto g) {
                constexpr int G = decltype(g)::value;
                if (rhs)
                    rhs_kernel<VT, G><<<row_grid(nn, G), kRowThreads, 0, st>>>(m.rp(), m.ci(), m.val.as<VT>(),
                                                                               x0.as<VT>(), b.as<VT>(), tmp.as<VT>(),
                                                                               nn);
                else
                    residual_kernel<VT, G><<<row_grid(nn, G), kRowThreads, 0, st>>>(m.rp(), m.ci(), m.val.as<VT>(),
                                                                                    x0.as<VT>(), b.as<VT>(), nn,
                                                                                    dstate());
            });
            SMAX_CUDA(cudaGetLastError());
        };
        cudaEvent_t e0 = nullptr, e1 = nullptr;
        SMAX_CUDA(cudaEventCreate(&e0));
        SMAX_CUDA(cudaEventCreate(&e1));
        int best = guess;
        float best_ms = 3.4e38f;
        try {
            for (int G = 1; G <= 32; G <<= 1) {
                launch(G);
                SMAX_CUDA(cudaEventRecord(e0, st));
                for (int r = 0; r < 3; ++r) launch(G);
                SMAX_CUDA(cudaEventRecord(e1, st));
                SMAX_CUDA(cudaEventSynchronize(e1));
                float ms = 0.f;
                SMAX_CUDA(cudaEventElapsedTime(&ms, e0, e1));
                if (ms < best_ms) {
                    best_ms = ms;
                    best = G;
                }
            }
        } catch (...) {
            cudaEventDestroy(e0);
            cudaEventDestroy(e1);
            throw;
        }
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        return best;
    }

    void read_state(cudaStream_t st) {
        SMAX_CUDA(cudaMemcpyAsync(h_state, state.p, sizeof(SolverState), cudaMemcpyDeviceToHost, st));
        SMAX_CUDA(cudaStreamSynchronize(st));
    }

    // ---- graphs
    template <typename F> cudaGraphExec_t capture(F &&f) {
        cudaStreamCaptureMode mode = cudaStreamCaptureModeThreadLocal;
        SMAX_CUDA(cudaStreamSynchronize(own));
        SMAX_CUDA(cudaStreamBeginCapture(own, mode));
        cudaGraph_t g = nullptr;
        try {
            f(own);
        } catch (...) {
            cudaStreamEndCapture(own, &g);
            if (g) cudaGraphDestroy(g);
            throw;
        }
        SMAX_CUDA(cudaStreamEndCapture(own, &g));
        cudaGraphExec_t e = nullptr;
        cudaError_t err = cudaGraphInstantiate(&e, g, 0);
        cudaGraphDestroy(g);
        cuda_check(err, "cudaGraphInstantiate");
        return e;
    }

    // prologue, then while (active) { block } as one graph: the while node's
    // condition is set by the decide kernels
    template <typename VT> cudaGraphExec_t build_loop(double tol, int cl, int limit) {
        SMAX_CUDA(cudaStreamSynchronize(own));
        cudaGraph_t g = nullptr;
        SMAX_CUDA(cudaGraphCreate(&g, 0));
        struct Holder {
            cudaGraph_t g;
            ~Holder() {
                if (g) cudaGraphDestroy(g);
            }
        } hold{g};
        cudaGraphConditionalHandle h;
        SMAX_CUDA(cudaGraphConditionalHandleCreate(&h, g, 0, 0));
        const cudaStreamCaptureMode mode = cudaStreamCaptureModeThreadLocal;
        // the prologue, captured into g, then the while node after it
        SMAX_CUDA(cudaStreamBeginCaptureToGraph(own, g, nullptr, nullptr, 0, mode));
        cudaGraph_t body = nullptr;
        try {
            prologue<VT>(tol, limit, h, true, own);
            cudaStreamCaptureStatus cs;
            const cudaGraphNode_t *deps = nullptr;
            size_t nd = 0;
            SMAX_CUDA(cudaStreamGetCaptureInfo(own, &cs, nullptr, nullptr, &deps, &nd));
            cudaGraphNodeParams cp = {};
            cp.type = cudaGraphNodeTypeConditional;
            cp.conditional.handle = h;
            cp.conditional.type = cudaGraphCondTypeWhile;
            cp.conditional.size = 1;
            cudaGraphNode_t node;
            SMAX_CUDA(cudaGraphAddNode(&node, g, deps, nd, &cp));
            body = cp.conditional.phGraph_out[0];
            SMAX_CUDA(cudaStreamUpdateCaptureDependencies(own, &node, 1, cudaStreamSetCaptureDependencies));
        } catch (...) {
            cudaGraph_t dummy = nullptr;
            cudaStreamEndCapture(own, &dummy);
            throw;
        }
        cudaGraph_t out = nullptr;
        SMAX_CUDA(cudaStreamEndCapture(own, &out));
        // the body: one block of iterations and its residual
        SMAX_CUDA(cudaStreamBeginCaptureToGraph(own, body, nullptr, nullptr, 0, mode));
        try {
            block<VT>(tol, cl, limit, h, true, own);
        } catch (...) {
            cudaGraph_t dummy = nullptr;
            cudaStreamEndCapture(own, &dummy);
            throw;
        }
        SMAX_CUDA(cudaStreamEndCapture(own, &out));
        cudaGraphExec_t e = nullptr;
        SMAX_CUDA(cudaGraphInstantiate(&e, g, 0));
        return e;
    }

    template <typename VT> void solve(const void *b_in, void *x_inout, const smax_solver_opts &o,
                                      smax_solver_stats &stats, cudaStream_t st) {
        const int cl = o.check_length;
        const int n_full = o.max_iters / cl;
        const int limit = n_full * cl;
        const int rem = o.max_iters - limit;
        const size_t vb = (size_t)vbytes * n;
        stats = smax_solver_stats{};
        if (n == 0) {
            // an empty residual is 0: no iteration runs
            stats.converged = 0.0 < o.tol;
            stats.n_checks = 1;
            last_checks = 0;
            return;
        }
        // the residual history keeps at most kMaxHistory entries (the count
        // of checks is still exact)
        const int want = (int)std::min<int64_t>((int64_t)n_full + 1, kMaxHistory);
        if (want > hist_cap) {
            hist.alloc(sizeof(double) * want);
            hist_cap = want;
        }
        SMAX_CUDA(cudaMemcpyAsync(b.p, b_in, vb, cudaMemcpyDefault, st));
        SMAX_CUDA(cudaMemcpyAsync(x0.p, x_inout, vb, cudaMemcpyDefault, st));
        if (kind == SMAX_SOLVER_JACOBI) SMAX_CUDA(cudaMemcpyAsync(x1.p, x_inout, vb, cudaMemcpyDefault, st));
        if (n <= kSmallRows) {
            // every driver: the whole loop in one CTA, one launch
            const size_t shm = (size_t)4 * vbytes * n;
            // one thread per row up to kSmallThreads: idle warps only add to every barrier
            const int threads = (int)std::min<int64_t>(kSmallThreads, std::max<int64_t>(32, (n + 31) / 32 * 32));
            if (kind == SMAX_SOLVER_JACOBI) {
                SMAX_CUDA(cudaFuncSetAttribute(small_jacobi<VT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                               (int)shm));
                small_jacobi<VT><<<1, threads, shm, st>>>(A.rp(), A.ci(), A.val.as<VT>(), D.as<VT>(),
                                                                b.as<VT>(), x0.as<VT>(), x1.as<VT>(), (int)n, o.tol,
                                                                o.max_iters, cl, hist.as<double>(), hist_cap,
                                                                dstate());
            } else {
                smax_kernel_s *t = K(tri);
                // the level sweep's arrays in shared memory too, when they fit
                const int64_t nl = t->dA.nnz, L = t->tri.n_levels();
                const size_t staged = shm + (size_t)vbytes * nl + sizeof(int) * (size_t)(n + (n + 1) + (L + 1) + nl);
                const int stage = staged <= (size_t)kSmallStageBytes ? 1 : 0;
                const size_t bytes = stage ? staged : shm;
                SMAX_CUDA(cudaFuncSetAttribute(small_gauss_seidel<VT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                               (int)bytes));
                small_gauss_seidel<VT><<<1, threads, bytes, st>>>(
                    A.rp(), A.ci(), A.val.as<VT>(), U.rp(), U.ci(), U.val.as<VT>(), t->dA.rp(), t->dA.ci(),
                    t->dA.val.as<VT>(), t->D.as<VT>(), t->tri.order.as<int>(), small_lvl.as<int>(), (int)L,
                    b.as<VT>(), x0.as<VT>(), (int)n, o.tol, o.max_iters, cl, hist.as<double>(), hist_cap, dstate(),
                    stage);
            }
            SMAX_CUDA(cudaGetLastError());
            read_state(st);
            const int n_iters = h_state->n_iters;
            const void *latest = (kind == SMAX_SOLVER_JACOBI && (n_iters & 1)) ? x1.p : x0.p;
            SMAX_CUDA(cudaMemcpyAsync(x_inout, latest, vb, cudaMemcpyDefault, st));
            SMAX_CUDA(cudaStreamSynchronize(st));
            stats.n_iters = n_iters;
            stats.residual_norm = h_state->norm;
            stats.converged = h_state->norm < o.tol;
            stats.n_checks = h_state->n_checks;
            stats.host_waits = 1;
            last_checks = h_state->n_checks;
            return;
        }
        const bool graphs = o.mode != SMAX_SOLVER_PLAIN;
        if (graphs && (g_tol != o.tol || g_limit != limit || g_cl != cl || g_hist != hist.p)) {
            release_graphs();
            g_tol = o.tol;
            g_limit = limit;
            g_cl = cl;
            g_hist = hist.p;
        }
        int waits = 0;
        if (o.mode == SMAX_SOLVER_DEVICE_LOOP) {
            if (!g_loop) g_loop = build_loop<VT>(o.tol, cl, limit);
            SMAX_CUDA(cudaGraphLaunch(g_loop, st));
        } else {
            if (graphs && !g_pro) {
                g_pro = capture([&](cudaStream_t cs) { prologue<VT>(o.tol, limit, 0, false, cs); });
                g_block = capture([&](cudaStream_t cs) { block<VT>(o.tol, cl, limit, 0, false, cs); });
            }
            if (graphs) SMAX_CUDA(cudaGraphLaunch(g_pro, st));
            else prologue<VT>(o.tol, limit, 0, false, st);
            read_state(st);
            ++waits;
            while (h_state->active) {
                if (graphs) SMAX_CUDA(cudaGraphLaunch(g_block, st));
                else block<VT>(o.tol, cl, limit, 0, false, st);
                read_state(st);
                ++waits;
            }
        }
        read_state(st);
        int n_iters = h_state->n_iters;
        const double norm = h_state->norm;
        // the iterations past the last full block run without a residual check
        if (norm > o.tol && n_iters < o.max_iters && rem > 0) {
            for (int j = 0; j < rem; ++j) iterate<VT>(j, st);
            n_iters += rem;
        }
        const void *latest = (kind == SMAX_SOLVER_JACOBI && (n_iters & 1)) ? x1.p : x0.p;
        SMAX_CUDA(cudaMemcpyAsync(x_inout, latest, vb, cudaMemcpyDefault, st));
        SMAX_CUDA(cudaStreamSynchronize(st));
        stats.n_iters = n_iters;
        stats.residual_norm = norm;
        stats.converged = norm < o.tol;
        stats.n_checks = h_state->n_checks;
        stats.host_waits = o.mode == SMAX_SOLVER_DEVICE_LOOP ? 1 : waits;
        last_checks = h_state->n_checks;
    }
};

namespace {

template <typename VT> void build_jacobi(smax_solver_s *s, const RegCRS &r, cudaStream_t st) {
    upload_crs(s->A, r, sizeof(VT), st);
    DevBuf status(sizeof(DevStatus));
    SMAX_CUDA(cudaMemsetAsync(status.p, 0, sizeof(DevStatus), st));
    validate_crs(s->A, status.as<DevStatus>(), st);
    check_status(status, st, "malformed matrix");
    s->D.alloc(sizeof(VT) * s->n);
    jacobi_diag_kernel<VT><<<flat_grid(s->n), 256, 0, st>>>(s->A.rp(), s->A.col.as<int>(), s->A.val.as<VT>(), s->n,
                                                            s->D.as<VT>(), status.as<DevStatus>());
    SMAX_CUDA(cudaGetLastError());
    check_status(status, st, "Jacobi needs a non-zero diagonal entry in every row");
    s->gA = s->tune_group<VT>(s->A, false, st);
}

template <typename VT> void build_gauss_seidel(smax_solver_s *s, const RegCRS &r, int float_type, cudaStream_t st) {
    upload_crs(s->A, r, sizeof(VT), st);
    DevBuf status(sizeof(DevStatus));
    SMAX_CUDA(cudaMemsetAsync(status.p, 0, sizeof(DevStatus), st));
    validate_crs(s->A, status.as<DevStatus>(), st);
    check_status(status, st, "malformed matrix");
    const int64_t n = s->n;
    DevBuf nl(sizeof(int) * n), nu(sizeof(int) * n), lrp(sizeof(int) * (n + 1));
    s->U.n_rows = n;
    s->U.n_cols = n;
    s->U.row_ptr.alloc(sizeof(int) * (n + 1));
    split_count_kernel<<<flat_grid(n), 256, 0, st>>>(s->A.rp(), s->A.ci(), n, nl.as<int>(), nu.as<int>());
    SMAX_CUDA(cudaGetLastError());
    counts_to_row_ptr(nl.as<int>(), n, lrp.as<int>(), st);
    counts_to_row_ptr(nu.as<int>(), n, s->U.row_ptr.as<int>(), st);
    int nnz_l = 0, nnz_u = 0;
    SMAX_CUDA(cudaMemcpyAsync(&nnz_l, lrp.as<int>() + n, sizeof(int), cudaMemcpyDeviceToHost, st));
    SMAX_CUDA(cudaMemcpyAsync(&nnz_u, s->U.row_ptr.as<int>() + n, sizeof(int), cudaMemcpyDeviceToHost, st));
    SMAX_CUDA(cudaStreamSynchronize(st));
    s->U.nnz = nnz_u;
    s->U.col.alloc(sizeof(int) * (nnz_u > 0 ? nnz_u : 1));
    s->U.val.alloc(sizeof(VT) * (nnz_u > 0 ? nnz_u : 1));
    DevBuf lci(sizeof(int) * (nnz_l > 0 ? nnz_l : 1)), lval(sizeof(VT) * (nnz_l > 0 ? nnz_l : 1));
    split_fill_kernel<VT><<<flat_grid(n), 256, 0, st>>>(s->A.rp(), s->A.ci(), s->A.val.as<VT>(), n, lrp.as<int>(),
                                                        lci.as<int>(), lval.as<VT>(), s->U.rp(), s->U.col.as<int>(),
                                                        s->U.val.as<VT>());
    SMAX_CUDA(cudaGetLastError());
    SMAX_CUDA(cudaStreamSynchronize(st));
    s->gA = s->tune_group<VT>(s->A, false, st);
    s->gU = s->tune_group<VT>(s->U, true, st);
    // the D+L solve: a SpTRSV kernel object of this platform on device arrays
    // (initialize copies them and peels the diagonal), launched without its
    // own graphs so that its launches join the solver's
    abi_check(smax_kernel_create(&s->tri, nullptr, SMAX_KERNEL_SPTRSV, SMAX_INT32, float_type));
    abi_check(smax_kernel_set_flag(s->tri, SMAX_FLAG_DEVICE_POINTERS, 1));
    abi_check(smax_kernel_set_flag(s->tri, SMAX_FLAG_SOLVE_MODE, SMAX_SOLVE_MERGED));
    abi_check(smax_kernel_register_A_crs(s->tri, n, n, nnz_l, lci.p, lrp.p, lval.p));
    abi_check(smax_kernel_register_dense(s->tri, 1, n, 1, s->x0.p));
    abi_check(smax_kernel_register_dense(s->tri, 2, n, 1, s->tmp.p));
    abi_check(smax_kernel_set_stream(s->tri, st));
    abi_check(smax_kernel_initialize(s->tri, 0, 0, 0));
    // one solve outside any capture builds the level schedule and pack
    SMAX_CUDA(cudaMemsetAsync(s->tmp.p, 0, sizeof(VT) * n, st));
    smax_kernel_s *t = K(s->tri);
    t->stream = st;
    apply_core(t, 0, 0);
    read_status(t);
    if (n > 0 && n <= kSmallRows) {
        // the one-CTA loop walks the SpTRSV plan's levels itself
        if (!t->tri.has_order) fail(SMAX_ERR_STATE, "the D+L plan has no level order");
        const std::vector<int> &lp = t->tri.lvl_ptr;
        s->small_lvl.alloc(sizeof(int) * lp.size());
        SMAX_CUDA(cudaMemcpyAsync(s->small_lvl.p, lp.data(), sizeof(int) * lp.size(), cudaMemcpyHostToDevice, st));
        SMAX_CUDA(cudaStreamSynchronize(st));
    }
}

}  // namespace

extern "C" {

smax_status smax_solver_create(smax_solver *out, int kind, int float_type, uint64_t n_rows, uint64_t nnz,
                               const void *row_ptr, const void *col, const void *val) {
    return guarded([&] {
        if (!out) fail(SMAX_ERR_BAD_ARG, "null output");
        if (kind != SMAX_SOLVER_JACOBI && kind != SMAX_SOLVER_GAUSS_SEIDEL) fail(SMAX_ERR_BAD_ARG, "unknown solver");
        if (float_type != SMAX_FLOAT32 && float_type != SMAX_FLOAT64)
            fail(SMAX_ERR_UNSUPPORTED_TYPE, "value type must be float32 or float64");
        if (!row_ptr || (nnz && (!col || !val))) fail(SMAX_ERR_BAD_ARG, "null matrix array");
        auto *s = new smax_solver_s();
        try {
            s->kind = kind;
            s->vbytes = float_type == SMAX_FLOAT64 ? 8 : 4;
            s->n = (int64_t)n_rows;
            SMAX_CUDA(cudaStreamCreateWithFlags(&s->own, cudaStreamNonBlocking));
            SMAX_CUDA(cudaMallocHost(reinterpret_cast<void **>(&s->h_state), sizeof(SolverState)));
            std::memset(s->h_state, 0, sizeof(SolverState));
            s->state.alloc(sizeof(SolverState));
            SMAX_CUDA(cudaMemsetAsync(s->state.p, 0, sizeof(SolverState), s->own));
            const size_t vb = (size_t)s->vbytes * (n_rows ? n_rows : 1);
            s->x0.alloc(vb);
            s->x1.alloc(vb);
            s->b.alloc(vb);
            s->tmp.alloc(vb);
            RegCRS r{true, n_rows, n_rows, nnz, const_cast<void *>(col), const_cast<void *>(row_ptr),
                     const_cast<void *>(val)};
            if (kind == SMAX_SOLVER_JACOBI) {
                if (s->vbytes == 8) build_jacobi<double>(s, r, s->own);
                else build_jacobi<float>(s, r, s->own);
            } else {
                if (s->vbytes == 8) build_gauss_seidel<double>(s, r, float_type, s->own);
                else build_gauss_seidel<float>(s, r, float_type, s->own);
            }
            SMAX_CUDA(cudaStreamSynchronize(s->own));
        } catch (...) {
            delete s;
            throw;
        }
        *out = s;
    });
}

smax_status smax_solver_solve(smax_solver s, const void *b, void *x, const smax_solver_opts *opts,
                              smax_solver_stats *stats, void *stream) {
    return guarded([&] {
        if (!s || !opts) fail(SMAX_ERR_BAD_ARG, "null argument");
        if (s->n && (!b || !x)) fail(SMAX_ERR_BAD_ARG, "null operand");
        if (opts->check_length < 1 || opts->max_iters < 0) fail(SMAX_ERR_BAD_ARG, "check_length >= 1, max_iters >= 0");
        if (opts->mode < SMAX_SOLVER_DEVICE_LOOP || opts->mode > SMAX_SOLVER_PLAIN)
            fail(SMAX_ERR_BAD_ARG, "unknown solver mode");
        if (std::isnan(opts->tol)) fail(SMAX_ERR_BAD_ARG, "tol is NaN");
        cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : s->own;
        smax_solver_stats out{};
        if (s->vbytes == 8) s->solve<double>(b, x, *opts, out, st);
        else s->solve<float>(b, x, *opts, out, st);
        if (s->tri) read_status(K(s->tri));
        if (stats) *stats = out;
    });
}

smax_status smax_solver_get_history(smax_solver s, double *out, int cap, int *count) {
    return guarded([&] {
        if (!s) fail(SMAX_ERR_BAD_ARG, "null solver");
        const int n = s->last_checks < s->hist_cap ? s->last_checks : s->hist_cap;
        const int m = n < cap ? n : cap;
        if (m > 0) {
            if (!out) fail(SMAX_ERR_BAD_ARG, "null output");
            SMAX_CUDA(cudaMemcpy(out, s->hist.p, sizeof(double) * m, cudaMemcpyDeviceToHost));
        }
        if (count) *count = s->last_checks;
    });
}

smax_status smax_solver_destroy(smax_solver s) {
    return guarded([&] { delete s; });
}

}  // extern "C"
