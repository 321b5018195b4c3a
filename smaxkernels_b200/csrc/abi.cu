// abi.cu -- exported C functions of include/smax_b200.h for contexts, kernel
// objects, registration and the initialize / apply / finalize cycle.
//
// Dispatch mirrors the reference's L2 kernel fronts (src/kernels/spmv.hpp:138-195,
// spmm.hpp:68-100): the kernel type and the flags pick the format and kernel.
#include <algorithm>
#include <cstring>
#include <optional>

#include "abi_internal.cuh"
#include "sptrsv_batch.cuh"

smax_kernel_s::~smax_kernel_s() {
    if (stream) cudaStreamSynchronize(stream);
    if (copy_stream) {
        cudaStreamSynchronize(copy_stream);
        cudaStreamDestroy(copy_stream);
    }
    for (auto &r : out_ranges) cudaEventDestroy(r.ev);
    for (auto e : ev_pool) cudaEventDestroy(e);
    if (own_stream) cudaStreamDestroy(own_stream);
}

using namespace smax;

namespace smax {

void require(bool c, int code, const char *msg) {
    if (!c) fail(code, msg);
}

smax_kernel_s *K(smax_kernel k) {
    require(k != nullptr, SMAX_ERR_BAD_ARG, "null kernel handle");
    return k;
}

namespace {
// The status word, after the work queued on the kernel's stream.
DevStatus fetch_status(smax_kernel_s *k) {
    DevStatus st{};
    SMAX_CUDA(cudaMemcpyAsync(&st, k->status.p, sizeof(st), cudaMemcpyDeviceToHost, k->stream));
    SMAX_CUDA(cudaStreamSynchronize(k->stream));
    return st;
}

// A recorded device error: clear it and report it.
void check_status(smax_kernel_s *k, const DevStatus &st) {
    if (st.code != 0) {
        SMAX_CUDA(cudaMemsetAsync(k->status.p, 0, sizeof(DevStatus), k->stream));
        SMAX_CUDA(cudaStreamSynchronize(k->stream));
        fail(st.code, "device reported error " + std::to_string(st.code) + " at index " + std::to_string(st.index));
    }
}
}  // namespace

void read_status(smax_kernel_s *k) {
    if (!k->status.p) return;
    check_status(k, fetch_status(k));
}

DevStatus *dstatus(smax_kernel_s *k) { return k->status.as<DevStatus>(); }

bool is_tri(const smax_kernel_s *k) { return k->ktype == SMAX_KERNEL_SPTRSV || k->ktype == SMAX_KERNEL_SPTRSM; }

void tri_plan(smax_kernel_s *k) {
    if (k->f_perm) {
        require(k->ctx != nullptr && k->ctx->n_levels > 0, SMAX_ERR_STATE,
                "level-scheduled solve needs the levels of generate_perm in the context");
        if (!k->tri_plan_valid || k->tri_levels_version != k->ctx->levels_version) {
            k->tri.release_graph();
            k->tri.build_given(k->ctx->lvl_ptr, k->dA.n_rows, k->f_upper, k->stream);
            k->tri_levels_version = k->ctx->levels_version;
            k->tri_plan_valid = true;
            ++k->tri_plan_serial;
        }
    } else if (!k->tri_plan_valid) {
        k->tri.release_graph();
        k->tri.build_own(k->dA, k->f_upper, k->stream);
        k->tri_plan_valid = true;
        ++k->tri_plan_serial;
    }
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

}  // namespace smax

namespace {

template <typename T> T *up(DevBuf &d, const void *h, uint64_t n, cudaStream_t st) {
    d.alloc(sizeof(T) * (n ? n : 1));
    if (n) SMAX_CUDA(cudaMemcpyAsync(d.p, h, sizeof(T) * n, cudaMemcpyHostToDevice, st));
    return d.as<T>();
}

// ------------------------------------------------------------------ SpMV --
void spmv_upload(smax_kernel_s *k) {
    cudaStream_t st = k->stream;
    if (k->f_scs) {
        const RegSCS &r = k->A_scs;
        require(r.set, SMAX_ERR_STATE, "register_A (SELL-C-sigma) before initialize");
        require(r.C > 0 && r.n_chunks * r.C == r.n_rows_padded && r.n_rows <= r.n_rows_padded, SMAX_ERR_BAD_ARG,
                "inconsistent SELL-C-sigma sizes");
        require(r.n_elements < (1ull << 31) && r.n_cols < (1ull << 31), SMAX_ERR_UNSUPPORTED,
                "int32 indices cannot address this matrix");
        DevSCS &d = k->dS;
        d.C = r.C; d.sigma = r.sigma; d.n_rows = r.n_rows; d.n_rows_padded = r.n_rows_padded;
        d.n_cols = r.n_cols; d.n_chunks = r.n_chunks; d.n_elements = r.n_elements; d.nnz = r.nnz;
        up<int>(d.chunk_ptr, r.chunk_ptr, r.n_chunks + 1, st);
        up<int>(d.chunk_len, r.chunk_lengths, r.n_chunks, st);
        up<int>(d.col, r.col, r.n_elements, st);
        d.val.alloc((size_t)k->vbytes * (r.n_elements ? r.n_elements : 1));
        if (r.n_elements)
            SMAX_CUDA(cudaMemcpyAsync(d.val.p, r.val, (size_t)k->vbytes * r.n_elements, cudaMemcpyHostToDevice, st));
        validate_scs(d, dstatus(k), st);
        read_status(k);
        scs_plan(d, k->vbytes, st);
    } else if (k->f_bcrs) {
        const RegBCRS &r = k->A_bcrs;
        require(r.set, SMAX_ERR_STATE, "register_A (BCRS) before initialize");
        require(r.hpad >= r.bh && r.wpad >= r.bw && r.hpad > 0 && r.wpad > 0, SMAX_ERR_BAD_ARG,
                "block paddings must be at least the block sizes");
        require(r.n_blocks < (1ull << 31) && r.n_rows < (1ull << 31), SMAX_ERR_UNSUPPORTED,
                "int32 indices cannot address this matrix");
        DevBCRS &d = k->dBc;
        d.n_rows = r.n_rows; d.n_cols = r.n_cols; d.n_blocks = r.n_blocks; d.bh = r.bh; d.bw = r.bw;
        d.hpad = r.hpad; d.wpad = r.wpad;
        up<int>(d.row_ptr, r.row_ptr, r.n_rows + 1, st);
        up<int>(d.col, r.col, r.n_blocks, st);
        const uint64_t nv = r.n_blocks * r.hpad * r.wpad;
        d.val.alloc((size_t)k->vbytes * (nv ? nv : 1));
        if (nv) SMAX_CUDA(cudaMemcpyAsync(d.val.p, r.val, (size_t)k->vbytes * nv, cudaMemcpyHostToDevice, st));
        validate_bcrs(d, dstatus(k), st);
        read_status(k);
        bcrs_plan(d, st);
    } else {
        require(k->A.set, SMAX_ERR_STATE, "register_A before initialize");
        upload_crs(k->dA, k->A, k->vbytes, st, crs_stream_pad());
        validate_crs(k->dA, dstatus(k), st);
        read_status(k);
        k->crs_plan = CrsTilePlan();
        k->crs_stream = CrsStreamPlan();
        if (k->spmv_variant == 2)
            k->crs_plan.build(k->dA.rp(), k->dA.n_rows, crs_default_cap(k->vbytes * 8), st);
        else
            k->crs_stream.build(k->dA.rp(), k->dA.n_rows, k->dA.nnz, k->vbytes, st);
    }
}

template <typename VT> void crs_spmv_any(smax_kernel_s *k, const VT *x, VT *y) {
    if (k->spmv_variant == 2)
        crs_spmv<VT>(k->crs_plan, k->dA.rp(), k->dA.ci(), k->dA.val.as<VT>(), x, y, k->stream);
    else
        crs_spmv_stream<VT>(k->crs_stream, k->dA.ci(), k->dA.val.as<VT>(), x, y, k->stream);
}

template <typename VT> void spmv_apply_t(smax_kernel_s *k, const VT *x, VT *y) {
    if (k->f_scs) {
        scs_spmv<VT>(k->dS, x, y, k->stream);
    } else if (k->f_bcrs) {
        k->dBc.col_major = k->f_block_col_major;
        bcrs_spmv<VT>(k->dBc, x, y, k->stream);
    } else {
        crs_spmv_any<VT>(k, x, y);
    }
}

// ------------------------------------------------------------------ SpMM --
void spmm_upload(smax_kernel_s *k) {
    require(k->A.set, SMAX_ERR_STATE, "register_A before initialize");
    upload_crs(k->dA, k->A, k->vbytes, k->stream, crs_stream_pad());
    validate_crs(k->dA, dstatus(k), k->stream);
    read_status(k);
    k->crs_stream = CrsStreamPlan();
    k->spmm_plan = SpmmPlan();  // its row ranges and staged tiles describe the previous matrix
    if (!k->f_row_major) k->crs_stream.build(k->dA.rp(), k->dA.n_rows, k->dA.nnz, k->vbytes, k->stream);
}

template <typename VT> void spmm_apply_t(smax_kernel_s *k, const VT *X, VT *Y) {
    const int64_t kk = (int64_t)(k->B.n_cols ? k->B.n_cols : 1);
    if (k->f_row_major) {
        crs_spmm_row_major<VT>(k->dA, kk, X, Y, k->stream, &k->spmm_plan, k->spmv_variant);
    } else {
        // column-major: the reference uses A's n_rows as the leading dimension
        // of both X and Y (src/kernels/spmm/spmm_cpu/spmm_cpu_crs_impl.hpp:29,44)
        const int64_t ld = k->dA.n_rows;
        for (int64_t v = 0; v < kk; ++v)
            crs_spmv_stream<VT>(k->crs_stream, k->dA.ci(), k->dA.val.as<VT>(), X + v * ld, Y + v * ld, k->stream);
    }
}

// ------------------------------------------------------- SpTRSV / SpTRSM --
// register_B is the solution x (X), register_C the right-hand side b (B)
// (src/kernels/sptrsv.hpp:40-58, sptrsm.hpp:40-60).

void tri_upload(smax_kernel_s *k) {
    require(k->A.set, SMAX_ERR_STATE, "register_A before initialize");
    require(k->A.n_rows == k->A.n_cols, SMAX_ERR_BAD_ARG, "triangular solves need a square matrix");
    cudaStream_t st = k->stream;
    upload_crs(k->dA, k->A, k->vbytes, st);
    validate_crs(k->dA, dstatus(k), st);
    read_status(k);
    peel_diag(k->dA, k->vbytes, k->D, dstatus(k), st);
    read_status(k);
    // the reference moves each diagonal entry to the end of its row in the
    // caller's arrays (sptrsv_cpu_core.hpp:21-38); mirror that
    if (k->A.nnz) {
        SMAX_CUDA(cudaMemcpyAsync(k->A.col, k->dA.col.p, sizeof(int) * k->A.nnz, cudaMemcpyDefault, st));
        SMAX_CUDA(cudaMemcpyAsync(k->A.val, k->dA.val.p, (size_t)k->vbytes * k->A.nnz, cudaMemcpyDefault, st));
    }
    SMAX_CUDA(cudaStreamSynchronize(st));
    k->tri_plan_valid = false;
}


template <typename VT> void tri_apply_t(smax_kernel_s *k, const VT *Bv, VT *Xv) {
    tri_plan(k);
    k->tri.set_allow_cluster(k->sweep_cluster);
    if constexpr (sizeof(VT) == 8) {
        if (k->refine_steps > 0) {
            require(k->ktype == SMAX_KERNEL_SPTRSV, SMAX_ERR_UNSUPPORTED,
                    "refinement is available for SpTRSV (one right-hand side)");
            refine_solve(k, Bv, Xv);
            return;
        }
    }
    const int64_t kk = k->ktype == SMAX_KERNEL_SPTRSM ? (int64_t)(k->B.n_cols ? k->B.n_cols : 1) : 1;
    const bool rm = k->ktype == SMAX_KERNEL_SPTRSM ? k->f_row_major : true;
    const int64_t ld = k->dA.n_rows;  // column-major blocks use A's n_rows (sptrsm_cpu_crs_impl.hpp:44-50)
    const int merge = tri_merge_rows(k);
    if (k->solve_mode == SMAX_SOLVE_PERSISTENT) {
        require(kk == 1, SMAX_ERR_UNSUPPORTED, "the persistent solve handles one right-hand side");
        tri_solve_persistent<VT>(k->tri, k->dA, k->D.as<VT>(), Bv, Xv, dstatus(k), k->persist_scratch,
                                 k->force_timeout, k->spin_limit, k->stream);
        return;
    }
    // the default runs sync-free (no barrier, no launch between levels) one
    // right-hand side over few wide levels, and blocks of k > 1 over many
    // narrow ones
    if (k->solve_mode == SMAX_SOLVE_SYNCFREE ||
        (k->solve_mode == SMAX_SOLVE_AUTO && syncfree_suits(k->tri, kk))) {
        if (tri_solve_syncfree<VT>(k->tri, k->dA, k->D.as<VT>(), Bv, Xv, k->vals_version, k->sf_ctl, k->spin_limit,
                                   k->force_timeout, dstatus(k), k->stream, kk, rm))
            return;
        // not applicable to this matrix or these operands: the merged solve
    }
    if (k->solve_mode == SMAX_SOLVE_AUTO || k->solve_mode == SMAX_SOLVE_GRAPH)
        tri_solve_graph<VT>(k->tri, k->dA, k->D.as<VT>(), Bv, Xv, kk, rm, ld, merge, k->vals_version, k->stream);
    else
        tri_solve<VT>(k->tri, k->dA, k->D.as<VT>(), Bv, Xv, kk, rm, ld, merge, k->vals_version, k->stream);
}

// ------------------------------------------------------------------ SpGEMM --
void spgemm_upload(smax_kernel_s *k) {
    require(k->A.set && k->Bm.set, SMAX_ERR_STATE, "register_A and register_B before initialize");
    require(k->A.n_cols == k->Bm.n_rows, SMAX_ERR_BAD_ARG, "A.n_cols must equal B.n_rows");
    upload_crs(k->dA, k->A, k->vbytes, k->stream);
    validate_crs(k->dA, dstatus(k), k->stream);
    read_status(k);
    upload_crs(k->dBm, k->Bm, k->vbytes, k->stream);
    validate_crs(k->dBm, dstatus(k), k->stream);
    read_status(k);
}

void spgemm_finalize(smax_kernel_s *k) {
    // the reference allocates C with new[] and hands it to the caller
    // (symbolic_phase_impl.hpp:132-151); so does this platform
    require(k->spgemm_done, SMAX_ERR_STATE, "apply before finalize");
    const DevCRS &c = k->dCm;
    int *rp = new int[c.n_rows + 1];
    int *col = new int[c.nnz > 0 ? c.nnz : 1];
    void *val = k->vbytes == 8 ? static_cast<void *>(new double[c.nnz > 0 ? c.nnz : 1])
                               : static_cast<void *>(new float[c.nnz > 0 ? c.nnz : 1]);
    SMAX_CUDA(cudaMemcpyAsync(rp, c.row_ptr.p, sizeof(int) * (c.n_rows + 1), cudaMemcpyDeviceToHost, k->stream));
    if (c.nnz) {
        SMAX_CUDA(cudaMemcpyAsync(col, c.col.p, sizeof(int) * c.nnz, cudaMemcpyDeviceToHost, k->stream));
        SMAX_CUDA(cudaMemcpyAsync(val, c.val.p, (size_t)k->vbytes * c.nnz, cudaMemcpyDeviceToHost, k->stream));
    }
    SMAX_CUDA(cudaStreamSynchronize(k->stream));
    *k->Cref.n_rows = (uint64_t)c.n_rows;
    *k->Cref.n_cols = (uint64_t)c.n_cols;
    *k->Cref.nnz = (uint64_t)c.nnz;
    *k->Cref.row_ptr = rp;
    *k->Cref.col = col;
    *k->Cref.val = val;
}


// Operand extents the kernel reads (B) and writes (C), in elements.
void check_extents(smax_kernel_s *k, uint64_t b_off, uint64_t c_off) {
    uint64_t need_b = 0, need_c = 0;
    switch (k->ktype) {
    case SMAX_KERNEL_SPMV:
        if (k->f_scs) { need_b = k->A_scs.n_cols; need_c = k->A_scs.n_rows_padded; }
        else if (k->f_bcrs) { need_b = k->A_bcrs.n_cols * k->A_bcrs.wpad; need_c = k->A_bcrs.n_rows * k->A_bcrs.hpad; }
        else { need_b = k->A.n_cols; need_c = k->A.n_rows; }
        break;
    case SMAX_KERNEL_SPMM: {
        const uint64_t kk = k->B.n_cols ? k->B.n_cols : 1;
        require(k->C.n_cols == k->B.n_cols, SMAX_ERR_BAD_ARG, "X and Y must have the same number of vectors");
        if (k->f_row_major) { need_b = k->A.n_cols * kk; need_c = k->A.n_rows * kk; }
        else { need_b = (kk - 1) * k->A.n_rows + k->A.n_cols; need_c = k->A.n_rows * kk; }
        break;
    }
    case SMAX_KERNEL_SPTRSV:
        need_b = k->A.n_rows;
        need_c = k->A.n_rows;
        break;
    case SMAX_KERNEL_SPTRSM: {
        const uint64_t kk = k->B.n_cols ? k->B.n_cols : 1;
        require(k->C.n_cols == k->B.n_cols, SMAX_ERR_BAD_ARG, "X and B must have the same number of vectors");
        need_b = k->A.n_rows * kk;
        need_c = k->A.n_rows * kk;
        break;
    }
    default: break;
    }
    require(b_off + need_b <= k->B.elems(), SMAX_ERR_BAD_ARG, "B (with offset) is smaller than the operator needs");
    require(c_off + need_c <= k->C.elems(), SMAX_ERR_BAD_ARG, "C (with offset) is smaller than the operator needs");
}

// ------------------------------------------- host-mode output download --
void record_out(smax_kernel_s *k, uint64_t off, uint64_t count) {
    // the same range written again: only its latest write is downloaded
    for (auto &r : k->out_ranges)
        if (r.off == off && r.count == count) {
            SMAX_CUDA(cudaEventRecord(r.ev, k->stream));
            return;
        }
    cudaEvent_t e;
    if (!k->ev_pool.empty()) {
        e = k->ev_pool.back();
        k->ev_pool.pop_back();
    } else {
        SMAX_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    }
    SMAX_CUDA(cudaEventRecord(e, k->stream));
    k->out_ranges.push_back({off, count, e});
}

// first element and element count of the output one apply writes
uint64_t out_offset(const smax_kernel_s *k, uint64_t b_off, uint64_t c_off) { return is_tri(k) ? b_off : c_off; }
uint64_t out_count(const smax_kernel_s *k) {
    const uint64_t kk = k->B.n_cols ? k->B.n_cols : 1;
    switch (k->ktype) {
    case SMAX_KERNEL_SPMV:
        if (k->f_scs) return k->A_scs.n_rows_padded;
        if (k->f_bcrs) return k->A_bcrs.n_rows * k->A_bcrs.hpad;
        return k->A.n_rows;
    case SMAX_KERNEL_SPMM: return k->A.n_rows * kk;
    case SMAX_KERNEL_SPTRSV: return k->A.n_rows;
    case SMAX_KERNEL_SPTRSM: return k->A.n_rows * kk;
    default: return 0;
    }
}

// CRS SpMV with the warp-stream kernel in host mode, large enough that the
// kernel time is worth hiding under the download of y: builds (once per
// upload) row blocks starting at entries that are multiples of 4 (the
// kernel's 16-byte loads), each with its own plan over the shared device copy.
// Block b holds about 2^b / (2^B - 1) of the entries: the first block is small,
// so y's download starts early, and each block computes in about the time
// the previous block's y takes to download (the kernel produces y about
// twice as fast as the host link takes it), so the link stays busy.
bool pipe_ready(smax_kernel_s *k) {
    if (k->ktype != SMAX_KERNEL_SPMV || k->f_scs || k->f_bcrs || k->spmv_variant == 2) return false;
    if (k->pipe_blocks < 2 || k->dA.n_rows < (1 << 18)) return false;
    auto &P = k->pipe;
    if (P.a_version == k->a_version) return P.blocks() > 0;
    P = smax_kernel_s::SpmvPipe();
    P.a_version = k->a_version;
    // the row blocks are cut on the host copy of row_ptr: A registered as
    // device arrays is not pipelined
    cudaPointerAttributes pa{};
    if (cudaPointerGetAttributes(&pa, k->A.row_ptr) != cudaSuccess) {
        (void)cudaGetLastError();
        return false;
    }
    if (pa.type == cudaMemoryTypeDevice || pa.type == cudaMemoryTypeManaged) return false;
    const int64_t n = k->dA.n_rows, nnz = k->dA.nnz;
    const int *rp = static_cast<const int *>(k->A.row_ptr);  // the registered host row pointer
    std::vector<int64_t> r0{0}, e0{0};
    const int nbk = std::min(k->pipe_blocks, 16);
    const double whole = (double)((1ll << nbk) - 1);
    for (int b = 1; b < nbk; ++b) {
        const int64_t target = (int64_t)((double)nnz * (double)((1ll << b) - 1) / whole);
        int64_t r = std::lower_bound(rp, rp + n + 1, (int)target) - rp;
        int64_t limit = std::min<int64_t>(n, r + 4096);
        while (r < limit && (rp[r] % 4) != 0) ++r;
        if (r >= limit || r <= r0.back() || rp[r] <= e0.back()) continue;
        r0.push_back(r);
        e0.push_back(rp[r]);
    }
    if (r0.size() < 2) return false;
    r0.push_back(n);
    e0.push_back(nnz);
    const int nb = (int)r0.size() - 1;
    P.plans.resize(nb);
    P.rps.resize(nb);
    for (int b = 0; b < nb; ++b) {
        const int64_t rows = r0[b + 1] - r0[b];
        std::vector<int> h(rows + 1);
        for (int64_t i = 0; i <= rows; ++i) h[i] = rp[r0[b] + i] - (int)e0[b];
        P.rps[b].alloc(sizeof(int) * (rows + 1));
        SMAX_CUDA(cudaMemcpyAsync(P.rps[b].p, h.data(), sizeof(int) * (rows + 1), cudaMemcpyHostToDevice, k->stream));
        P.plans[b].build(P.rps[b].as<int>(), rows, e0[b + 1] - e0[b], k->vbytes, k->stream);
    }
    P.r0 = std::move(r0);
    P.e0 = std::move(e0);
    return true;
}

template <typename VT> void apply_pipe_t(smax_kernel_s *k, const VT *x, VT *y, uint64_t c_off) {
    const auto &P = k->pipe;
    for (int b = 0; b < P.blocks(); ++b) {
        crs_spmv_stream<VT>(P.plans[b], k->dA.ci() + P.e0[b], k->dA.val.as<VT>() + P.e0[b], x, y + P.r0[b],
                            k->stream);
        record_out(k, c_off + (uint64_t)P.r0[b], (uint64_t)(P.r0[b + 1] - P.r0[b]));
    }
}

void apply_pipelined(smax_kernel_s *k, uint64_t b_off, uint64_t c_off) {
    const void *b = dev_b(k, b_off);
    void *c = dev_c(k, c_off);
    if (k->vbytes == 8) apply_pipe_t<double>(k, static_cast<const double *>(b), static_cast<double *>(c), c_off);
    else apply_pipe_t<float>(k, static_cast<const float *>(b), static_cast<float *>(c), c_off);
}

// wait: return only when x (and b) are on the device, as the reference's
// initialize does; run() does not wait, since its apply is ordered after the
// copies on the same stream and its finalize waits for the results
void do_initialize(smax_kernel_s *k, bool wait = true) {
    double t0 = wall_s();
    if (k->ktype == SMAX_KERNEL_SPGEMM) {
        require(k->Cref.set, SMAX_ERR_STATE, "register_C before initialize");
        if (k->a_dirty) {
            spgemm_upload(k);
            k->a_dirty = false;
            ++k->a_version;
            ++k->vals_version;
        }
        k->timers["initialize"] += wall_s() - t0;
        return;
    }
    require(k->B.set && k->C.set, SMAX_ERR_STATE, "register_B and register_C before initialize");
    if (k->a_dirty) {
        switch (k->ktype) {
        case SMAX_KERNEL_SPMV: spmv_upload(k); break;
        case SMAX_KERNEL_SPMM: spmm_upload(k); break;
        case SMAX_KERNEL_SPTRSV:
        case SMAX_KERNEL_SPTRSM: tri_upload(k); break;
        default: fail(SMAX_ERR_UNSUPPORTED, "kernel type not available in this build");
        }
        k->a_dirty = false;
        ++k->a_version;
        ++k->vals_version;
    }
    if (!k->f_device) {
        size_t bb = (size_t)k->B.elems() * k->vbytes, cb = (size_t)k->C.elems() * k->vbytes;
        k->dB.ensure(bb);
        k->dC.ensure(cb);
        // the kernel's input: B (x / X) for SpMV and SpMM; C (b / B) for
        // solves, and their X too (a solve reads the current x for entries
        // outside its triangle, as the reference's loops do)
        if (is_tri(k) && cb)
            SMAX_CUDA(cudaMemcpyAsync(k->dC.p, k->C.val, cb, cudaMemcpyHostToDevice, k->stream));
        if (bb) SMAX_CUDA(cudaMemcpyAsync(k->dB.p, k->B.val, bb, cudaMemcpyHostToDevice, k->stream));
    }
    if (wait) SMAX_CUDA(cudaStreamSynchronize(k->stream));
    k->timers["initialize"] += wall_s() - t0;
}

// The "apply" stopwatch: a pair of CUDA events around one apply, unless the
// kernel's timers are off (SMAX_FLAG_TIMERS).
struct ApplyStopwatch {
    std::optional<EventInterval> iv;
    explicit ApplyStopwatch(smax_kernel_s *k) {
        if (!k->timers_on) return;
        k->timers["apply"] += k->apply_events.trim(512);
        iv.emplace(k->apply_events, k->stream);
    }
    void close() {
        if (iv) iv->close();
    }
};

void do_apply(smax_kernel_s *k, uint64_t b_off, uint64_t c_off) {
    require(!k->a_dirty, SMAX_ERR_STATE, "initialize before apply");
    if (k->ktype == SMAX_KERNEL_SPGEMM) {
        // offsets are ignored, as in the reference (src/kernels/spgemm.hpp:108-130)
        ApplyStopwatch sw(k);
        SpgemmTimes *times = k->timers_on ? &k->spgemm_times : nullptr;
        if (k->vbytes == 8) spgemm<double>(k->dA, k->dBm, k->dCm, k->spgemm_work, times, k->stream);
        else spgemm<float>(k->dA, k->dBm, k->dCm, k->spgemm_work, times, k->stream);
        sw.close();
        if (times) {
            const SpgemmTimes &t = *times;
            k->timers["Symbolic_Setup"] += t.setup;
            k->timers["Fused_Gustavson"] += t.fused;
            k->timers["Alloc_C"] += t.alloc;
            k->timers["Compress"] += t.compress;
            k->timers["symbolic_phase"] += t.setup + t.alloc;
            k->timers["numerical_phase"] += t.fused + t.compress;
        }
        k->spgemm_done = true;
        return;
    }
    check_extents(k, b_off, c_off);
    ApplyStopwatch sw(k);
    if (!k->f_device && pipe_ready(k)) {
        apply_pipelined(k, b_off, c_off);  // records one output range per row block
    } else {
        apply_core(k, b_off, c_off);
        if (!k->f_device) record_out(k, out_offset(k, b_off, c_off), out_count(k));
    }
    sw.close();
}

}  // namespace

// The launches of one apply (no stopwatch events).
void smax::apply_core(smax_kernel_s *k, uint64_t b_off, uint64_t c_off) {
    const void *b = dev_b(k, b_off);
    void *c = dev_c(k, c_off);
    const bool f64 = k->vbytes == 8;
    switch (k->ktype) {
    case SMAX_KERNEL_SPMV:
        if (f64) spmv_apply_t<double>(k, static_cast<const double *>(b), static_cast<double *>(c));
        else spmv_apply_t<float>(k, static_cast<const float *>(b), static_cast<float *>(c));
        break;
    case SMAX_KERNEL_SPMM:
        if (f64) spmm_apply_t<double>(k, static_cast<const double *>(b), static_cast<double *>(c));
        else spmm_apply_t<float>(k, static_cast<const float *>(b), static_cast<float *>(c));
        break;
    case SMAX_KERNEL_SPTRSV:
    case SMAX_KERNEL_SPTRSM: {
        // solves read C (right-hand sides) and write B (solution)
        void *x = const_cast<void *>(b);
        const void *rhs = c;
        if (f64) tri_apply_t<double>(k, static_cast<const double *>(rhs), static_cast<double *>(x));
        else tri_apply_t<float>(k, static_cast<const float *>(rhs), static_cast<float *>(x));
        break;
    }
    default: fail(SMAX_ERR_UNSUPPORTED, "kernel type not available in this build");
    }
}

void smax::build_crs_plans(smax_kernel_s *k) {
    k->crs_plan = CrsTilePlan();
    k->crs_plan.build(k->dA.rp(), k->dA.n_rows, crs_default_cap(k->vbytes * 8), k->stream);
    k->crs_stream = CrsStreamPlan();
    k->crs_stream.build(k->dA.rp(), k->dA.n_rows, k->dA.nnz, k->vbytes, k->stream);
    SMAX_CUDA(cudaStreamSynchronize(k->stream));
}

namespace {

void do_finalize(smax_kernel_s *k) {
    double t0 = wall_s();
    if (k->ktype == SMAX_KERNEL_SPGEMM) {
        spgemm_finalize(k);
        k->timers["apply"] += k->apply_events.drain();
        k->timers["finalize"] += wall_s() - t0;
        return;
    }
    if (!k->f_device && !k->out_ranges.empty()) {
        // exactly the ranges apply() wrote, each as soon as it is complete
        if (!k->copy_stream)
            SMAX_CUDA(cudaStreamCreateWithFlags(&k->copy_stream, cudaStreamNonBlocking));
        const bool solve = is_tri(k);
        char *host = static_cast<char *>(solve ? k->B.val : k->C.val);
        const char *dev = static_cast<const char *>(solve ? k->dB.p : k->dC.p);
        const size_t vb = (size_t)k->vbytes;
        for (const auto &r : k->out_ranges) {
            SMAX_CUDA(cudaStreamWaitEvent(k->copy_stream, r.ev, 0));
            if (r.count)
                SMAX_CUDA(cudaMemcpyAsync(host + r.off * vb, dev + r.off * vb, r.count * vb, cudaMemcpyDeviceToHost,
                                          k->copy_stream));
        }
        // the status word is read while the output downloads: its copy waits
        // only for the kernels on the kernel's stream; an error is reported
        // once no download into the caller's memory is in flight
        const DevStatus st = k->status.p ? fetch_status(k) : DevStatus{};
        SMAX_CUDA(cudaStreamSynchronize(k->copy_stream));
        for (const auto &r : k->out_ranges) k->ev_pool.push_back(r.ev);
        k->out_ranges.clear();
        if (k->status.p) check_status(k, st);
    } else {
        SMAX_CUDA(cudaStreamSynchronize(k->stream));
        read_status(k);
    }
    k->timers["apply"] += k->apply_events.drain();
    k->timers["finalize"] += wall_s() - t0;
}

}  // namespace

extern "C" {

int smax_abi_version(void) { return SMAX_B200_ABI_VERSION; }

const char *smax_last_error(void) { return smax::last_error(); }

smax_status smax_test_fail_device_alloc(int64_t n) {
    if (n < 0) {
        smax::set_last_error("smax_test_fail_device_alloc: n must be >= 0");
        return SMAX_ERR_BAD_ARG;
    }
    smax::arm_device_alloc_failure(n);
    return SMAX_OK;
}

uint64_t smax_test_device_alloc_count(void) { return (uint64_t)smax::device_alloc_count(); }

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

smax_status smax_ctx_set_levels(smax_ctx ctx, int n_levels, const int *lvl_ptr) {
    return guarded([&] {
        require(ctx != nullptr, SMAX_ERR_BAD_ARG, "null context");
        require(n_levels >= 0 && (lvl_ptr != nullptr || n_levels == 0), SMAX_ERR_BAD_ARG, "bad level pointer");
        std::vector<int> lp(lvl_ptr, lvl_ptr + n_levels + 1);
        require(lp.empty() || lp[0] == 0, SMAX_ERR_BAD_ARG, "the level pointer must start at 0");
        for (int i = 1; i <= n_levels; ++i)
            require(lp[i] >= lp[i - 1], SMAX_ERR_BAD_ARG, "the level pointer must not decrease");
        ctx->lvl_ptr = std::move(lp);
        ctx->n_levels = n_levels;
        ctx->levels_version++;
    });
}

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
        case SMAX_FLAG_MAT_PERM:
            if (v != kk->f_perm) kk->tri_plan_valid = false;
            kk->f_perm = v;
            break;
        case SMAX_FLAG_MAT_UPPER_TRIANG:
            if (v != kk->f_upper) kk->tri_plan_valid = false;
            kk->f_upper = v;
            break;
        case SMAX_FLAG_MAT_LOWER_TRIANG: kk->f_lower = v; break;
        case SMAX_FLAG_VEC_ROW_MAJOR:
            if (v != kk->f_row_major) kk->a_dirty = true;
            kk->f_row_major = v;
            break;
        case SMAX_FLAG_MAT_SCS:
            if (v != kk->f_scs) kk->a_dirty = true;
            kk->f_scs = v;
            break;
        case SMAX_FLAG_MAT_BCRS:
            if (v != kk->f_bcrs) kk->a_dirty = true;
            kk->f_bcrs = v;
            break;
        case SMAX_FLAG_BLOCK_COLUMN_MAJOR: kk->f_block_col_major = v; break;
        case SMAX_FLAG_KERNEL_IMPL: kk->impl = value; break;
        case SMAX_FLAG_DEVICE_POINTERS: kk->f_device = v; break;
        case SMAX_FLAG_A_DIRTY: kk->a_dirty = kk->a_dirty || v; break;
        case SMAX_FLAG_SPMV_VARIANT:
            require(value >= 0 && value <= 2, SMAX_ERR_BAD_ARG, "SpMV variant must be 0, 1 or 2");
            if (value != kk->spmv_variant) kk->a_dirty = true;  // plans differ per variant
            kk->spmv_variant = value;
            break;
        case SMAX_FLAG_SPIN_LIMIT:
            require(value > 0, SMAX_ERR_BAD_ARG, "spin limit must be positive");
            kk->spin_limit = (long long)value * 1000;
            break;
        case SMAX_FLAG_TEST_FORCE_TIMEOUT: kk->force_timeout = v; break;
        case SMAX_FLAG_SOLVE_MODE:
            require(value >= SMAX_SOLVE_AUTO && value <= SMAX_SOLVE_SYNCFREE, SMAX_ERR_BAD_ARG,
                    "unknown solve mode");
            kk->solve_mode = value;
            break;
        case SMAX_FLAG_REFINE:
            require(value >= 0 && value <= 64, SMAX_ERR_BAD_ARG, "refinement steps must be in [0, 64]");
            require(value == 0 || kk->ftype == SMAX_FLOAT64, SMAX_ERR_UNSUPPORTED_TYPE,
                    "refinement needs a float64 kernel (the FP32 copy is made internally)");
            kk->refine_steps = value;
            break;
        case SMAX_FLAG_REFINE_TOL:
            require(value >= 0 && value <= 16, SMAX_ERR_BAD_ARG, "refinement tolerance exponent must be in [0, 16]");
            kk->refine_tol = value;
            break;
        case SMAX_FLAG_SWEEP_CLUSTER: kk->sweep_cluster = v; break;
        case SMAX_FLAG_TIMERS: kk->timers_on = v; break;
        case SMAX_FLAG_SPMV_PIPELINE:
            require(value >= 0 && value <= 64, SMAX_ERR_BAD_ARG, "pipeline blocks must be in [0, 64]");
            kk->pipe_blocks = value;
            kk->pipe.a_version = ~0ull;
            break;
        case SMAX_FLAG_LEVEL_MERGE:
            require(value >= 0, SMAX_ERR_BAD_ARG, "level merge threshold must be >= 0");
            kk->level_merge = value;
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

smax_status smax_kernel_register_A_scs(smax_kernel k, uint64_t C, uint64_t sigma, uint64_t n_rows,
                                       uint64_t n_rows_padded, uint64_t n_cols, uint64_t n_chunks,
                                       uint64_t n_elements, uint64_t nnz, void *chunk_ptr, void *chunk_lengths,
                                       void *col, void *val, void *perm) {
    return guarded([&] {
        smax_kernel_s *kk = K(k);
        require(chunk_ptr && chunk_lengths, SMAX_ERR_BAD_ARG, "null chunk_ptr/chunk_lengths");
        require(n_elements == 0 || (col && val), SMAX_ERR_BAD_ARG, "null col/val");
        kk->A_scs = RegSCS{true, C, sigma, n_rows, n_rows_padded, n_cols, n_chunks, n_elements, nnz,
                           chunk_ptr, chunk_lengths, col, val, perm};
        kk->a_dirty = true;
    });
}

smax_status smax_kernel_register_A_bcrs(smax_kernel k, uint64_t n_rows, uint64_t n_cols, uint64_t n_blocks,
                                        uint64_t b_height, uint64_t b_width, uint64_t height_pad,
                                        uint64_t width_pad, void *col, void *row_ptr, void *val) {
    return guarded([&] {
        smax_kernel_s *kk = K(k);
        require(row_ptr != nullptr, SMAX_ERR_BAD_ARG, "null row_ptr");
        require(n_blocks == 0 || (col && val), SMAX_ERR_BAD_ARG, "null col/val");
        kk->A_bcrs = RegBCRS{true, n_rows, n_cols, n_blocks, b_height, b_width, height_pad, width_pad,
                             col, row_ptr, val};
        kk->a_dirty = true;
    });
}

smax_status smax_kernel_register_B_crs(smax_kernel k, uint64_t n_rows, uint64_t n_cols, uint64_t nnz, void *col,
                                       void *row_ptr, void *val) {
    return guarded([&] {
        smax_kernel_s *kk = K(k);
        require(row_ptr != nullptr, SMAX_ERR_BAD_ARG, "null row_ptr");
        require(nnz == 0 || (col && val), SMAX_ERR_BAD_ARG, "null col/val");
        kk->Bm = RegCRS{true, n_rows, n_cols, nnz, col, row_ptr, val};
        kk->a_dirty = true;
    });
}

smax_status smax_kernel_register_C_crs_ref(smax_kernel k, uint64_t *n_rows, uint64_t *n_cols, uint64_t *nnz,
                                           void **col, void **row_ptr, void **val) {
    return guarded([&] {
        smax_kernel_s *kk = K(k);
        require(n_rows && n_cols && nnz && col && row_ptr && val, SMAX_ERR_BAD_ARG, "null output reference");
        kk->Cref = RegCRSRef{true, n_rows, n_cols, nnz, col, row_ptr, val};
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
        do_initialize(kk, false);
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

smax_status smax_kernel_swap_operands(smax_kernel k) {
    return guarded([&] {
        smax_kernel_s *kk = K(k);
        require(kk->ktype == SMAX_KERNEL_SPMV || kk->ktype == SMAX_KERNEL_SPMM, SMAX_ERR_UNSUPPORTED,
                "swap_operands not supported for this kernel");
        std::swap(kk->B, kk->C);
        std::swap(kk->dB, kk->dC);
    });
}

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
