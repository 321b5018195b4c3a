// adjoint_abi.cu -- smax_kernel_adjoint and smax_kernel_update_A_values.
//
// The adjoint of an SpMV kernel is one warp-stream SpMV with the transposed
// copy A^T (built on the first call) plus a sampled outer product on A's
// pattern; the adjoint of an SpTRSV kernel is a triangular solve with L^T on
// the forward schedule's level sets swept in reverse, followed by the same
// outer product scaled by -1.  Kernels: adjoint.cu, sptrsv.cu.
#include "abi_internal.cuh"

using namespace smax;

namespace {

bool crs_spmv_kernel(const smax_kernel_s *k) { return k->ktype == SMAX_KERNEL_SPMV && !k->f_scs && !k->f_bcrs; }

// A caller operand on the device: the pointer itself with device pointers,
// otherwise a staging buffer, filled from the host for inputs.
void *stage(smax_kernel_s *k, int slot, const void *p, uint64_t n, bool input) {
    if (!p) return nullptr;
    if (k->f_device) return const_cast<void *>(p);
    DevBuf &b = k->adj_stage[slot];
    b.ensure((size_t)k->vbytes * (n ? n : 1));
    if (input && n) SMAX_CUDA(cudaMemcpyAsync(b.p, p, (size_t)k->vbytes * n, cudaMemcpyHostToDevice, k->stream));
    return b.p;
}

void ensure_adjoint(smax_kernel_s *k) {
    if (k->ktype == SMAX_KERNEL_SPMV) {
        if (k->adj_version != k->a_version) {
            build_transpose(k->dA, k->vbytes, false, true, k->adj, k->stream);
            k->adj_version = k->a_version;
        }
        return;
    }
    tri_plan(k);
    if (k->adj_version != k->a_version) {
        // L^T with each diagonal last in its row: the rows of L^T list L's
        // entries in descending row order for a lower L, ascending for upper
        build_transpose(k->dA, k->vbytes, !k->f_upper, false, k->adj, k->stream);
        check_diag_last(k->adj.at, dstatus(k), k->stream);
        read_status(k);
        k->adj_version = k->a_version;
    }
    if (k->adj_plan_serial != k->tri_plan_serial) {
        k->adj_plan.assign_reverse(k->tri, k->stream);
        k->adj_plan_serial = k->tri_plan_serial;
    }
    k->adj_plan.set_allow_cluster(k->sweep_cluster);
}

template <typename VT> void adjoint_t(smax_kernel_s *k, const VT *x, const VT *g, VT *din, VT *dval) {
    cudaStream_t st = k->stream;
    if (k->ktype == SMAX_KERNEL_SPMV) {
        if (din) crs_spmv_stream<VT>(k->adj.plan, k->adj.at.ci(), k->adj.at.val.as<VT>(), g, din, st);
        if (dval) sddmm_outer<VT>(k->dA, k->adj.row_of.as<int>(), VT(1), g, x, dval, st);
        return;
    }
    const int64_t n = k->dA.n_rows;
    VT *lam = din;
    if (!lam) {
        DevBuf &b = k->adj_stage[2];
        b.ensure(sizeof(VT) * (n ? n : 1));
        lam = b.as<VT>();
    }
    const int merge = tri_merge_rows(k);
    if (k->solve_mode == SMAX_SOLVE_AUTO || k->solve_mode == SMAX_SOLVE_GRAPH)
        tri_solve_graph<VT>(k->adj_plan, k->adj.at, k->D.as<VT>(), g, lam, 1, true, n, merge, k->vals_version, st);
    else
        tri_solve<VT>(k->adj_plan, k->adj.at, k->D.as<VT>(), g, lam, 1, true, n, merge, k->vals_version, st);
    if (dval) sddmm_outer<VT>(k->dA, k->adj.row_of.as<int>(), VT(-1), lam, x, dval, st);
}

}  // namespace

extern "C" {

smax_status smax_kernel_adjoint(smax_kernel k, const void *x, const void *g, void *d_in, void *d_val) {
    return guarded([&] {
        smax_kernel_s *kk = K(k);
        require(crs_spmv_kernel(kk) || kk->ktype == SMAX_KERNEL_SPTRSV, SMAX_ERR_UNSUPPORTED,
                "adjoints exist for CRS SpMV and SpTRSV kernels");
        require(!kk->a_dirty, SMAX_ERR_STATE, "initialize before adjoint");
        require(g != nullptr, SMAX_ERR_BAD_ARG, "null gradient");
        const bool spmv = kk->ktype == SMAX_KERNEL_SPMV;
        const uint64_t n_x = spmv ? kk->A.n_cols : kk->A.n_rows;
        const uint64_t n_g = kk->A.n_rows;
        const uint64_t nnz = kk->A.nnz;
        if (!x) require(kk->B.set && kk->B.elems() >= n_x, SMAX_ERR_STATE, "no x given and no registered B");
        ensure_adjoint(kk);
        const void *dx = x ? stage(kk, 0, x, n_x, true) : dev_b(kk, 0);
        const void *dg = stage(kk, 1, g, n_g, true);
        void *din = stage(kk, 2, d_in, n_x, false);
        void *dval = stage(kk, 3, d_val, nnz, false);
        if (kk->vbytes == 8)
            adjoint_t<double>(kk, static_cast<const double *>(dx), static_cast<const double *>(dg),
                              static_cast<double *>(din), static_cast<double *>(dval));
        else
            adjoint_t<float>(kk, static_cast<const float *>(dx), static_cast<const float *>(dg),
                             static_cast<float *>(din), static_cast<float *>(dval));
        SMAX_CUDA(cudaGetLastError());
        if (!kk->f_device) {
            if (d_in && n_x)
                SMAX_CUDA(cudaMemcpyAsync(d_in, din, (size_t)kk->vbytes * n_x, cudaMemcpyDeviceToHost, kk->stream));
            if (d_val && nnz)
                SMAX_CUDA(cudaMemcpyAsync(d_val, dval, (size_t)kk->vbytes * nnz, cudaMemcpyDeviceToHost, kk->stream));
            read_status(kk);  // synchronises
        }
    });
}

smax_status smax_kernel_update_A_values(smax_kernel k, const void *val) {
    return guarded([&] {
        smax_kernel_s *kk = K(k);
        require(crs_spmv_kernel(kk) || kk->ktype == SMAX_KERNEL_SPMM || is_tri(kk), SMAX_ERR_UNSUPPORTED,
                "value updates exist for CRS SpMV, SpMM, SpTRSV and SpTRSM kernels");
        require(!kk->a_dirty, SMAX_ERR_STATE, "initialize before updating values");
        const uint64_t nnz = (uint64_t)kk->dA.nnz;
        require(val != nullptr || nnz == 0, SMAX_ERR_BAD_ARG, "null values");
        if (nnz)
            SMAX_CUDA(cudaMemcpyAsync(kk->dA.val.p, val, (size_t)kk->vbytes * nnz,
                                      kk->f_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, kk->stream));
        if (is_tri(kk)) refresh_diag(kk->dA, kk->vbytes, kk->D, dstatus(kk), kk->stream);
        if (kk->adj_version == kk->a_version) refresh_transpose_values(kk->dA, kk->vbytes, kk->adj, kk->stream);
        ++kk->vals_version;
        // solves check the new diagonal; host sources must be consumed before returning
        if (is_tri(kk) || !kk->f_device) read_status(kk);
    });
}

}  // extern "C"
