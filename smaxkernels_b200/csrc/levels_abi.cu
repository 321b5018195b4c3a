// levels_abi.cu -- exported level-set and permutation utilities (SMAX::Utils,
// src/utils/permutations.hpp), computed on the GPU from host arrays.
#include <cstring>
#include <string>

#include "kernel_obj.cuh"
#include "levels.cuh"

using namespace smax;

namespace {

struct Stream {
    cudaStream_t s = nullptr;
    Stream() { SMAX_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking)); }
    ~Stream() {
        if (s) {
            cudaStreamSynchronize(s);
            cudaStreamDestroy(s);
        }
    }
};

// Uploads a CRS pattern (values optional) and validates it; square matrices only.
void upload_pattern(DevCRS &a, uint64_t n, const void *row_ptr, const void *col, const void *val, int vbytes,
                    cudaStream_t s) {
    RegCRS r{true, n, n, 0, const_cast<void *>(col), const_cast<void *>(row_ptr), const_cast<void *>(val)};
    int nnz = 0;
    if (n > 0) std::memcpy(&nnz, static_cast<const int *>(row_ptr) + n, sizeof(int));
    if (nnz < 0) fail(SMAX_ERR_BAD_ARG, "row_ptr[n] is negative");
    r.nnz = (uint64_t)nnz;
    upload_crs(a, r, vbytes, s);  // val == nullptr: pattern only
    DevBuf st(sizeof(DevStatus));
    SMAX_CUDA(cudaMemsetAsync(st.p, 0, sizeof(DevStatus), s));
    validate_crs(a, st.as<DevStatus>(), s);
    DevStatus h{};
    SMAX_CUDA(cudaMemcpyAsync(&h, st.p, sizeof(h), cudaMemcpyDeviceToHost, s));
    SMAX_CUDA(cudaStreamSynchronize(s));
    if (h.code) fail(h.code, "malformed CRS pattern (code " + std::to_string(h.code) + " at index " +
                                 std::to_string(h.index) + ")");
}

void *host_new(size_t bytes) { return ::operator new[](bytes ? bytes : 1); }

}  // namespace

extern "C" {

smax_status smax_utils_build_symmetric_crs(int int_type, uint64_t n_rows, const void *row_ptr, const void *col,
                                           void **sym_row_ptr, void **sym_col, uint64_t *sym_nnz) {
    return guarded([&] {
        if (int_type != SMAX_INT32) fail(SMAX_ERR_UNSUPPORTED_TYPE, "only int32 indices are supported");
        if (!row_ptr || !sym_row_ptr || !sym_col || !sym_nnz) fail(SMAX_ERR_BAD_ARG, "null argument");
        Stream s;
        DevCRS a;
        upload_pattern(a, n_rows, row_ptr, col, nullptr, 4, s.s);
        DevBuf srp, scol;
        int64_t snnz = 0;
        build_symmetric(a, srp, scol, snnz, s.s);
        void *hr = host_new(sizeof(int) * (n_rows + 1));
        void *hc = host_new(sizeof(int) * snnz);
        SMAX_CUDA(cudaMemcpyAsync(hr, srp.p, sizeof(int) * (n_rows + 1), cudaMemcpyDeviceToHost, s.s));
        if (snnz) SMAX_CUDA(cudaMemcpyAsync(hc, scol.p, sizeof(int) * snnz, cudaMemcpyDeviceToHost, s.s));
        SMAX_CUDA(cudaStreamSynchronize(s.s));
        *sym_row_ptr = hr;
        *sym_col = hc;
        *sym_nnz = (uint64_t)snnz;
    });
}

smax_status smax_utils_generate_perm(smax_ctx ctx, int int_type, uint64_t n_rows, const void *row_ptr,
                                     const void *col, int *perm, int *inv_perm, const char *type) {
    return guarded([&] {
        if (int_type != SMAX_INT32) fail(SMAX_ERR_UNSUPPORTED_TYPE, "only int32 indices are supported");
        if (!ctx || !row_ptr || (n_rows && (!perm || !inv_perm)) || !type) fail(SMAX_ERR_BAD_ARG, "null argument");
        const std::string t(type);
        const bool colouring = t == "SC" || t == "PC" || t == "PC_BAL";
        if (t != "BFS" && t != "RS" && t != "NONE" && !colouring)
            fail(SMAX_ERR_BAD_ARG, "Permutation type: " + t + " does not exist. Please choose a type in: BFS, RS, "
                                   "SC, PC, PC_BAL, NONE.");
        if (n_rows >= (1ull << 31)) fail(SMAX_ERR_UNSUPPORTED, "int32 indices cannot address this matrix");
        const int64_t n = (int64_t)n_rows;
        Stream s;
        std::vector<int> lvl_ptr;
        DevBuf dperm(sizeof(int) * (n ? n : 1)), dinv(sizeof(int) * (n ? n : 1));
        if (t == "NONE") {
            std::vector<int> id(n);
            for (int64_t i = 0; i < n; ++i) id[i] = (int)i;
            lvl_ptr.resize(n + 1);
            for (int64_t i = 0; i <= n; ++i) lvl_ptr[i] = (int)i;
            if (n) std::memcpy(perm, id.data(), sizeof(int) * n);
            if (n) std::memcpy(inv_perm, id.data(), sizeof(int) * n);
        } else {
            DevCRS a;
            upload_pattern(a, n_rows, row_ptr, col, nullptr, 4, s.s);
            DevBuf srp, scol, lvl, order;
            int64_t snnz = 0;
            build_symmetric(a, srp, scol, snnz, s.s);
            int nl = 0;
            if (t == "SC") {
                nl = colour_sc(srp.as<int>(), scol.as<int>(), n, lvl, s.s);
            } else if (colouring) {
                nl = colour_pc(srp.as<int>(), scol.as<int>(), n, lvl, s.s);
                if (t == "PC_BAL") nl = colour_balance(srp.as<int>(), scol.as<int>(), n, lvl, nl, s.s);
            } else {
                nl = rs_levels(srp.as<int>(), scol.as<int>(), n, lvl, s.s);
            }
            // every type but BFS: the identity stably sorted by level (colour)
            level_order(lvl.as<int>(), n, nl, order, lvl_ptr, s.s);
            if (n > 0 && lvl_ptr.back() != n) fail(SMAX_ERR_STATE, "level sweep did not reach every row");
            const int *p = order.as<int>();
            if (t == "BFS") {
                bfs_order(srp.as<int>(), scol.as<int>(), n, lvl_ptr, order.as<int>(), dperm, s.s);
                p = dperm.as<int>();
            }
            inverse_perm(p, n, dinv.as<int>(), s.s);
            if (n) SMAX_CUDA(cudaMemcpyAsync(perm, p, sizeof(int) * n, cudaMemcpyDeviceToHost, s.s));
            if (n) SMAX_CUDA(cudaMemcpyAsync(inv_perm, dinv.p, sizeof(int) * n, cudaMemcpyDeviceToHost, s.s));
            SMAX_CUDA(cudaStreamSynchronize(s.s));
        }
        ctx->lvl_ptr = std::move(lvl_ptr);
        ctx->n_levels = (int)ctx->lvl_ptr.size() - 1;
        ctx->levels_version++;
    });
}

smax_status smax_utils_sanity_check_perm(int int_type, uint64_t n_rows, const void *row_ptr, const void *col,
                                         const int *colors, int *valid, int64_t *first_bad_row) {
    return guarded([&] {
        if (int_type != SMAX_INT32) fail(SMAX_ERR_UNSUPPORTED_TYPE, "only int32 indices are supported");
        if (!row_ptr || !valid || (n_rows && !colors)) fail(SMAX_ERR_BAD_ARG, "null argument");
        const int64_t n = (int64_t)n_rows;
        Stream s;
        DevCRS a;
        upload_pattern(a, n_rows, row_ptr, col, nullptr, 4, s.s);
        DevBuf dc(sizeof(int) * (n ? n : 1));
        if (n) SMAX_CUDA(cudaMemcpyAsync(dc.p, colors, sizeof(int) * n, cudaMemcpyHostToDevice, s.s));
        int64_t bad = -1;
        *valid = colours_valid(a.rp(), a.ci(), n, dc.as<int>(), &bad, s.s) ? 1 : 0;
        if (first_bad_row) *first_bad_row = bad;
    });
}

smax_status smax_utils_apply_mat_perm(int int_type, int float_type, uint64_t n_rows, const void *row_ptr,
                                      const void *col, const void *val, void *perm_row_ptr, void *perm_col,
                                      void *perm_val, const int *perm, const int *inv_perm) {
    return guarded([&] {
        if (int_type != SMAX_INT32) fail(SMAX_ERR_UNSUPPORTED_TYPE, "only int32 indices are supported");
        if (float_type != SMAX_FLOAT32 && float_type != SMAX_FLOAT64)
            fail(SMAX_ERR_UNSUPPORTED_TYPE, "value type must be float32 or float64");
        if (!row_ptr || !perm_row_ptr || (n_rows && (!perm || !inv_perm))) fail(SMAX_ERR_BAD_ARG, "null argument");
        const int vbytes = float_type == SMAX_FLOAT64 ? 8 : 4;
        const int64_t n = (int64_t)n_rows;
        for (int64_t i = 0; i < n; ++i)
            if (perm[i] < 0 || perm[i] >= n || inv_perm[i] < 0 || inv_perm[i] >= n)
                fail(SMAX_ERR_BAD_ARG, "perm / inv_perm entry out of range");
        Stream s;
        DevCRS a;
        upload_pattern(a, n_rows, row_ptr, col, val, vbytes, s.s);
        DevBuf dp(sizeof(int) * (n ? n : 1)), di(sizeof(int) * (n ? n : 1));
        if (n) {
            SMAX_CUDA(cudaMemcpyAsync(dp.p, perm, sizeof(int) * n, cudaMemcpyHostToDevice, s.s));
            SMAX_CUDA(cudaMemcpyAsync(di.p, inv_perm, sizeof(int) * n, cudaMemcpyHostToDevice, s.s));
        }
        DevCRS out;
        apply_mat_perm(a, dp.as<int>(), di.as<int>(), vbytes, out, s.s);
        SMAX_CUDA(cudaMemcpyAsync(perm_row_ptr, out.row_ptr.p, sizeof(int) * (n + 1), cudaMemcpyDeviceToHost, s.s));
        if (a.nnz) {
            SMAX_CUDA(cudaMemcpyAsync(perm_col, out.col.p, sizeof(int) * a.nnz, cudaMemcpyDeviceToHost, s.s));
            SMAX_CUDA(cudaMemcpyAsync(perm_val, out.val.p, (size_t)vbytes * a.nnz, cudaMemcpyDeviceToHost, s.s));
        }
        SMAX_CUDA(cudaStreamSynchronize(s.s));
    });
}

smax_status smax_utils_apply_vec_perm(int float_type, uint64_t n_rows, const void *vec, void *vec_perm,
                                      const int *perm) {
    return guarded([&] {
        if (float_type != SMAX_FLOAT32 && float_type != SMAX_FLOAT64)
            fail(SMAX_ERR_UNSUPPORTED_TYPE, "value type must be float32 or float64");
        const int vbytes = float_type == SMAX_FLOAT64 ? 8 : 4;
        const int64_t n = (int64_t)n_rows;
        if (n == 0) return;
        if (!vec || !vec_perm || !perm) fail(SMAX_ERR_BAD_ARG, "null argument");
        Stream s;
        DevBuf dv((size_t)vbytes * n), dp(sizeof(int) * n), dout((size_t)vbytes * n), st(sizeof(DevStatus));
        SMAX_CUDA(cudaMemcpyAsync(dv.p, vec, (size_t)vbytes * n, cudaMemcpyHostToDevice, s.s));
        SMAX_CUDA(cudaMemcpyAsync(dp.p, perm, sizeof(int) * n, cudaMemcpyHostToDevice, s.s));
        for (int64_t i = 0; i < n; ++i)
            if (perm[i] < 0 || perm[i] >= n) fail(SMAX_ERR_BAD_ARG, "perm entry out of range");
        apply_vec_perm(dv.p, dp.as<int>(), n, vbytes, dout.p, s.s);
        SMAX_CUDA(cudaMemcpyAsync(vec_perm, dout.p, (size_t)vbytes * n, cudaMemcpyDeviceToHost, s.s));
        SMAX_CUDA(cudaStreamSynchronize(s.s));
    });
}

}  // extern "C"
