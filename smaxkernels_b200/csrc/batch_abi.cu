// batch_abi.cu -- exported batched SpTRSV (include/smax_b200.h).
#include "sptrsv_batch.cuh"

using namespace smax;

struct smax_batch_s {
    TriBatch tb;
};

extern "C" {

smax_status smax_batch_sptrsv_create(smax_batch *out, int float_type, int n_mats, const uint64_t *n_rows,
                                     const uint64_t *nnz, void *const *row_ptr, void *const *col, void *const *val) {
    return guarded([&] {
        if (!out || n_mats < 0 || (n_mats && (!n_rows || !nnz || !row_ptr || !col || !val)))
            fail(SMAX_ERR_BAD_ARG, "null argument");
        if (float_type != SMAX_FLOAT32 && float_type != SMAX_FLOAT64)
            fail(SMAX_ERR_UNSUPPORTED_TYPE, "value type must be float32 or float64");
        std::vector<RegCRS> mats(n_mats);
        for (int m = 0; m < n_mats; ++m) {
            if (!row_ptr[m] || (nnz[m] && (!col[m] || !val[m]))) fail(SMAX_ERR_BAD_ARG, "null matrix array");
            mats[m] = RegCRS{true, n_rows[m], n_rows[m], nnz[m], col[m], row_ptr[m], val[m]};
        }
        auto *b = new smax_batch_s();
        cudaStream_t st = nullptr;
        try {
            SMAX_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
            b->tb.build(float_type == SMAX_FLOAT64 ? 8 : 4, mats, st);
            SMAX_CUDA(cudaStreamDestroy(st));
        } catch (...) {
            if (st) cudaStreamDestroy(st);
            delete b;
            throw;
        }
        *out = b;
    });
}

smax_status smax_batch_sptrsv_solve(smax_batch b, const void *rhs, void *x, int mode, void *stream) {
    return guarded([&] {
        if (!b) fail(SMAX_ERR_BAD_ARG, "null batch");
        if (b->tb.n_rows && (!rhs || !x)) fail(SMAX_ERR_BAD_ARG, "null operand");
        cudaStream_t st = static_cast<cudaStream_t>(stream);
        const bool f64 = b->tb.vbytes == 8;
        switch (mode) {
        case SMAX_SOLVE_AUTO:
        case SMAX_SOLVE_GRAPH:
            if (f64) b->tb.solve_graph<double>(static_cast<const double *>(rhs), static_cast<double *>(x), st);
            else b->tb.solve_graph<float>(static_cast<const float *>(rhs), static_cast<float *>(x), st);
            break;
        case SMAX_SOLVE_MERGED:
            if (f64) b->tb.solve_persistent<double>(static_cast<const double *>(rhs), static_cast<double *>(x), st);
            else b->tb.solve_persistent<float>(static_cast<const float *>(rhs), static_cast<float *>(x), st);
            break;
        case SMAX_SOLVE_PER_LEVEL:
            if (f64) b->tb.solve_per_level<double>(static_cast<const double *>(rhs), static_cast<double *>(x), st);
            else b->tb.solve_per_level<float>(static_cast<const float *>(rhs), static_cast<float *>(x), st);
            break;
        default: fail(SMAX_ERR_BAD_ARG, "unknown batch solve mode");
        }
    });
}

uint64_t smax_batch_row_offset(smax_batch b, int m) {
    if (!b || m < 0 || m > b->tb.n_mats) return 0;
    return m == b->tb.n_mats ? (uint64_t)b->tb.n_rows : (uint64_t)b->tb.row_off[m];
}

smax_status smax_batch_info(smax_batch b, uint64_t *n_rows, int *total_levels, int *max_levels) {
    return guarded([&] {
        if (!b) fail(SMAX_ERR_BAD_ARG, "null batch");
        if (n_rows) *n_rows = (uint64_t)b->tb.n_rows;
        if (total_levels) *total_levels = b->tb.total_levels;
        if (max_levels) {
            int mx = 0;
            for (int l : b->tb.mat_levels) mx = l > mx ? l : mx;
            *max_levels = mx;
        }
    });
}

smax_status smax_batch_destroy(smax_batch b) {
    return guarded([&] { delete b; });
}

}  // extern "C"
