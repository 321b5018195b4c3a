// utils_abi.cu -- exported Utils entry points (format conversion; level sets
// and permutations live in levels_abi.cu).  They mirror SMAX::Utils
// (src/utils.hpp:12-87): host arrays in, new host arrays out, the work done on
// the GPU.  Returned arrays are allocated like the reference allocates them
// (new[] of the element type) and are released with delete[] or smax_free_host.
#include <new>

#include "kernel_obj.cuh"

using namespace smax;

namespace {

struct UtilStream {
    cudaStream_t s = nullptr;
    UtilStream() { SMAX_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking)); }
    ~UtilStream() {
        if (s) {
            cudaStreamSynchronize(s);
            cudaStreamDestroy(s);
        }
    }
};

struct UtilStatus {
    DevBuf buf;
    UtilStatus(cudaStream_t s) {
        buf.alloc(sizeof(DevStatus));
        SMAX_CUDA(cudaMemsetAsync(buf.p, 0, sizeof(DevStatus), s));
    }
    DevStatus *p() { return buf.as<DevStatus>(); }
    void check(cudaStream_t s) {
        DevStatus h{};
        SMAX_CUDA(cudaMemcpyAsync(&h, buf.p, sizeof(h), cudaMemcpyDeviceToHost, s));
        SMAX_CUDA(cudaStreamSynchronize(s));
        if (h.code) fail(h.code, "malformed input (code " + std::to_string(h.code) + " at index " +
                                     std::to_string(h.index) + ")");
    }
};

void check_types(int int_type, int float_type) {
    if (int_type != SMAX_INT32) fail(SMAX_ERR_UNSUPPORTED_TYPE, "only int32 indices are supported");
    if (float_type != SMAX_FLOAT32 && float_type != SMAX_FLOAT64)
        fail(SMAX_ERR_UNSUPPORTED_TYPE, "value type must be float32 or float64");
}

// new[] of the element size (operator new[] of the byte count, as new T[n]
// does for trivially destructible T)
void *host_new(size_t bytes) { return ::operator new[](bytes ? bytes : 1); }

void *download(const void *dev, size_t bytes, cudaStream_t s) {
    void *h = host_new(bytes);
    if (bytes) {
        cudaError_t e = cudaMemcpyAsync(h, dev, bytes, cudaMemcpyDeviceToHost, s);
        if (e != cudaSuccess) {
            ::operator delete[](h);
            cuda_check(e, "cudaMemcpyAsync");
        }
    }
    return h;
}

}  // namespace

extern "C" {

void smax_free_host(void *p) { ::operator delete[](p); }

smax_status smax_utils_convert_crs_to_scs(int int_type, int float_type, uint64_t n_rows, uint64_t n_cols,
                                          uint64_t nnz, const void *col, const void *row_ptr, const void *val,
                                          uint64_t C, uint64_t sigma, uint64_t *meta, void **chunk_ptr,
                                          void **chunk_lengths, void **col_out, void **val_out, void **perm) {
    return guarded([&] {
        check_types(int_type, float_type);
        if (!meta || !chunk_ptr || !chunk_lengths || !col_out || !val_out || !perm)
            fail(SMAX_ERR_BAD_ARG, "null output pointer");
        if (C == 0 || sigma == 0) fail(SMAX_ERR_BAD_ARG, "C and sigma must be positive");
        const int vbytes = float_type == SMAX_FLOAT64 ? 8 : 4;
        UtilStream us;
        UtilStatus ust(us.s);
        DevCRS a;
        upload_crs(a, RegCRS{true, n_rows, n_cols, nnz, const_cast<void *>(col), const_cast<void *>(row_ptr),
                             const_cast<void *>(val)},
                   vbytes, us.s);
        validate_crs(a, ust.p(), us.s);
        ust.check(us.s);
        DevSCS s;
        DevBuf dperm;
        crs_to_scs(a, vbytes, (int64_t)C, (int64_t)sigma, s, dperm, us.s);
        void *cp = download(s.chunk_ptr.p, sizeof(int) * (s.n_chunks + 1), us.s);
        void *cl = download(s.chunk_len.p, sizeof(int) * s.n_chunks, us.s);
        void *co = download(s.col.p, sizeof(int) * s.n_elements, us.s);
        void *vo = download(s.val.p, (size_t)vbytes * s.n_elements, us.s);
        void *pm = download(dperm.p, sizeof(int) * n_rows, us.s);
        SMAX_CUDA(cudaStreamSynchronize(us.s));
        meta[0] = s.n_rows;
        meta[1] = s.n_rows_padded;
        meta[2] = s.n_cols;
        meta[3] = s.n_chunks;
        meta[4] = s.n_elements;
        meta[5] = s.nnz;
        *chunk_ptr = cp;
        *chunk_lengths = cl;
        *col_out = co;
        *val_out = vo;
        *perm = pm;
    });
}

smax_status smax_utils_convert_crs_to_bcrs(int int_type, int float_type, uint64_t n_rows, uint64_t n_cols,
                                           uint64_t nnz, const void *col, const void *row_ptr, const void *val,
                                           uint64_t b_height, uint64_t b_width, uint64_t height_pad,
                                           uint64_t width_pad, int block_column_major, uint64_t *meta,
                                           void **col_out, void **row_ptr_out, void **val_out) {
    return guarded([&] {
        check_types(int_type, float_type);
        if (!meta || !col_out || !row_ptr_out || !val_out) fail(SMAX_ERR_BAD_ARG, "null output pointer");
        const int vbytes = float_type == SMAX_FLOAT64 ? 8 : 4;
        UtilStream us;
        UtilStatus ust(us.s);
        DevCRS a;
        upload_crs(a, RegCRS{true, n_rows, n_cols, nnz, const_cast<void *>(col), const_cast<void *>(row_ptr),
                             const_cast<void *>(val)},
                   vbytes, us.s);
        validate_crs(a, ust.p(), us.s);
        ust.check(us.s);
        DevBCRS b;
        crs_to_bcrs(a, vbytes, (int64_t)b_height, (int64_t)b_width, (int64_t)height_pad, (int64_t)width_pad,
                    block_column_major != 0, b, us.s);
        void *co = download(b.col.p, sizeof(int) * b.n_blocks, us.s);
        void *ro = download(b.row_ptr.p, sizeof(int) * (b.n_rows + 1), us.s);
        void *vo = download(b.val.p, (size_t)vbytes * b.n_blocks * b.hpad * b.wpad, us.s);
        SMAX_CUDA(cudaStreamSynchronize(us.s));
        meta[0] = b.n_rows;
        meta[1] = b.n_cols;
        meta[2] = b.n_blocks;
        meta[3] = b.bh;
        meta[4] = b.bw;
        meta[5] = b.hpad;
        meta[6] = b.wpad;
        *col_out = co;
        *row_ptr_out = ro;
        *val_out = vo;
    });
}

}  // extern "C"
