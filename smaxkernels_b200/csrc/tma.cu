// tma.cu -- host side of tma.cuh: the gather tensor map of a dense vector.
//
// cuTensorMapEncodeTiled is a driver-API call; it is looked up once through
// the runtime (cudaGetDriverEntryPoint) so the library keeps linking the CUDA
// runtime only.
#include <mutex>

#include "tma.cuh"

namespace smax {

namespace {

using EncodeTiledFn = CUresult (*)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                   const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_fn() {
    static std::once_flag once;
    static EncodeTiledFn fn = nullptr;
    std::call_once(once, [] {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<EncodeTiledFn>(p);
        else
            (void)cudaGetLastError();
    });
    return fn;
}

}  // namespace

bool make_gather_map(CUtensorMap *map, const void *x, int64_t n, int vbytes) {
    if (vbytes != 4 && vbytes != 8) return false;
    const int rw = 32 / vbytes;  // elements per 32-byte row
    const int64_t rows = n / rw;
    if (rows < 1 || (reinterpret_cast<uintptr_t>(x) & 15u) != 0) return false;
    if (rows > (int64_t)0xFFFFFFFF) return false;
    EncodeTiledFn fn = encode_fn();
    if (!fn) return false;
    const cuuint64_t dims[2] = {(cuuint64_t)rw, (cuuint64_t)rows};
    const cuuint64_t strides[1] = {32};  // bytes between rows (a multiple of 16)
    const cuuint32_t box[2] = {(cuuint32_t)rw, 1};  // 32 bytes wide, one row high (tile::gather4)
    const cuuint32_t estride[2] = {1, 1};
    CUtensorMap m;
    const CUresult r = fn(&m, vbytes == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2,
                          const_cast<void *>(x), dims, strides, box, estride, CU_TENSOR_MAP_INTERLEAVE_NONE,
                          CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_NONE,
                          CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return false;
    *map = m;
    return true;
}

}  // namespace smax
