// spgemm.cuh -- Gustavson SpGEMM C = A*B (spgemm.cu).
#pragma once

#include "spmv_formats.cuh"

namespace smax {

struct SpgemmTimes {
    double setup = 0, fused = 0, alloc = 0, compress = 0;  // seconds, CUDA events
    long long products = 0;                                // sum over rows of the product counts
};

// C's columns per row are in first-touch order and its values are summed in
// the reference's product order.
template <typename VT> void spgemm(const DevCRS &A, const DevCRS &B, DevCRS &C, SpgemmTimes *times, cudaStream_t st);

}  // namespace smax
