// spgemm.cuh -- Gustavson SpGEMM C = A*B (spgemm.cu).
#pragma once

#include "spmv_formats.cuh"

namespace smax {

struct SpgemmTimes {
    double setup = 0, fused = 0, alloc = 0, compress = 0;  // seconds, CUDA events
};

// Device workspace of the multiply, kept by the caller across applies: every
// buffer only grows, so repeated products of same-shaped matrices allocate
// nothing after the first.
struct SpgemmWork {
    DevBuf P, Poff, lists, counts, count, pcol, pval, scan_tmp;
    DevBuf wts, wsz, woff, wkeys, wfirst, wvals, wpos;
    DevBuf masks;              // merge path: each row's first-touch mask
    bool direct_hint = false;  // the last apply took the direct merge path
};

// C's columns per row are in first-touch order and its values are summed in
// the reference's product order.  C's buffers grow as needed and are reused.
template <typename VT>
void spgemm(const DevCRS &A, const DevCRS &B, DevCRS &C, SpgemmWork &w, SpgemmTimes *times, cudaStream_t st);

}  // namespace smax
