// tma.cuh -- tensor-memory-accelerator (TMA) pieces for the x gathers of the
// sparse kernels: a row-gather tensor map over a dense vector, mbarrier
// helpers with bounded waits, and the four-row gather load.
//
// The gather map views a vector x of n elements as a 2-D tensor of
// floor(n / RW) rows of RW = 32 / sizeof(VT) elements (one 32-byte L2 sector
// per row).  One `cp.async.bulk.tensor.2d ... tile::gather4` copies four such
// rows, chosen by four row indices, into 128 consecutive bytes of shared
// memory and signals an mbarrier with the byte count.  The rules this code
// keeps (checked on the host before any launch that uses a map):
//   * the base address is 16-byte aligned and the row stride (32 bytes) is a
//     multiple of 16 bytes;
//   * the box is RW elements wide (32 bytes, a multiple of 16) and one row
//     high, as tile::gather4 requires;
//   * the innermost coordinate of every copy is 0, so its byte offset is
//     always a multiple of 16;
//   * every shared-memory destination is 128-byte aligned;
//   * no multicast: every load reads this GPU's own memory into its own CTA.
// Elements past the last full row (n % RW of them) are not covered by the
// map; kernels read those through ordinary loads.
#pragma once

#include <cuda.h>

#include "common.cuh"

namespace smax {

// Builds the gather map of x (n elements of vbytes bytes).  Returns false,
// leaving the map untouched, when x is not 16-byte aligned or n < RW; the
// caller then uses its ordinary-load path.
bool make_gather_map(CUtensorMap *map, const void *x, int64_t n, int vbytes);

// rows of the gather map of an n-element vector
inline int64_t gather_rows(int64_t n, int vbytes) { return n / (32 / vbytes); }

// ------------------------------------------------------------ device side --
__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

// makes initialised mbarriers visible to the async (TMA) proxy
__device__ __forceinline__ void mbar_fence_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// orders this thread's earlier generic-proxy shared-memory accesses before
// later async-proxy (TMA) writes to the same bytes
__device__ __forceinline__ void fence_proxy_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.release.cta.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
                 "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.acquire.cta.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Waits for phase `parity` of bar to complete, at most `limit` polls (each
// try_wait itself blocks for a bounded, hardware-chosen time).  Returns false
// when the limit ran out.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, uint32_t parity, long long limit) {
    for (long long i = 0; i < limit; ++i)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}

// Copies rows r0..r3 of the gather map (32 bytes each) to dst (128-byte
// aligned shared memory, 128 bytes) and adds 128 bytes to bar's tx count.
__device__ __forceinline__ void tma_gather4(void *dst, const CUtensorMap *map, int r0, int r1, int r2, int r3,
                                            uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile::gather4.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3, %4, %5, %6}], [%7];" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(0), "r"(r0), "r"(r1), "r"(r2), "r"(r3), "r"(smem_u32(bar))
        : "memory");
}

}  // namespace smax
