// common.cuh -- shared runtime pieces of the sm_100a platform: status codes,
// error capture, RAII device buffers, launch helpers and cache-hinted loads.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <cstdio>
#include <stdexcept>
#include <string>
#include <utility>

#include "../../include/smax_b200.h"

namespace smax {

// ----------------------------------------------------------------- errors --
// Every exported function converts a thrown smax::Error into its status code
// and keeps the message for smax_last_error(); nothing on this platform calls
// exit() or traps (the reference's CUDA launchers exit on error,
// src/kernels/spmv/spmv_cuda/spmv_cuda_crs_impl.cu:38-45).
struct Error : std::runtime_error {
    int code;
    Error(int c, const std::string &m) : std::runtime_error(m), code(c) {}
};

void set_last_error(const std::string &m);
const char *last_error();

[[noreturn]] inline void fail(int code, const std::string &m) { throw Error(code, m); }

inline void cuda_check(cudaError_t e, const char *what) {
    if (e != cudaSuccess) {
        int code = (e == cudaErrorMemoryAllocation) ? SMAX_ERR_OOM : SMAX_ERR_CUDA;
        fail(code, std::string(what) + ": " + cudaGetErrorString(e));
    }
}

#define SMAX_CUDA(call) ::smax::cuda_check((call), #call)

template <typename F> int guarded(F &&f) {
    try {
        f();
        return SMAX_OK;
    } catch (const Error &e) {
        set_last_error(e.what());
        return e.code;
    } catch (const std::bad_alloc &) {
        set_last_error("host allocation failed");
        return SMAX_ERR_OOM;
    } catch (const std::exception &e) {
        set_last_error(e.what());
        return SMAX_ERR_BAD_ARG;
    } catch (...) {
        set_last_error("unknown error");
        return SMAX_ERR_BAD_ARG;
    }
}

// ------------------------------------------------- allocation accounting --
// Every device allocation of the platform goes through DevBuf::alloc, which
// counts it and asks this hook first.  When a test has armed it
// (smax_test_fail_device_alloc(n)), the n-th allocation from then on fails
// exactly as an out-of-memory cudaMalloc would (SMAX_ERR_OOM), without
// calling cudaMalloc, and the hook disarms itself.
bool device_alloc_should_fail();
void arm_device_alloc_failure(long long n);  // n >= 1: fail the n-th allocation from now; 0: off
long long device_alloc_count();

// --------------------------------------------------------- device buffers --
// Owning, move-only device allocation.  Size 0 allocates nothing.
struct DevBuf {
    void *p = nullptr;
    size_t bytes = 0;
    DevBuf() = default;
    explicit DevBuf(size_t b) { alloc(b); }
    DevBuf(const DevBuf &) = delete;
    DevBuf &operator=(const DevBuf &) = delete;
    DevBuf(DevBuf &&o) noexcept : p(o.p), bytes(o.bytes) { o.p = nullptr; o.bytes = 0; }
    DevBuf &operator=(DevBuf &&o) noexcept {
        if (this != &o) {
            release();
            p = o.p; bytes = o.bytes;
            o.p = nullptr; o.bytes = 0;
        }
        return *this;
    }
    ~DevBuf() { release(); }
    void alloc(size_t b) {
        release();
        if (b) {
            if (device_alloc_should_fail())
                fail(SMAX_ERR_OOM, "cudaMalloc of " + std::to_string(b) + " bytes failed (injected by the test hook)");
            cudaError_t e = cudaMalloc(&p, b);
            if (e != cudaSuccess) {
                p = nullptr;
                (void)cudaGetLastError();
                fail(SMAX_ERR_OOM, "cudaMalloc of " + std::to_string(b) + " bytes failed: " +
                                       cudaGetErrorString(e));
            }
        }
        bytes = b;
    }
    // grows (never shrinks) to at least b bytes; contents are not preserved
    void ensure(size_t b) {
        if (b > bytes) alloc(b);
    }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        bytes = 0;
    }
    template <typename T> T *as() const { return static_cast<T *>(p); }
};

inline unsigned ceil_div_u(uint64_t a, uint64_t b) { return (unsigned)((a + b - 1) / b); }

// number of SMs of the current device (148 on B200), cached per device
int sm_count();
int64_t l2_bytes();  // L2 capacity of the current device

// The legacy default stream (NULL / cudaStreamLegacy) and the per-thread
// default stream cannot be captured into a CUDA graph.
inline bool is_capturable(cudaStream_t s) {
    return s != nullptr && s != cudaStreamLegacy && s != cudaStreamPerThread;
}

// A private stream fenced to a caller's stream with events: work issued on it
// between enter() and leave() is ordered after everything queued on the
// caller's stream before enter() and before everything queued after leave().
struct AuxStream {
    cudaStream_t s = nullptr;
    cudaEvent_t in = nullptr, out = nullptr;
    cudaStream_t enter(cudaStream_t caller) {
        if (!s) {
            cuda_check(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking), "cudaStreamCreateWithFlags");
            cuda_check(cudaEventCreateWithFlags(&in, cudaEventDisableTiming), "cudaEventCreate");
            cuda_check(cudaEventCreateWithFlags(&out, cudaEventDisableTiming), "cudaEventCreate");
        }
        cuda_check(cudaEventRecord(in, caller), "cudaEventRecord");
        cuda_check(cudaStreamWaitEvent(s, in, 0), "cudaStreamWaitEvent");
        return s;
    }
    void leave(cudaStream_t caller) {
        cuda_check(cudaEventRecord(out, s), "cudaEventRecord");
        cuda_check(cudaStreamWaitEvent(caller, out, 0), "cudaStreamWaitEvent");
    }
    AuxStream() = default;
    AuxStream(const AuxStream &) = delete;
    AuxStream &operator=(const AuxStream &) = delete;
    ~AuxStream() {
        if (s) {
            cudaStreamSynchronize(s);
            cudaStreamDestroy(s);
        }
        if (in) cudaEventDestroy(in);
        if (out) cudaEventDestroy(out);
    }
};

// ----------------------------------------------------- cache-hinted loads --
// Matrix streams are read exactly once per product: load them with the
// streaming (evict-first) hint so they do not displace the gathered vector,
// which is re-read through L2 about nnz/n times per sweep.
template <typename T> __device__ __forceinline__ T ld_stream(const T *p) { return __ldcs(p); }
template <typename T> __device__ __forceinline__ T ld_keep(const T *p) { return __ldg(p); }
template <typename T> __device__ __forceinline__ void st_stream(T *p, T v) { __stcs(p, v); }

// Device-side error word: kernels record the first failure (code, index)
// instead of trapping; the host reads it after the stream is synchronised.
struct DevStatus {
    int code;
    int pad;
    long long index;
};

__device__ __forceinline__ void report(DevStatus *st, int code, long long index) {
    if (atomicCAS(&st->code, 0, code) == 0) st->index = index;
}

} // namespace smax
