// kernel_obj.cuh -- the C ABI's context and kernel objects.
//
// A smax_kernel_s holds what the reference keeps in a registered SMAX::Kernel
// (KernelContext, Args, Flags, Timers: src/kernel.hpp:7-127,
// src/kernels/<k>/<k>_common.hpp) plus this platform's device-resident state:
// the matrix is uploaded once and kept in HBM across run() calls, and every
// launch goes to the kernel's own stream.
#pragma once

#include <map>
#include <memory>
#include <string>
#include <vector>

#include "common.cuh"
#include "spmv_crs.cuh"

struct smax_ctx_s {
    // UtilitiesContainer (src/common.hpp:187-195): written by generate_perm,
    // read by level-scheduled SpTRSV/SpTRSM kernels.
    int n_levels = 0;
    std::vector<int> lvl_ptr;
    uint64_t levels_version = 0;  // bumped whenever the level sets change
};

namespace smax {

struct RegCRS {
    bool set = false;
    uint64_t n_rows = 0, n_cols = 0, nnz = 0;
    void *col = nullptr, *row_ptr = nullptr, *val = nullptr;
};

struct RegDense {
    bool set = false;
    uint64_t n_rows = 0, n_cols = 0;
    void *val = nullptr;
    uint64_t elems() const { return n_rows * (n_cols ? n_cols : 1); }
};

// Device copy of a CRS matrix (int32 indices).
struct DevCRS {
    int64_t n_rows = 0, n_cols = 0, nnz = 0;
    DevBuf row_ptr, col, val;
    // pad: col/val are allocated and zero-filled up to a multiple of `pad` entries
    void upload(const RegCRS &r, int vbytes, cudaStream_t st, int64_t pad = 1);
    const int *rp() const { return row_ptr.as<int>(); }
    const int *ci() const { return col.as<int>(); }
};

void validate_crs(const DevCRS &m, DevStatus *st, cudaStream_t s);

struct PendingEvents {
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> live, spare;
    std::pair<cudaEvent_t, cudaEvent_t> acquire();
    double drain();  // waits for and sums all live intervals (seconds)
    ~PendingEvents();
};

}  // namespace smax

struct smax_kernel_s {
    smax_ctx ctx = nullptr;
    int ktype = 0, itype = 0, ftype = 0;
    int vbytes = 8;

    // Flags (src/kernels/*/..._common.hpp "struct Flags")
    bool f_perm = false, f_upper = false, f_lower = false, f_row_major = false;
    bool f_scs = false, f_bcrs = false, f_block_col_major = false, f_device = false;
    int impl = 0;

    // Args as registered (host pointers unless f_device for B/C)
    smax::RegCRS A;
    smax::RegDense B, C;
    bool a_dirty = true;

    // device state
    cudaStream_t stream = nullptr;      // current stream (own or the caller's)
    cudaStream_t own_stream = nullptr;  // created with the kernel
    smax::DevCRS dA;
    smax::DevBuf dB, dC;
    smax::CrsTilePlan crs_plan;
    smax::CrsStreamPlan crs_stream;
    int spmv_variant = 0;  // 0 auto, 1 warp-stream, 2 row-tile
    smax::DevBuf status;  // smax::DevStatus

    // stopwatches
    std::map<std::string, double> timers;
    smax::PendingEvents apply_events;

    ~smax_kernel_s();
};
