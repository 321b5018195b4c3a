// kernel_obj.cuh -- the C ABI's context and kernel objects.
//
// A smax_kernel_s holds what the reference keeps in a registered SMAX::Kernel
// (KernelContext, Args, Flags, Timers: src/kernel.hpp:7-127,
// src/kernels/<k>/<k>_common.hpp) plus this platform's device-resident state:
// the matrix is uploaded once and kept in HBM across run() calls, and every
// launch goes to the kernel's stream.
#pragma once

#include <map>
#include <memory>
#include <string>
#include <vector>

#include "common.cuh"
#include "spmv_crs.cuh"
#include "spmv_formats.cuh"
#include "spgemm.cuh"
#include "sptrsv.cuh"
#include "adjoint.cuh"
#include "refine.cuh"

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

// register_A with 13 SELL-C-sigma arguments (src/kernels/spmv.hpp:25-53)
struct RegSCS {
    bool set = false;
    uint64_t C = 0, sigma = 0, n_rows = 0, n_rows_padded = 0, n_cols = 0, n_chunks = 0, n_elements = 0, nnz = 0;
    void *chunk_ptr = nullptr, *chunk_lengths = nullptr, *col = nullptr, *val = nullptr, *perm = nullptr;
};

// register_A with 10 BCRS arguments (src/kernels/spmv.hpp:54-76)
struct RegBCRS {
    bool set = false;
    uint64_t n_rows = 0, n_cols = 0, n_blocks = 0, bh = 0, bw = 0, hpad = 0, wpad = 0;
    void *col = nullptr, *row_ptr = nullptr, *val = nullptr;
};

// register_C of SpGEMM: where the result's sizes and arrays are written
// (src/kernels/spgemm.hpp:68-83)
struct RegCRSRef {
    bool set = false;
    uint64_t *n_rows = nullptr, *n_cols = nullptr, *nnz = nullptr;
    void **col = nullptr, **row_ptr = nullptr, **val = nullptr;
};

struct RegDense {
    bool set = false;
    uint64_t n_rows = 0, n_cols = 0;
    void *val = nullptr;
    uint64_t elems() const { return n_rows * (n_cols ? n_cols : 1); }
};

// pad: col/val are allocated and zero-filled up to a multiple of `pad` entries
void upload_crs(DevCRS &d, const RegCRS &r, int vbytes, cudaStream_t st, int64_t pad = 1);
void validate_crs(const DevCRS &m, DevStatus *st, cudaStream_t s);

struct PendingEvents {
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> live, spare;
    std::pair<cudaEvent_t, cudaEvent_t> acquire();
    double drain();  // waits for and sums all live intervals (seconds)
    // sums and recycles all but the newest `keep` intervals once more than
    // 2*keep are live (bounds the event count of long apply() loops)
    double trim(size_t keep);
    // returns an acquired interval to the spare list unsummed (its end event
    // was never recorded: the timed work threw)
    void drop(std::pair<cudaEvent_t, cudaEvent_t> p);
    ~PendingEvents();
};

// One stopwatch interval around a block of launches on `s`: the start event
// is recorded on construction, the end event by close().  If the block
// throws before close(), the interval is dropped, so a later drain() never
// reads an event that was not recorded.
struct EventInterval {
    PendingEvents &pe;
    cudaStream_t s;
    std::pair<cudaEvent_t, cudaEvent_t> ev;
    bool closed = false;
    EventInterval(PendingEvents &p, cudaStream_t st) : pe(p), s(st), ev(p.acquire()) {
        const cudaError_t e = cudaEventRecord(ev.first, s);
        if (e != cudaSuccess) {
            pe.drop(ev);
            cuda_check(e, "cudaEventRecord(interval start)");
        }
    }
    void close() {
        SMAX_CUDA(cudaEventRecord(ev.second, s));
        closed = true;
    }
    ~EventInterval() {
        if (!closed) pe.drop(ev);
    }
    EventInterval(const EventInterval &) = delete;
    EventInterval &operator=(const EventInterval &) = delete;
};

double wall_s();

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
    smax::RegSCS A_scs;
    smax::RegBCRS A_bcrs;
    smax::RegDense B, C;
    smax::RegCRS Bm;       // SpGEMM's B
    smax::RegCRSRef Cref;  // SpGEMM's C
    bool a_dirty = true;

    // device state
    cudaStream_t stream = nullptr;      // current stream (own or the caller's)
    cudaStream_t own_stream = nullptr;  // created with the kernel
    smax::DevCRS dA;
    smax::DevSCS dS;
    smax::DevBCRS dBc;
    smax::DevBuf dB, dC;
    smax::CrsTilePlan crs_plan;
    smax::CrsStreamPlan crs_stream;
    smax::SpmmPlan spmm_plan;  // row ranges of the row-major SpMM walk
    int spmv_variant = 0;  // 0 auto, 1 warp-stream, 2 row-tile
    smax::DevBuf status;   // smax::DevStatus

    // SpGEMM
    smax::DevCRS dBm, dCm;
    smax::SpgemmTimes spgemm_times;
    smax::SpgemmWork spgemm_work;
    bool spgemm_done = false;

    // triangular solves (SpTRSV / SpTRSM)
    smax::DevBuf D;                 // peeled diagonal
    smax::TriPlan tri;
    bool tri_plan_valid = false;
    uint64_t tri_plan_serial = 0;   // bumped whenever tri is rebuilt
    uint64_t tri_levels_version = 0;
    int solve_mode = 0;             // SMAX_SOLVE_*
    int level_merge = -1;           // rows*k of levels merged into one-CTA runs; -1 = default
    bool force_timeout = false;     // test knob of the persistent solve's grid barrier
    long long spin_limit = 20000000; // polls before a grid barrier gives up
    smax::DevBuf persist_scratch;
    smax::DevBuf sf_ctl;  // task counter, abort flag of the sync-free solve

    // versions of the device copy of A: pattern + values (each upload), values
    // alone (each upload or value update)
    uint64_t a_version = 0, vals_version = 0;

    // reverse mode (adjoint_abi.cu): A^T or L^T and the reversed level plan
    smax::DevTranspose adj;
    smax::TriPlan adj_plan;
    uint64_t adj_version = ~0ull, adj_plan_serial = ~0ull;
    smax::DevBuf adj_stage[4];      // device staging of host operands (x, g, d_in, d_val)

    // FP32 solve + FP64 residual refinement (refine.cu); 0 steps = off
    int refine_steps = 0, refine_tol = 0;
    bool sweep_cluster = false;     // allow cluster runs in the level-pack solves
    bool timers_on = true;          // SMAX_FLAG_TIMERS: CUDA-event stopwatches around every apply
    smax::RefineState refine;

    // host-pointer mode: output ranges written by apply() since the last
    // finalize(), each with the event after which it is complete; finalize
    // downloads exactly these on copy_stream
    struct OutRange {
        uint64_t off, count;
        cudaEvent_t ev;
    };
    std::vector<OutRange> out_ranges;
    std::vector<cudaEvent_t> ev_pool;
    cudaStream_t copy_stream = nullptr;

    // CRS SpMV in host-pointer mode: row blocks whose results are downloaded
    // while later blocks still compute (built on first use)
    struct SpmvPipe {
        uint64_t a_version = ~0ull;
        std::vector<int64_t> r0, e0;           // first row / entry of each block, plus an end sentinel
        std::vector<smax::CrsStreamPlan> plans;
        std::vector<smax::DevBuf> rps;         // rebased row pointers
        int blocks() const { return (int)plans.size(); }
    } pipe;
    int pipe_blocks = 6;                        // SMAX_FLAG_SPMV_PIPELINE (0: off)

    // stopwatches
    std::map<std::string, double> timers;
    smax::PendingEvents apply_events;

    ~smax_kernel_s();
};
