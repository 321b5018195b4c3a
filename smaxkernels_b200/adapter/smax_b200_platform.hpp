// smax_b200_platform.hpp -- the B200 platform of a SmaxKernels build: the
// PlatformType::CUDA arms of its five kernels, over this library's C ABI
// (include/smax_b200.h).  Header-only, C++17; compiled into the SmaxKernels
// translation units when SMAX_B200_MODE is 1.
//
// A SmaxKernels checkout gains the platform through a few small edits that
// patch_reference.py (next to this file) applies to a copy of its src/:
//   * common.hpp includes this header, and KernelContext (src/common.hpp:37-44)
//     holds the platform's per-kernel state, released by its destructor;
//   * SPMV::initialize_cuda / apply_cuda / finalize_cuda
//     (src/kernels/spmv/spmv_cuda.hpp:137-184) call B200::spmv;
//   * the CPU-only dispatchers of SpMM, SpGEMM, SpTRSV and SpTRSM
//     (src/kernels/spmm.hpp:68-84, spgemm.hpp:91-105, sptrsv.hpp:74-88,
//     sptrsm.hpp:67-81) gain a PlatformType::CUDA arm calling B200::spmm / spgemm / sptrsv / sptrsm;
//   * Interface::register_kernel (src/interface.cpp:63-67) accepts
//     PlatformType::CUDA without the reference's own CUDA build and, with
//     SMAX_B200_ROUTE_ALL=1, registers every kernel on this platform (the
//     way the reference's own unit tests run on a B200).
//
// Semantics follow the reference's CUDA platform: initialize registers the
// operands the kernel's Args hold and uploads A (on every initialize, as the
// reference's CUDA initialize copies it), apply runs on the GPU, finalize
// brings the result back into the registered host arrays.  Index arrays of
// other integer types than int32 are widened on the host (this platform
// computes with int32 indices) and narrowed back where the reference writes
// them: SpTRSV/SpTRSM move each row's diagonal to its end in the caller's A,
// and SpGEMM returns C's arrays (new[], in the kernel's index type).
#pragma once

#include <atomic>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <iostream>
#include <limits>
#include <stdexcept>
#include <string>
#include <vector>

#include "smax_b200.h"

namespace SMAX {
namespace B200 {

using ULL = unsigned long long;
enum class Phase { Initialize, Apply, Finalize };

// ------------------------------------------------------------ accounting --
// Phases run on the platform; with SMAX_B200_REPORT set in the environment
// the counts are printed at exit (the adapter test checks them).
struct Report {
    std::atomic<long> kernels{0}, initialize{0}, apply{0}, finalize{0};
    ~Report() {
        if (std::getenv("SMAX_B200_REPORT"))
            std::cout << "smax_b200 platform: " << kernels.load() << " kernels, " << initialize.load()
                      << " initialize, " << apply.load() << " apply, " << finalize.load() << " finalize\n";
    }
};
inline Report &report() {
    static Report r;
    return r;
}

// int32 view of an index array of the kernel's IntType
class Index32 {
  public:
    const int32_t *view(IntType it, const void *p, uint64_t n) {
        if (it == IntType::INT32 || p == nullptr) return static_cast<const int32_t *>(p);
        buf_.resize(n);
        for (uint64_t i = 0; i < n; ++i) buf_[i] = narrow(read(it, p, i));
        return buf_.data();
    }
    // copies the (possibly reordered) int32 values back into the caller's array
    void store_back(IntType it, void *p, uint64_t n) const {
        if (it == IntType::INT32 || p == nullptr) return;
        for (uint64_t i = 0; i < n; ++i) write(it, p, i, buf_[i]);
    }
    static long long read(IntType it, const void *p, uint64_t i) {
        switch (it) {
        case IntType::INT16: return static_cast<const int16_t *>(p)[i];
        case IntType::INT32: return static_cast<const int32_t *>(p)[i];
        case IntType::INT64: return static_cast<const int64_t *>(p)[i];
        case IntType::UINT16: return static_cast<const uint16_t *>(p)[i];
        case IntType::UINT32: return static_cast<const uint32_t *>(p)[i];
        case IntType::UINT64: {
            const uint64_t v = static_cast<const uint64_t *>(p)[i];
            if (v > (uint64_t)std::numeric_limits<long long>::max()) throw std::runtime_error("index out of range");
            return (long long)v;
        }
        }
        throw std::runtime_error("unknown index type");
    }
    static void write(IntType it, void *p, uint64_t i, long long v) {
        switch (it) {
        case IntType::INT16: static_cast<int16_t *>(p)[i] = (int16_t)v; return;
        case IntType::INT32: static_cast<int32_t *>(p)[i] = (int32_t)v; return;
        case IntType::INT64: static_cast<int64_t *>(p)[i] = (int64_t)v; return;
        case IntType::UINT16: static_cast<uint16_t *>(p)[i] = (uint16_t)v; return;
        case IntType::UINT32: static_cast<uint32_t *>(p)[i] = (uint32_t)v; return;
        case IntType::UINT64: static_cast<uint64_t *>(p)[i] = (uint64_t)v; return;
        }
    }
    static void *alloc(IntType it, uint64_t n) {  // new[] of the index type, as the reference allocates
        const uint64_t m = n ? n : 1;
        switch (it) {
        case IntType::INT16: return new int16_t[m];
        case IntType::INT32: return new int32_t[m];
        case IntType::INT64: return new int64_t[m];
        case IntType::UINT16: return new uint16_t[m];
        case IntType::UINT32: return new uint32_t[m];
        case IntType::UINT64: return new uint64_t[m];
        }
        throw std::runtime_error("unknown index type");
    }

  private:
    std::vector<int32_t> buf_;
    static int32_t narrow(long long v) {
        if (v < std::numeric_limits<int32_t>::min() || v > std::numeric_limits<int32_t>::max())
            throw std::runtime_error("index does not fit the platform's int32 indices");
        return (int32_t)v;
    }
};

// the platform's state of one registered kernel (KernelContext::b200)
struct State {
    smax_ctx ctx = nullptr;
    smax_kernel k = nullptr;
    Index32 a_col, a_rp, a_cp, a_cl, a_perm, b_col, b_rp;
    // SpGEMM result in this library's int32 arrays, for other index types
    uint64_t c_rows = 0, c_cols = 0, c_nnz = 0;
    void *c_col = nullptr, *c_rp = nullptr, *c_val = nullptr;
    State() = default;
    State(const State &) = delete;
    State &operator=(const State &) = delete;
    ~State() {
        if (k) smax_kernel_destroy(k);
        if (ctx) smax_ctx_destroy(ctx);
    }
};

inline void release(void *p) { delete static_cast<State *>(p); }

inline void ok(smax_status s, const char *what) {
    if (s != SMAX_OK) throw std::runtime_error(std::string(what) + ": " + smax_last_error());
}

inline State &state(KernelContext *kc) {
    if (!kc->b200) {
        State *s = new State();
        try {
            ok(smax_ctx_create(&s->ctx), "smax_ctx_create");
            // indices are widened to int32 on the host; values keep their type
            ok(smax_kernel_create(&s->k, s->ctx, (int)kc->kernel_type, SMAX_INT32, (int)kc->float_type),
               "smax_kernel_create");
        } catch (...) {
            delete s;
            throw;
        }
        kc->b200 = s;
        ++report().kernels;
    }
    return *static_cast<State *>(kc->b200);
}

inline void flag(State &s, int f, int v) { ok(smax_kernel_set_flag(s.k, f, v), "set_flag"); }

// The reference's status convention: 0 on success, 1 (with a message) on error.
template <typename F> int guarded(const char *kernel, F &&f) {
    try {
        f();
        return 0;
    } catch (const std::exception &e) {
        std::cerr << "[SMAX B200] " << kernel << ": " << e.what() << "\n";
        return 1;
    }
}

inline void run_phase(State &s, Phase ph, ULL a, ULL b, ULL c) {
    switch (ph) {
    case Phase::Initialize: ok(smax_kernel_initialize(s.k, a, b, c), "initialize"); ++report().initialize; break;
    case Phase::Apply: ok(smax_kernel_apply(s.k, a, b, c), "apply"); ++report().apply; break;
    case Phase::Finalize: ok(smax_kernel_finalize(s.k, a, b, c), "finalize"); ++report().finalize; break;
    }
}

template <typename CRS> void register_crs_A(State &s, IntType it, CRS &m) {
    ok(smax_kernel_register_A_crs(s.k, m.n_rows, m.n_cols, m.nnz,
                                  const_cast<int32_t *>(s.a_col.view(it, m.col, m.nnz)),
                                  const_cast<int32_t *>(s.a_rp.view(it, m.row_ptr, m.n_rows + 1)), m.val),
       "register_A");
}

inline void register_dense(State &s, int slot, const DenseMatrix &d, bool matrix) {
    ok(smax_kernel_register_dense(s.k, slot, d.n_rows, matrix ? d.n_cols : 1, d.val),
       slot == 1 ? "register_B" : "register_C");
}

// ------------------------------------------------------------------ SpMV --
template <typename Args, typename Flags>
int spmv(Phase ph, KernelContext *kc, Args *a, Flags *f, ULL A_off, ULL x_off, ULL y_off) {
    return guarded("SpMV", [&] {
        State &s = state(kc);
        const IntType it = kc->int_type;
        if (ph == Phase::Initialize) {
            flag(s, SMAX_FLAG_MAT_SCS, f->is_mat_scs);
            flag(s, SMAX_FLAG_MAT_BCRS, f->is_mat_bcrs);
            flag(s, SMAX_FLAG_BLOCK_COLUMN_MAJOR, f->is_block_column_major);
            flag(s, SMAX_FLAG_KERNEL_IMPL, (int)f->kernel_type);
            if (f->is_mat_scs) {
                auto &m = *a->A->scs;
                ok(smax_kernel_register_A_scs(
                       s.k, m.C, m.sigma, m.n_rows, m.n_rows_padded, m.n_cols, m.n_chunks, m.n_elements, m.nnz,
                       const_cast<int32_t *>(s.a_cp.view(it, m.chunk_ptr, m.n_chunks + 1)),
                       const_cast<int32_t *>(s.a_cl.view(it, m.chunk_lengths, m.n_chunks)),
                       const_cast<int32_t *>(s.a_col.view(it, m.col, m.n_elements)), m.val,
                       const_cast<int32_t *>(s.a_perm.view(it, m.perm, m.n_rows))),
                   "register_A");
            } else if (f->is_mat_bcrs) {
                auto &m = *a->A->bcrs;
                ok(smax_kernel_register_A_bcrs(s.k, m.n_rows, m.n_cols, m.nnz, m.b_height, m.b_width, m.height_pad,
                                               m.width_pad, const_cast<int32_t *>(s.a_col.view(it, m.col, m.nnz)),
                                               const_cast<int32_t *>(s.a_rp.view(it, m.row_ptr, m.n_rows + 1)),
                                               m.val),
                   "register_A");
            } else {
                register_crs_A(s, it, *a->A->crs);
            }
            register_dense(s, 1, *a->x, false);
            register_dense(s, 2, *a->y, false);
        }
        run_phase(s, ph, A_off, x_off, y_off);
    });
}

// ------------------------------------------------------------------ SpMM --
template <typename Args, typename Flags>
int spmm(Phase ph, KernelContext *kc, Args *a, Flags *f, ULL A_off, ULL X_off, ULL Y_off) {
    return guarded("SpMM", [&] {
        State &s = state(kc);
        if (ph == Phase::Initialize) {
            flag(s, SMAX_FLAG_VEC_ROW_MAJOR, f->vec_row_major);
            register_crs_A(s, kc->int_type, *a->A->crs);
            register_dense(s, 1, *a->X, true);
            register_dense(s, 2, *a->Y, true);
        }
        run_phase(s, ph, A_off, X_off, Y_off);
    });
}

// ---------------------------------------------------------------- SpGEMM --
template <typename Args, typename Flags> int spgemm(Phase ph, KernelContext *kc, Args *a, Flags *) {
    return guarded("SpGEMM", [&] {
        State &s = state(kc);
        const IntType it = kc->int_type;
        auto &C = *a->C->crs;
        if (ph == Phase::Initialize) {
            register_crs_A(s, it, *a->A->crs);
            auto &B = *a->B->crs;
            ok(smax_kernel_register_B_crs(s.k, B.n_rows, B.n_cols, B.nnz,
                                          const_cast<int32_t *>(s.b_col.view(it, B.col, B.nnz)),
                                          const_cast<int32_t *>(s.b_rp.view(it, B.row_ptr, B.n_rows + 1)), B.val),
               "register_B");
            if (it == IntType::INT32)  // C's arrays go straight to the caller
                ok(smax_kernel_register_C_crs_ref(s.k, static_cast<uint64_t *>(C.n_rows),
                                                  static_cast<uint64_t *>(C.n_cols), static_cast<uint64_t *>(C.nnz),
                                                  C.col, C.row_ptr, C.val),
                   "register_C");
            else
                ok(smax_kernel_register_C_crs_ref(s.k, &s.c_rows, &s.c_cols, &s.c_nnz, &s.c_col, &s.c_rp, &s.c_val),
                   "register_C");
        }
        run_phase(s, ph, 0, 0, 0);
        if (ph == Phase::Finalize && it != IntType::INT32 && s.c_col) {
            // narrow this library's int32 arrays into new[] arrays of the index type
            void *col = Index32::alloc(it, s.c_nnz), *rp = Index32::alloc(it, s.c_rows + 1);
            for (uint64_t i = 0; i < s.c_nnz; ++i) Index32::write(it, col, i, static_cast<int32_t *>(s.c_col)[i]);
            for (uint64_t i = 0; i <= s.c_rows; ++i) Index32::write(it, rp, i, static_cast<int32_t *>(s.c_rp)[i]);
            delete[] static_cast<int32_t *>(s.c_col);
            delete[] static_cast<int32_t *>(s.c_rp);
            *static_cast<ULL *>(C.n_rows) = s.c_rows;
            *static_cast<ULL *>(C.n_cols) = s.c_cols;
            *static_cast<ULL *>(C.nnz) = s.c_nnz;
            *C.col = col;
            *C.row_ptr = rp;
            *C.val = s.c_val;
            s.c_col = s.c_rp = s.c_val = nullptr;
        }
    });
}

// -------------------------------------------------------- SpTRSV / SpTRSM --
// register_B is the solution, register_C the right-hand side
// (src/kernels/sptrsv.hpp:40-58, sptrsm.hpp:40-60); with set_mat_perm the
// solve runs on the Interface's level sets (UtilitiesContainer::lvl_ptr).
template <typename Args, typename Flags>
void tri_initialize(State &s, KernelContext *kc, Args *a, Flags *f, const DenseMatrix &x, const DenseMatrix &b,
                    bool matrix) {
    flag(s, SMAX_FLAG_MAT_PERM, f->mat_permuted);
    flag(s, SMAX_FLAG_MAT_UPPER_TRIANG, f->mat_upper_triang);
    flag(s, SMAX_FLAG_MAT_LOWER_TRIANG, f->mat_lower_triang);
    if (f->mat_permuted && a->uc && a->uc->lvl_ptr)
        ok(smax_ctx_set_levels(s.ctx, a->uc->n_levels, a->uc->lvl_ptr), "levels");
    register_crs_A(s, kc->int_type, *a->A->crs);
    register_dense(s, 1, x, matrix);
    register_dense(s, 2, b, matrix);
}

template <typename Args, typename Flags> int sptrsv(Phase ph, KernelContext *kc, Args *a, Flags *f) {
    return guarded("SpTRSV", [&] {
        State &s = state(kc);
        if (ph == Phase::Initialize) tri_initialize(s, kc, a, f, *a->x, *a->y, false);
        run_phase(s, ph, 0, 0, 0);
        // initialize moved each row's diagonal to its end (in the widened copy)
        if (ph == Phase::Initialize) s.a_col.store_back(kc->int_type, a->A->crs->col, a->A->crs->nnz);
    });
}

template <typename Args, typename Flags> int sptrsm(Phase ph, KernelContext *kc, Args *a, Flags *f) {
    return guarded("SpTRSM", [&] {
        State &s = state(kc);
        if (ph == Phase::Initialize) {
            flag(s, SMAX_FLAG_VEC_ROW_MAJOR, f->vec_row_major);
            tri_initialize(s, kc, a, f, *a->X, *a->Y, true);
        }
        run_phase(s, ph, 0, 0, 0);
        if (ph == Phase::Initialize) s.a_col.store_back(kc->int_type, a->A->crs->col, a->A->crs->nnz);
    });
}

// ---------------------------------------------- dispatcher arms by label --
// The CPU-only dispatchers of the reference pass a label ending in
// _initialize, _apply or _finalize; the CUDA arm each gains maps it to a phase
// and calls its kernel's function above.
inline Phase phase_of(const char *label) {
    const std::string s(label);
    auto ends = [&](const char *t) {
        const size_t n = std::strlen(t);
        return s.size() >= n && s.compare(s.size() - n, n, t) == 0;
    };
    if (ends("initialize")) return Phase::Initialize;
    if (ends("finalize")) return Phase::Finalize;
    return Phase::Apply;
}

}  // namespace B200

inline KernelContext::~KernelContext() { B200::release(b200); }

}  // namespace SMAX
