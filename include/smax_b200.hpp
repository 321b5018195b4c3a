// smax_b200.hpp -- C++ mirror of the SmaxKernels user interface over the
// B200 C ABI (smax_b200.h); header-only, C++17.
//
// Names, argument orders and return conventions follow the reference:
//   SMAX::Interface   (src/interface.hpp:21-48, src/interface.cpp:43-57)
//   SMAX::Kernel      (src/kernel.hpp:7-127): register_A/B/C pick the format by
//                     argument count (src/kernels/spmv.hpp:25-115, spmm.hpp:24-61,
//                     spgemm.hpp:34-83, sptrsv.hpp:23-58, sptrsm.hpp:23-60) and
//                     throw std::runtime_error on a bad count; initialize /
//                     apply / finalize / run return 0 or 1 (SMAX_CHECK_ERROR,
//                     src/macros.hpp:16-20) and log the error
//   SMAX::Utils       (src/utils.hpp:12-87)
// The work runs on the GPU (PlatformType::CUDA); nothing here falls back to
// the host.  Extensions of this platform (device pointers, streams, solve
// schemes, adjoints, refinement, autotuning) are extra methods of Kernel.
#pragma once

#include <cstdint>
#include <iostream>
#include <memory>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <unordered_map>
#include <vector>

#include "smax_b200.h"

namespace smax_b200 {

using ULL = unsigned long long;

enum class KernelType { SPMV = SMAX_KERNEL_SPMV, SPMM = SMAX_KERNEL_SPMM, SPGEMM = SMAX_KERNEL_SPGEMM,
                        SPTRSV = SMAX_KERNEL_SPTRSV, SPTRSM = SMAX_KERNEL_SPTRSM };
enum class PlatformType { CPU = 0, CUDA = 1 };
enum class IntType { INT16 = SMAX_INT16, INT32 = SMAX_INT32, INT64 = SMAX_INT64, UINT16 = SMAX_UINT16,
                     UINT32 = SMAX_UINT32, UINT64 = SMAX_UINT64 };
enum class FloatType { FLOAT32 = SMAX_FLOAT32, FLOAT64 = SMAX_FLOAT64 };
enum class SpMVType { naive_thread_per_row = 0, naive_warp_group = 1, naive_warp_shuffle = 2 };

namespace detail {

inline int check(smax_status s, const char *what) {
    if (s == SMAX_OK) return 0;
    std::cerr << "[smax_b200] " << what << " failed (" << s << "): " << smax_last_error() << "\n";
    return 1;
}

inline void require(smax_status s, const char *what) {
    if (s != SMAX_OK) throw std::runtime_error(std::string(what) + ": " + smax_last_error());
}

template <typename T> uint64_t u64(T v) {
    static_assert(std::is_integral<std::decay_t<T>>::value, "size arguments must be integers");
    return static_cast<uint64_t>(v);
}

template <typename T> void *vp(T *p) { return const_cast<void *>(static_cast<const void *>(p)); }

template <typename VT> constexpr int float_code() {
    static_assert(std::is_same<VT, double>::value || std::is_same<VT, float>::value,
                  "values must be float or double");
    return std::is_same<VT, double>::value ? SMAX_FLOAT64 : SMAX_FLOAT32;
}

}  // namespace detail

class Kernel {
  public:
    Kernel(smax_ctx ctx, KernelType type, IntType it, FloatType ft) : type_(type) {
        detail::require(smax_kernel_create(&h_, ctx, (int)type, (int)it, (int)ft), "register_kernel");
    }
    ~Kernel() {
        if (h_) smax_kernel_destroy(h_);
    }
    Kernel(const Kernel &) = delete;
    Kernel &operator=(const Kernel &) = delete;

    // -- registration (src/kernel.hpp:113-126) ------------------------------
    template <typename... Args> int register_A(Args &&...a) {
        constexpr std::size_t n = sizeof...(Args);
        if constexpr (n == 6) return reg_crs_A(a...);
        else if constexpr (n == 10) return reg_bcrs_A(a...);
        else if constexpr (n == 13) return reg_scs_A(a...);
        else throw std::runtime_error("register_A expects 6 (CRS), 10 (BCRS) or 13 (SELL-C-sigma) args");
    }
    template <typename... Args> int register_B(Args &&...a) {
        constexpr std::size_t n = sizeof...(Args);
        if constexpr (n == 6) return reg_crs_B(a...);  // SpGEMM's B
        else if constexpr (n == 2 || n == 3) return reg_dense(1, a...);
        else throw std::runtime_error("register_B expects 2 or 3 args (6 for SpGEMM)");
    }
    template <typename... Args> int register_C(Args &&...a) {
        constexpr std::size_t n = sizeof...(Args);
        if constexpr (n == 6) {
            if (type_ != KernelType::SPGEMM) throw std::runtime_error("register_C with 6 args is SpGEMM's");
            return reg_crs_ref_C(a...);
        } else if constexpr (n == 2 || n == 3) {
            return reg_dense(2, a...);
        } else {
            throw std::runtime_error("register_C expects 2 or 3 args (6 for SpGEMM)");
        }
    }

    // -- execution (src/kernel.hpp:48-52, 99-111) ---------------------------
    int initialize(ULL A_offset = 0, ULL B_offset = 0, ULL C_offset = 0) {
        return detail::check(smax_kernel_initialize(h_, A_offset, B_offset, C_offset), "initialize");
    }
    int apply(ULL A_offset = 0, ULL B_offset = 0, ULL C_offset = 0) {
        return detail::check(smax_kernel_apply(h_, A_offset, B_offset, C_offset), "apply");
    }
    int finalize(ULL A_offset = 0, ULL B_offset = 0, ULL C_offset = 0) {
        return detail::check(smax_kernel_finalize(h_, A_offset, B_offset, C_offset), "finalize");
    }
    int run(ULL A_offset = 0, ULL B_offset = 0, ULL C_offset = 0) {
        if (initialize(A_offset, B_offset, C_offset)) return 1;
        if (apply(A_offset, B_offset, C_offset)) return 1;
        return finalize(A_offset, B_offset, C_offset);
    }
    int swap_operands() { return detail::check(smax_kernel_swap_operands(h_), "swap_operands"); }

    // -- flags (src/kernel.hpp:58-90) ----------------------------------------
    int set_mat_perm(bool v) { return flag(SMAX_FLAG_MAT_PERM, v); }
    int set_mat_upper_triang(bool v) { return flag(SMAX_FLAG_MAT_UPPER_TRIANG, v); }
    int set_mat_lower_triang(bool v) { return flag(SMAX_FLAG_MAT_LOWER_TRIANG, v); }
    int set_vec_row_major(bool v) { return flag(SMAX_FLAG_VEC_ROW_MAJOR, v); }
    int set_mat_scs(bool v) { return flag(SMAX_FLAG_MAT_SCS, v); }
    int set_mat_bcrs(bool v) { return flag(SMAX_FLAG_MAT_BCRS, v); }
    int set_block_column_major(bool v) { return flag(SMAX_FLAG_BLOCK_COLUMN_MAJOR, v); }
    int set_kernel_implementation(SpMVType t) { return flag(SMAX_FLAG_KERNEL_IMPL, (int)t); }

    // -- platform extensions -------------------------------------------------
    int set_device_pointers(bool v) { return flag(SMAX_FLAG_DEVICE_POINTERS, v); }
    int mark_A_dirty() { return flag(SMAX_FLAG_A_DIRTY, 1); }
    int set_spmv_variant(int v) { return flag(SMAX_FLAG_SPMV_VARIANT, v); }
    int set_solve_mode(int mode) { return flag(SMAX_FLAG_SOLVE_MODE, mode); }
    int set_level_merge(int rows) { return flag(SMAX_FLAG_LEVEL_MERGE, rows); }
    int set_sweep_cluster(bool v) { return flag(SMAX_FLAG_SWEEP_CLUSTER, v); }
    int set_spmv_pipeline(int blocks) { return flag(SMAX_FLAG_SPMV_PIPELINE, blocks); }
    int set_timers(bool on) { return flag(SMAX_FLAG_TIMERS, on ? 1 : 0); }
    int set_spin_limit(int kilo_polls) { return flag(SMAX_FLAG_SPIN_LIMIT, kilo_polls); }
    int set_refine(int steps, int tol_exp = 0) {
        return flag(SMAX_FLAG_REFINE, steps) || flag(SMAX_FLAG_REFINE_TOL, tol_exp);
    }
    int refine_stats(int *steps, double *last_rel) {
        return detail::check(smax_kernel_get_refine_stats(h_, steps, last_rel), "refine_stats");
    }
    int adjoint(const void *g, void *d_in, void *d_val, const void *x = nullptr) {
        return detail::check(smax_kernel_adjoint(h_, x, g, d_in, d_val), "adjoint");
    }
    int update_A_values(const void *val) {
        return detail::check(smax_kernel_update_A_values(h_, val), "update_A_values");
    }
    int autotune(smax_tuning *out = nullptr) {
        smax_tuning t{};
        const int rc = detail::check(smax_kernel_autotune(h_, &t), "autotune");
        if (out) *out = t;
        return rc;
    }
    int sync() { return detail::check(smax_kernel_sync(h_), "sync"); }
    int set_stream(void *cuda_stream) { return detail::check(smax_kernel_set_stream(h_, cuda_stream), "set_stream"); }
    double timer(const char *name) const {
        double s = 0.0;
        smax_kernel_get_timer(h_, name, &s);
        return s;
    }
    smax_kernel handle() const { return h_; }
    KernelType type() const { return type_; }

  private:
    smax_kernel h_ = nullptr;
    KernelType type_;

    int flag(int f, int v) { return detail::check(smax_kernel_set_flag(h_, f, v), "set_flag"); }

    template <typename S0, typename S1, typename S2, typename I, typename R, typename V>
    int reg_crs_A(S0 n_rows, S1 n_cols, S2 nnz, I *col, R *row_ptr, V *val) {
        return detail::check(smax_kernel_register_A_crs(h_, detail::u64(n_rows), detail::u64(n_cols),
                                                        detail::u64(nnz), detail::vp(col), detail::vp(row_ptr),
                                                        detail::vp(val)),
                             "register_A");
    }
    template <typename S0, typename S1, typename S2, typename S3, typename S4, typename S5, typename S6, typename I,
              typename R, typename V>
    int reg_bcrs_A(S0 n_rows, S1 n_cols, S2 n_blocks, S3 bh, S4 bw, S5 hpad, S6 wpad, I *col, R *row_ptr, V *val) {
        return detail::check(smax_kernel_register_A_bcrs(h_, detail::u64(n_rows), detail::u64(n_cols),
                                                         detail::u64(n_blocks), detail::u64(bh), detail::u64(bw),
                                                         detail::u64(hpad), detail::u64(wpad), detail::vp(col),
                                                         detail::vp(row_ptr), detail::vp(val)),
                             "register_A");
    }
    template <typename S0, typename S1, typename S2, typename S3, typename S4, typename S5, typename S6, typename S7,
              typename I0, typename I1, typename I2, typename V, typename P>
    int reg_scs_A(S0 C, S1 sigma, S2 n_rows, S3 n_rows_padded, S4 n_cols, S5 n_chunks, S6 n_elements, S7 nnz,
                  I0 *chunk_ptr, I1 *chunk_lengths, I2 *col, V *val, P *perm) {
        return detail::check(
            smax_kernel_register_A_scs(h_, detail::u64(C), detail::u64(sigma), detail::u64(n_rows),
                                       detail::u64(n_rows_padded), detail::u64(n_cols), detail::u64(n_chunks),
                                       detail::u64(n_elements), detail::u64(nnz), detail::vp(chunk_ptr),
                                       detail::vp(chunk_lengths), detail::vp(col), detail::vp(val), detail::vp(perm)),
            "register_A");
    }
    template <typename S0, typename S1, typename S2, typename I, typename R, typename V>
    int reg_crs_B(S0 n_rows, S1 n_cols, S2 nnz, I *col, R *row_ptr, V *val) {
        return detail::check(smax_kernel_register_B_crs(h_, detail::u64(n_rows), detail::u64(n_cols),
                                                        detail::u64(nnz), detail::vp(col), detail::vp(row_ptr),
                                                        detail::vp(val)),
                             "register_B");
    }
    template <typename I, typename V>
    int reg_crs_ref_C(ULL *n_rows, ULL *n_cols, ULL *nnz, I **col, I **row_ptr, V **val) {
        static_assert(sizeof(ULL) == sizeof(uint64_t), "64-bit sizes");
        return detail::check(smax_kernel_register_C_crs_ref(h_, reinterpret_cast<uint64_t *>(n_rows),
                                                            reinterpret_cast<uint64_t *>(n_cols),
                                                            reinterpret_cast<uint64_t *>(nnz),
                                                            reinterpret_cast<void **>(col),
                                                            reinterpret_cast<void **>(row_ptr),
                                                            reinterpret_cast<void **>(val)),
                             "register_C");
    }
    template <typename S0, typename V> int reg_dense(int slot, S0 n_rows, V *val) {
        return detail::check(smax_kernel_register_dense(h_, slot, detail::u64(n_rows), 1, detail::vp(val)),
                             slot == 1 ? "register_B" : "register_C");
    }
    template <typename S0, typename S1, typename V> int reg_dense(int slot, S0 n_rows, S1 n_cols, V *val) {
        return detail::check(smax_kernel_register_dense(h_, slot, detail::u64(n_rows), detail::u64(n_cols),
                                                        detail::vp(val)),
                             slot == 1 ? "register_B" : "register_C");
    }
};

class Utils {
  public:
    explicit Utils(smax_ctx ctx) : ctx_(ctx) {}

    // Utils::convert_crs_to_scs (src/utils.hpp:26-32); arrays allocated with new[]
    template <typename IT, typename VT, typename ST>
    int convert_crs_to_scs(const ST _n_rows, const ST _n_cols, const ST _nnz, const IT *_col, const IT *_row_ptr,
                           const VT *_val, const ST C, const ST sigma, ST &n_rows, ST &n_rows_padded, ST &n_cols,
                           ST &n_chunks, ST &n_elements, ST &nnz, IT *&chunk_ptr, IT *&chunk_lengths, IT *&col,
                           VT *&val, IT *&perm) {
        static_assert(sizeof(IT) == 4, "int32 indices");
        uint64_t meta[6] = {};
        void *p[5] = {};
        const int rc = detail::check(
            smax_utils_convert_crs_to_scs(SMAX_INT32, detail::float_code<VT>(), detail::u64(_n_rows),
                                          detail::u64(_n_cols), detail::u64(_nnz), _col, _row_ptr, _val,
                                          detail::u64(C), detail::u64(sigma), meta, &p[0], &p[1], &p[2], &p[3],
                                          &p[4]),
            "convert_crs_to_scs");
        if (rc) return rc;
        n_rows = (ST)meta[0];
        n_rows_padded = (ST)meta[1];
        n_cols = (ST)meta[2];
        n_chunks = (ST)meta[3];
        n_elements = (ST)meta[4];
        nnz = (ST)meta[5];
        chunk_ptr = static_cast<IT *>(p[0]);
        chunk_lengths = static_cast<IT *>(p[1]);
        col = static_cast<IT *>(p[2]);
        val = static_cast<VT *>(p[3]);
        perm = static_cast<IT *>(p[4]);
        return 0;
    }

    // Utils::convert_crs_to_bcrs (src/utils.hpp:38-47)
    template <typename IT, typename VT, typename ST>
    int convert_crs_to_bcrs(const ST _n_rows, const ST _n_cols, const ST _nnz, const IT *_col, const IT *_row_ptr,
                            const VT *_val, ST &n_rows, ST &n_cols, ST &nnz, ST &b_height, ST &b_width,
                            ST &height_pad, ST &width_pad, IT *&col, IT *&row_ptr, VT *&val,
                            const ST target_b_height, const ST target_b_width, const ST target_height_pad,
                            const ST target_width_pad, const bool block_column_major) {
        static_assert(sizeof(IT) == 4, "int32 indices");
        uint64_t meta[7] = {};
        void *p[3] = {};
        const int rc = detail::check(
            smax_utils_convert_crs_to_bcrs(SMAX_INT32, detail::float_code<VT>(), detail::u64(_n_rows),
                                           detail::u64(_n_cols), detail::u64(_nnz), _col, _row_ptr, _val,
                                           detail::u64(target_b_height), detail::u64(target_b_width),
                                           detail::u64(target_height_pad), detail::u64(target_width_pad),
                                           block_column_major ? 1 : 0, meta, &p[0], &p[1], &p[2]),
            "convert_crs_to_bcrs");
        if (rc) return rc;
        n_rows = (ST)meta[0];
        n_cols = (ST)meta[1];
        nnz = (ST)meta[2];
        b_height = (ST)meta[3];
        b_width = (ST)meta[4];
        height_pad = (ST)meta[5];
        width_pad = (ST)meta[6];
        col = static_cast<IT *>(p[0]);
        row_ptr = static_cast<IT *>(p[1]);
        val = static_cast<VT *>(p[2]);
        return 0;
    }

    // Utils::build_symmetric_crs (src/utils.hpp:34-36)
    template <typename IT, typename ST>
    int build_symmetric_crs(IT *A_row_ptr, IT *A_col, ST A_n_rows, IT *&A_sym_row_ptr, IT *&A_sym_col,
                            ST &A_sym_nnz) {
        void *rp = nullptr, *cl = nullptr;
        uint64_t nz = 0;
        const int rc = detail::check(smax_utils_build_symmetric_crs(SMAX_INT32, detail::u64(A_n_rows), A_row_ptr,
                                                                    A_col, &rp, &cl, &nz),
                                     "build_symmetric_crs");
        if (rc) return rc;
        A_sym_row_ptr = static_cast<IT *>(rp);
        A_sym_col = static_cast<IT *>(cl);
        A_sym_nnz = (ST)nz;
        return 0;
    }

    // Utils::generate_perm (src/utils.hpp:68-70); the level pointer is kept by the Interface
    template <typename IT>
    void generate_perm(int A_n_rows, IT *A_row_ptr, IT *A_col, int *perm, int *inv_perm,
                       std::string type = std::string("BFS")) {
        detail::require(smax_utils_generate_perm(ctx_, SMAX_INT32, (uint64_t)A_n_rows, A_row_ptr, A_col, perm,
                                                 inv_perm, type.c_str()),
                        "generate_perm");
    }

    // Utils::apply_mat_perm / apply_vec_perm (src/utils.hpp:76-82)
    template <typename IT, typename VT>
    void apply_mat_perm(int A_n_rows, IT *A_row_ptr, IT *A_col, VT *A_val, IT *A_perm_row_ptr, IT *A_perm_col,
                        VT *A_perm_val, int *perm, int *inv_perm) {
        detail::require(smax_utils_apply_mat_perm(SMAX_INT32, detail::float_code<VT>(), (uint64_t)A_n_rows,
                                                  A_row_ptr, A_col, A_val, A_perm_row_ptr, A_perm_col, A_perm_val,
                                                  perm, inv_perm),
                        "apply_mat_perm");
    }
    template <typename VT> void apply_vec_perm(int n_rows, VT *vec, VT *vec_perm, int *perm) {
        detail::require(smax_utils_apply_vec_perm(detail::float_code<VT>(), (uint64_t)n_rows, vec, vec_perm, perm),
                        "apply_vec_perm");
    }

    // Utils::sanity_check_perm (src/utils/permutations.hpp:794-818)
    template <typename IT> bool sanity_check_perm(int A_n_rows, const IT *A_row_ptr, const IT *A_col, const int *colors) {
        int valid = 0;
        detail::require(smax_utils_sanity_check_perm(SMAX_INT32, (uint64_t)A_n_rows, A_row_ptr, A_col, colors, &valid,
                                                     nullptr),
                        "sanity_check_perm");
        return valid != 0;
    }

    // The examples' Matrix Market reader + convert_coo_to_crs
    // (examples/matrix_structs.hpp:52-180, 338-387): CRS arrays allocated with
    // new[] (release with smax_free_host)
    template <typename VT>
    int read_mtx(const std::string &path, uint64_t &n_rows, uint64_t &n_cols, uint64_t &nnz, int *&row_ptr, int *&col,
                 VT *&val) {
        void *rp = nullptr, *cl = nullptr, *vl = nullptr;
        const int rc = detail::check(smax_utils_read_mtx(path.c_str(), detail::float_code<VT>(), &n_rows, &n_cols, &nnz,
                                                         &rp, &cl, &vl),
                                     "read_mtx");
        if (rc) return rc;
        row_ptr = static_cast<int *>(rp);
        col = static_cast<int *>(cl);
        val = static_cast<VT *>(vl);
        return 0;
    }

  private:
    smax_ctx ctx_;
};

// The reference's solver programs (examples/applications/jacobi,
// gauss_seidel) on device-resident operators: smax_solver_* with RAII.
class Solver {
  public:
    enum Kind { JACOBI = SMAX_SOLVER_JACOBI, GAUSS_SEIDEL = SMAX_SOLVER_GAUSS_SEIDEL };
    template <typename VT>
    Solver(Kind kind, uint64_t n_rows, uint64_t nnz, const int *row_ptr, const int *col, const VT *val)
        : vbytes_(sizeof(VT)) {
        detail::require(smax_solver_create(&s_, kind, detail::float_code<VT>(), n_rows, nnz, row_ptr, col, val),
                        "Solver");
    }
    ~Solver() {
        if (s_) smax_solver_destroy(s_);
    }
    Solver(const Solver &) = delete;
    Solver &operator=(const Solver &) = delete;

    // the applications' loop from the initial guess in x; the solution is left in x
    template <typename VT>
    smax_solver_stats solve(const VT *b, VT *x, double tol = 1e-8, int max_iters = 1000, int check_length = 5,
                            int mode = SMAX_SOLVER_DEVICE_LOOP, void *stream = nullptr) {
        if (sizeof(VT) != vbytes_) throw std::runtime_error("Solver::solve: value type differs from the matrix");
        smax_solver_opts o{tol, max_iters, check_length, mode};
        smax_solver_stats st{};
        detail::require(smax_solver_solve(s_, b, x, &o, &st, stream), "Solver::solve");
        return st;
    }
    std::vector<double> history() const {
        int count = 0;
        detail::require(smax_solver_get_history(s_, nullptr, 0, &count), "Solver::history");
        std::vector<double> h(count);
        if (count) detail::require(smax_solver_get_history(s_, h.data(), count, &count), "Solver::history");
        return h;
    }

  private:
    smax_solver s_ = nullptr;
    size_t vbytes_;
};

class Interface {
  public:
    Utils *utils = nullptr;

    Interface() {
        detail::require(smax_ctx_create(&ctx_), "Interface");
        utils_.reset(new Utils(ctx_));
        utils = utils_.get();
    }
    ~Interface() {
        kernels_.clear();
        if (ctx_) smax_ctx_destroy(ctx_);
    }
    Interface(const Interface &) = delete;
    Interface &operator=(const Interface &) = delete;

    // Interface::register_kernel (src/interface.hpp:33-36): this platform
    // serves PlatformType::CUDA; other platforms return 1.
    int register_kernel(const std::string &name, KernelType type, PlatformType platform = PlatformType::CUDA,
                        IntType it = IntType::INT32, FloatType ft = FloatType::FLOAT64) {
        if (platform != PlatformType::CUDA) {
            std::cerr << "[smax_b200] Platform not supported\n";
            return 1;
        }
        try {
            kernels_[name].reset(new Kernel(ctx_, type, it, ft));
        } catch (const std::exception &e) {
            std::cerr << "[smax_b200] " << e.what() << "\n";
            kernels_.erase(name);
            return 1;
        }
        return 0;
    }

    // Interface::kernel (src/interface.cpp:43-51): unknown names throw
    Kernel *kernel(const std::string &name) {
        auto it = kernels_.find(name);
        if (it == kernels_.end()) throw std::runtime_error("Kernel '" + name + "' does not exist");
        return it->second.get();
    }

    int get_n_levels() const { return smax_ctx_get_n_levels(ctx_); }
    int get_level_ptr_at(int idx) const { return smax_ctx_get_level_ptr_at(ctx_, idx); }
    // a level pointer computed elsewhere (n_levels + 1 entries)
    int set_levels(int n_levels, const int *lvl_ptr) {
        return detail::check(smax_ctx_set_levels(ctx_, n_levels, lvl_ptr), "set_levels");
    }

    // Utils::print_timers (src/utils.hpp:24): stopwatches of every kernel
    void print_timers() const {
        for (const auto &kv : kernels_)
            for (const char *t : {"initialize", "apply", "finalize"})
                std::cout << kv.first << " " << t << ": " << kv.second->timer(t) << " s\n";
    }

  private:
    smax_ctx ctx_ = nullptr;
    std::unique_ptr<Utils> utils_;
    std::unordered_map<std::string, std::unique_ptr<Kernel>> kernels_;
};

}  // namespace smax_b200
