// ref_shim.cpp -- C-ABI shim around the UNMODIFIED SmaxKernels reference.
//
// TEST INFRASTRUCTURE ONLY.  This file is compiled (by oracle/Makefile) together
// with the reference's own sources, read in place from the reference checkout,
// into oracle/_ref/libsmax_ref.so.  Only tests/, __graft_entry__.smoke() and the
// CPU-baseline leg of bench.py load that library: as a checker of the product and
// as the timed "reference" CPU arm.  The product (smaxkernels_b200) never links it.
//
// Every function drives the reference through its public API exactly as the
// reference's own tests and benchmarks do:
//   SMAX::Interface::register_kernel / kernel()->register_A/B/C / run()
//   (src/interface.hpp:21-48, src/kernel.hpp:99-126)
//   SMAX::Utils::convert_crs_to_scs / convert_crs_to_bcrs / generate_perm /
//   build_symmetric_crs / apply_mat_perm / apply_vec_perm (src/utils.hpp:12-87)
//
// The reference defines non-inline functions in headers (src/kernels/*/..._cpu.hpp,
// src/utils/timers.hpp), so the whole reference is built as ONE translation unit:
// this file includes interface.cpp and error_handler.cpp directly.

#include "interface.cpp"
#include "error_handler.cpp"
// the examples' Matrix Market reader and COO/CRS structs (examples/)
#include "mmio.cpp"
#include "matrix_structs.hpp"

#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

namespace {

using SMAX::ULL;
thread_local std::string g_err;

template <typename F> int guarded(F &&f) {
    try {
        return f();
    } catch (const std::exception &e) {
        g_err = e.what();
        return -1;
    } catch (...) {
        g_err = "unknown exception";
        return -1;
    }
}

SMAX::FloatType ftype(int vbits) {
    return vbits == 32 ? SMAX::FloatType::FLOAT32 : SMAX::FloatType::FLOAT64;
}

template <typename T> T *copy_new(const T *src, size_t n) {
    T *d = new T[n > 0 ? n : 1];
    if (n)
        std::memcpy(d, src, n * sizeof(T));
    return d;
}

// Registers the levels of a previous generate_perm (or caller-supplied ones) in
// the Interface's UtilitiesContainer, the state crs_sptrsv_lvl reads
// (src/kernels/sptrsv/sptrsv_cpu/sptrsv_cpu_core.hpp:74-84).
void set_levels(SMAX::Interface *smax, int n_levels, const int *lvl_ptr) {
    delete[] smax->utils->uc->lvl_ptr;
    smax->utils->uc->lvl_ptr = copy_new(lvl_ptr, (size_t)n_levels + 1);
    smax->utils->uc->n_levels = n_levels;
}

double now_s() {
    using clk = std::chrono::steady_clock;
    return std::chrono::duration<double>(clk::now().time_since_epoch()).count();
}

// Times apply() only, after one initialize(), like the reference benchmark
// harness (examples/benchmarks/benchmarks_common.hpp:60-95): warm-up, then
// `reps` back-to-back applies.  Returns seconds per apply.
double time_applies(SMAX::Interface *smax, const std::string &name, int warm,
                    int reps) {
    smax->kernel(name)->initialize();
    for (int i = 0; i < warm; ++i)
        smax->kernel(name)->apply();
    double t0 = now_s();
    for (int i = 0; i < reps; ++i)
        smax->kernel(name)->apply();
    double t1 = now_s();
    smax->kernel(name)->finalize();
    return (t1 - t0) / (reps > 0 ? reps : 1);
}

} // namespace

extern "C" {

const char *ref_last_error(void) { return g_err.c_str(); }

int ref_set_threads(int n) {
#ifdef _OPENMP
    if (n > 0)
        omp_set_num_threads(n);
    return omp_get_max_threads();
#else
    (void)n;
    return 1;
#endif
}

void ref_free_int(int *p) { delete[] p; }
void ref_free_val(int vbits, void *p) {
    if (vbits == 32)
        delete[] static_cast<float *>(p);
    else
        delete[] static_cast<double *>(p);
}

// ---------------------------------------------------------------- SpMV CRS --
int ref_spmv_crs(int vbits, uint64_t n_rows, uint64_t n_cols, uint64_t nnz,
                 int *col, int *row_ptr, void *val, void *x, void *y) {
    return guarded([&] {
        SMAX::Interface smax;
        smax.register_kernel("k", SMAX::KernelType::SPMV,
                             SMAX::PlatformType::CPU, SMAX::IntType::INT32,
                             ftype(vbits));
        smax.kernel("k")->register_A(n_rows, n_cols, nnz, col, row_ptr, val);
        smax.kernel("k")->register_B(n_cols, x);
        smax.kernel("k")->register_C(n_rows, y);
        return smax.kernel("k")->run();
    });
}

double ref_time_spmv_crs(int vbits, uint64_t n_rows, uint64_t n_cols,
                         uint64_t nnz, int *col, int *row_ptr, void *val,
                         void *x, void *y, int warm, int reps) {
    double t = -1.0;
    int rc = guarded([&] {
        SMAX::Interface smax;
        smax.register_kernel("k", SMAX::KernelType::SPMV,
                             SMAX::PlatformType::CPU, SMAX::IntType::INT32,
                             ftype(vbits));
        smax.kernel("k")->register_A(n_rows, n_cols, nnz, col, row_ptr, val);
        smax.kernel("k")->register_B(n_cols, x);
        smax.kernel("k")->register_C(n_rows, y);
        t = time_applies(&smax, "k", warm, reps);
        return 0;
    });
    return rc == 0 ? t : -1.0;
}

// ---------------------------------------------------------------- SpMV SCS --
int ref_spmv_scs(int vbits, uint64_t C, uint64_t sigma, uint64_t n_rows,
                 uint64_t n_rows_padded, uint64_t n_cols, uint64_t n_chunks,
                 uint64_t n_elements, uint64_t nnz, int *chunk_ptr,
                 int *chunk_lengths, int *col, void *val, int *perm, void *x,
                 void *y) {
    return guarded([&] {
        SMAX::Interface smax;
        smax.register_kernel("k", SMAX::KernelType::SPMV,
                             SMAX::PlatformType::CPU, SMAX::IntType::INT32,
                             ftype(vbits));
        smax.kernel("k")->set_mat_scs(true);
        smax.kernel("k")->register_A(C, sigma, n_rows, n_rows_padded, n_cols,
                                     n_chunks, n_elements, nnz, chunk_ptr,
                                     chunk_lengths, col, val, perm);
        uint64_t vs = n_rows_padded > n_cols ? n_rows_padded : n_cols;
        smax.kernel("k")->register_B(vs, x);
        smax.kernel("k")->register_C(vs, y);
        return smax.kernel("k")->run();
    });
}

double ref_time_spmv_scs(int vbits, uint64_t C, uint64_t sigma,
                         uint64_t n_rows, uint64_t n_rows_padded,
                         uint64_t n_cols, uint64_t n_chunks,
                         uint64_t n_elements, uint64_t nnz, int *chunk_ptr,
                         int *chunk_lengths, int *col, void *val, int *perm,
                         void *x, void *y, int warm, int reps) {
    double t = -1.0;
    int rc = guarded([&] {
        SMAX::Interface smax;
        smax.register_kernel("k", SMAX::KernelType::SPMV,
                             SMAX::PlatformType::CPU, SMAX::IntType::INT32,
                             ftype(vbits));
        smax.kernel("k")->set_mat_scs(true);
        smax.kernel("k")->register_A(C, sigma, n_rows, n_rows_padded, n_cols,
                                     n_chunks, n_elements, nnz, chunk_ptr,
                                     chunk_lengths, col, val, perm);
        uint64_t vs = n_rows_padded > n_cols ? n_rows_padded : n_cols;
        smax.kernel("k")->register_B(vs, x);
        smax.kernel("k")->register_C(vs, y);
        t = time_applies(&smax, "k", warm, reps);
        return 0;
    });
    return rc == 0 ? t : -1.0;
}

// --------------------------------------------------------------- SpMV BCRS --
int ref_spmv_bcrs(int vbits, uint64_t n_rows, uint64_t n_cols,
                  uint64_t n_blocks, uint64_t b_h, uint64_t b_w,
                  uint64_t h_pad, uint64_t w_pad, int *col, int *row_ptr,
                  void *val, int col_major, void *x, void *y) {
    return guarded([&] {
        SMAX::Interface smax;
        smax.register_kernel("k", SMAX::KernelType::SPMV,
                             SMAX::PlatformType::CPU, SMAX::IntType::INT32,
                             ftype(vbits));
        smax.kernel("k")->set_mat_bcrs(true);
        smax.kernel("k")->register_A(n_rows, n_cols, n_blocks, b_h, b_w, h_pad,
                                     w_pad, col, row_ptr, val);
        smax.kernel("k")->register_B(n_cols * w_pad, x);
        smax.kernel("k")->register_C(n_rows * h_pad, y);
        smax.kernel("k")->set_block_column_major(col_major != 0);
        return smax.kernel("k")->run();
    });
}

double ref_time_spmv_bcrs(int vbits, uint64_t n_rows, uint64_t n_cols,
                          uint64_t n_blocks, uint64_t b_h, uint64_t b_w,
                          uint64_t h_pad, uint64_t w_pad, int *col,
                          int *row_ptr, void *val, int col_major, void *x,
                          void *y, int warm, int reps) {
    double t = -1.0;
    int rc = guarded([&] {
        SMAX::Interface smax;
        smax.register_kernel("k", SMAX::KernelType::SPMV,
                             SMAX::PlatformType::CPU, SMAX::IntType::INT32,
                             ftype(vbits));
        smax.kernel("k")->set_mat_bcrs(true);
        smax.kernel("k")->register_A(n_rows, n_cols, n_blocks, b_h, b_w, h_pad,
                                     w_pad, col, row_ptr, val);
        smax.kernel("k")->register_B(n_cols * w_pad, x);
        smax.kernel("k")->register_C(n_rows * h_pad, y);
        smax.kernel("k")->set_block_column_major(col_major != 0);
        t = time_applies(&smax, "k", warm, reps);
        return 0;
    });
    return rc == 0 ? t : -1.0;
}

// -------------------------------------------------------------------- SpMM --
int ref_spmm(int vbits, int row_major, uint64_t n_rows, uint64_t n_cols,
             uint64_t nnz, int *col, int *row_ptr, void *val, uint64_t k,
             void *X, void *Y) {
    return guarded([&] {
        SMAX::Interface smax;
        smax.register_kernel("k", SMAX::KernelType::SPMM,
                             SMAX::PlatformType::CPU, SMAX::IntType::INT32,
                             ftype(vbits));
        smax.kernel("k")->register_A(n_rows, n_cols, nnz, col, row_ptr, val);
        smax.kernel("k")->register_B(n_cols, k, X);
        smax.kernel("k")->register_C(n_rows, k, Y);
        smax.kernel("k")->set_vec_row_major(row_major != 0);
        return smax.kernel("k")->run();
    });
}

double ref_time_spmm(int vbits, int row_major, uint64_t n_rows,
                     uint64_t n_cols, uint64_t nnz, int *col, int *row_ptr,
                     void *val, uint64_t k, void *X, void *Y, int warm,
                     int reps) {
    double t = -1.0;
    int rc = guarded([&] {
        SMAX::Interface smax;
        smax.register_kernel("k", SMAX::KernelType::SPMM,
                             SMAX::PlatformType::CPU, SMAX::IntType::INT32,
                             ftype(vbits));
        smax.kernel("k")->register_A(n_rows, n_cols, nnz, col, row_ptr, val);
        smax.kernel("k")->register_B(n_cols, k, X);
        smax.kernel("k")->register_C(n_rows, k, Y);
        smax.kernel("k")->set_vec_row_major(row_major != 0);
        t = time_applies(&smax, "k", warm, reps);
        return 0;
    });
    return rc == 0 ? t : -1.0;
}

// ------------------------------------------------------------------ SpGEMM --
// C's arrays are allocated by the reference with new[] (ownership passes to
// the caller, src/kernels/spgemm/spgemm_cpu/symbolic_phase_impl.hpp:132-151);
// release them with ref_free_int / ref_free_val.
int ref_spgemm(int vbits, uint64_t a_n_rows, uint64_t a_n_cols,
               uint64_t a_nnz, int *a_col, int *a_row_ptr, void *a_val,
               uint64_t b_n_rows, uint64_t b_n_cols, uint64_t b_nnz,
               int *b_col, int *b_row_ptr, void *b_val, uint64_t *c_meta,
               int **c_col, int **c_row_ptr, void **c_val) {
    return guarded([&] {
        SMAX::Interface smax;
        smax.register_kernel("k", SMAX::KernelType::SPGEMM,
                             SMAX::PlatformType::CPU, SMAX::IntType::INT32,
                             ftype(vbits));
        smax.kernel("k")->register_A(a_n_rows, a_n_cols, a_nnz, a_col,
                                     a_row_ptr, a_val);
        smax.kernel("k")->register_B(b_n_rows, b_n_cols, b_nnz, b_col,
                                     b_row_ptr, b_val);
        ULL nr = 0, nc = 0, nz = 0;
        int *cc = nullptr, *cr = nullptr;
        void *cv = nullptr;
        smax.kernel("k")->register_C(&nr, &nc, &nz, &cc, &cr, &cv);
        int rc = smax.kernel("k")->run();
        c_meta[0] = nr;
        c_meta[1] = nc;
        c_meta[2] = nz;
        *c_col = cc;
        *c_row_ptr = cr;
        *c_val = cv;
        return rc;
    });
}

double ref_time_spgemm(int vbits, uint64_t n_rows, uint64_t n_cols,
                       uint64_t nnz, int *col, int *row_ptr, void *val,
                       int reps) {
    double t = -1.0;
    int rc = guarded([&] {
        double acc = 0.0;
        for (int r = 0; r < reps; ++r) {
            SMAX::Interface smax;
            smax.register_kernel("k", SMAX::KernelType::SPGEMM,
                                 SMAX::PlatformType::CPU, SMAX::IntType::INT32,
                                 ftype(vbits));
            smax.kernel("k")->register_A(n_rows, n_cols, nnz, col, row_ptr,
                                         val);
            smax.kernel("k")->register_B(n_rows, n_cols, nnz, col, row_ptr,
                                         val);
            ULL nr = 0, nc = 0, nz = 0;
            int *cc = nullptr, *cr = nullptr;
            void *cv = nullptr;
            smax.kernel("k")->register_C(&nr, &nc, &nz, &cc, &cr, &cv);
            smax.kernel("k")->initialize();
            double t0 = now_s();
            smax.kernel("k")->apply();
            acc += now_s() - t0;
            smax.kernel("k")->finalize();
            delete[] cc;
            delete[] cr;
            ref_free_val(vbits, cv);
        }
        t = acc / (reps > 0 ? reps : 1);
        return 0;
    });
    return rc == 0 ? t : -1.0;
}

// ------------------------------------------------------------------ SpTRSV --
// NOTE: like the reference, initialize() swaps each row's diagonal entry to the
// end of the row IN THE CALLER'S col/val arrays
// (src/kernels/sptrsv/sptrsv_cpu/sptrsv_cpu_crs_helpers_impl.hpp:9-38).
// x is the solution (register_B), b the right-hand side (register_C).
int ref_sptrsv(int vbits, int upper, int permuted, uint64_t n_rows,
               uint64_t n_cols, uint64_t nnz, int *col, int *row_ptr,
               void *val, void *x, void *b, int n_levels, const int *lvl_ptr) {
    return guarded([&] {
        SMAX::Interface smax;
        smax.register_kernel("k", SMAX::KernelType::SPTRSV,
                             SMAX::PlatformType::CPU, SMAX::IntType::INT32,
                             ftype(vbits));
        if (permuted) {
            set_levels(&smax, n_levels, lvl_ptr);
            smax.kernel("k")->set_mat_perm(true);
        }
        if (upper)
            smax.kernel("k")->set_mat_upper_triang(true);
        smax.kernel("k")->register_A(n_rows, n_cols, nnz, col, row_ptr, val);
        smax.kernel("k")->register_B(n_cols, x);
        smax.kernel("k")->register_C(n_rows, b);
        return smax.kernel("k")->run();
    });
}

double ref_time_sptrsv(int vbits, int upper, int permuted, uint64_t n_rows,
                       uint64_t n_cols, uint64_t nnz, int *col, int *row_ptr,
                       void *val, void *x, void *b, int n_levels,
                       const int *lvl_ptr, int warm, int reps) {
    double t = -1.0;
    int rc = guarded([&] {
        SMAX::Interface smax;
        smax.register_kernel("k", SMAX::KernelType::SPTRSV,
                             SMAX::PlatformType::CPU, SMAX::IntType::INT32,
                             ftype(vbits));
        if (permuted) {
            set_levels(&smax, n_levels, lvl_ptr);
            smax.kernel("k")->set_mat_perm(true);
        }
        if (upper)
            smax.kernel("k")->set_mat_upper_triang(true);
        smax.kernel("k")->register_A(n_rows, n_cols, nnz, col, row_ptr, val);
        smax.kernel("k")->register_B(n_cols, x);
        smax.kernel("k")->register_C(n_rows, b);
        t = time_applies(&smax, "k", warm, reps);
        return 0;
    });
    return rc == 0 ? t : -1.0;
}

// ------------------------------------------------------------------ SpTRSM --
int ref_sptrsm(int vbits, int row_major, int upper, uint64_t n_rows,
               uint64_t n_cols, uint64_t nnz, int *col, int *row_ptr,
               void *val, uint64_t k, void *X, void *B) {
    return guarded([&] {
        SMAX::Interface smax;
        smax.register_kernel("k", SMAX::KernelType::SPTRSM,
                             SMAX::PlatformType::CPU, SMAX::IntType::INT32,
                             ftype(vbits));
        // SpTRSM has no set_mat_upper_triang override in the reference
        // (src/kernels/sptrsm.hpp:62-65): the call returns 1 and the flag
        // stays false, so `upper` can only select the lower solve.
        if (upper)
            smax.kernel("k")->set_mat_upper_triang(true);
        smax.kernel("k")->register_A(n_rows, n_cols, nnz, col, row_ptr, val);
        smax.kernel("k")->register_B(n_cols, k, X);
        smax.kernel("k")->register_C(n_rows, k, B);
        smax.kernel("k")->set_vec_row_major(row_major != 0);
        return smax.kernel("k")->run();
    });
}

double ref_time_sptrsm(int vbits, int row_major, uint64_t n_rows,
                       uint64_t n_cols, uint64_t nnz, int *col, int *row_ptr,
                       void *val, uint64_t k, void *X, void *B, int warm,
                       int reps) {
    double t = -1.0;
    int rc = guarded([&] {
        SMAX::Interface smax;
        smax.register_kernel("k", SMAX::KernelType::SPTRSM,
                             SMAX::PlatformType::CPU, SMAX::IntType::INT32,
                             ftype(vbits));
        smax.kernel("k")->register_A(n_rows, n_cols, nnz, col, row_ptr, val);
        smax.kernel("k")->register_B(n_cols, k, X);
        smax.kernel("k")->register_C(n_rows, k, B);
        smax.kernel("k")->set_vec_row_major(row_major != 0);
        t = time_applies(&smax, "k", warm, reps);
        return 0;
    });
    return rc == 0 ? t : -1.0;
}

// ------------------------------------------------------------- conversions --
int ref_convert_crs_to_scs(int vbits, uint64_t n_rows, uint64_t n_cols,
                           uint64_t nnz, const int *col, const int *row_ptr,
                           const void *val, uint64_t C, uint64_t sigma,
                           uint64_t *meta, int **chunk_ptr, int **chunk_lengths,
                           int **o_col, void **o_val, int **perm) {
    return guarded([&] {
        SMAX::Interface smax;
        ULL m[6] = {0, 0, 0, 0, 0, 0};
        if (vbits == 32) {
            float *ov = nullptr;
            smax.utils->convert_crs_to_scs<int, float, ULL>(
                n_rows, n_cols, nnz, col, row_ptr, (const float *)val, C, sigma,
                m[0], m[1], m[2], m[3], m[4], m[5], *chunk_ptr, *chunk_lengths,
                *o_col, ov, *perm);
            *o_val = ov;
        } else {
            double *ov = nullptr;
            smax.utils->convert_crs_to_scs<int, double, ULL>(
                n_rows, n_cols, nnz, col, row_ptr, (const double *)val, C,
                sigma, m[0], m[1], m[2], m[3], m[4], m[5], *chunk_ptr,
                *chunk_lengths, *o_col, ov, *perm);
            *o_val = ov;
        }
        for (int i = 0; i < 6; ++i)
            meta[i] = m[i];
        return 0;
    });
}

int ref_convert_crs_to_bcrs(int vbits, uint64_t n_rows, uint64_t n_cols,
                            uint64_t nnz, const int *col, const int *row_ptr,
                            const void *val, uint64_t bh, uint64_t bw,
                            uint64_t hpad, uint64_t wpad, int col_major,
                            uint64_t *meta, int **o_col, int **o_row_ptr,
                            void **o_val) {
    return guarded([&] {
        SMAX::Interface smax;
        ULL m[7] = {0, 0, 0, 0, 0, 0, 0};
        if (vbits == 32) {
            float *ov = nullptr;
            smax.utils->convert_crs_to_bcrs<int, float, ULL>(
                n_rows, n_cols, nnz, col, row_ptr, (const float *)val, m[0],
                m[1], m[2], m[3], m[4], m[5], m[6], *o_col, *o_row_ptr, ov, bh,
                bw, hpad, wpad, col_major != 0);
            *o_val = ov;
        } else {
            double *ov = nullptr;
            smax.utils->convert_crs_to_bcrs<int, double, ULL>(
                n_rows, n_cols, nnz, col, row_ptr, (const double *)val, m[0],
                m[1], m[2], m[3], m[4], m[5], m[6], *o_col, *o_row_ptr, ov, bh,
                bw, hpad, wpad, col_major != 0);
            *o_val = ov;
        }
        for (int i = 0; i < 7; ++i)
            meta[i] = m[i];
        return 0;
    });
}

// --------------------------------------------------- levels / permutations --
int ref_build_symmetric_crs(uint64_t n_rows, int *row_ptr, int *col,
                            int **sym_row_ptr, int **sym_col,
                            uint64_t *sym_nnz) {
    return guarded([&] {
        SMAX::Interface smax;
        ULL nz = 0;
        ULL n = n_rows;
        smax.utils->build_symmetric_crs<int, ULL>(row_ptr, col, n, *sym_row_ptr,
                                                  *sym_col, nz);
        *sym_nnz = nz;
        return 0;
    });
}

// lvl_ptr_out receives a new[] copy of the Interface's level pointer
// (src/utils/permutations.hpp:556-579); free it with ref_free_int.
int ref_generate_perm(int n_rows, int *row_ptr, int *col, int *perm,
                      int *inv_perm, const char *type, int *n_levels,
                      int **lvl_ptr_out) {
    return guarded([&] {
        SMAX::Interface smax;
        smax.utils->generate_perm<int>(n_rows, row_ptr, col, perm, inv_perm,
                                       std::string(type));
        *n_levels = smax.get_n_levels();
        *lvl_ptr_out = copy_new(smax.utils->uc->lvl_ptr, (size_t)*n_levels + 1);
        return 0;
    });
}

double ref_time_generate_perm(int n_rows, int *row_ptr, int *col, int *perm,
                              int *inv_perm, const char *type) {
    double t = -1.0;
    int rc = guarded([&] {
        SMAX::Interface smax;
        double t0 = now_s();
        smax.utils->generate_perm<int>(n_rows, row_ptr, col, perm, inv_perm,
                                       std::string(type));
        t = now_s() - t0;
        return 0;
    });
    return rc == 0 ? t : -1.0;
}

int ref_apply_mat_perm(int vbits, int n_rows, int *row_ptr, int *col,
                       void *val, int *p_row_ptr, int *p_col, void *p_val,
                       int *perm, int *inv_perm) {
    return guarded([&] {
        SMAX::Interface smax;
        if (vbits == 32)
            smax.utils->apply_mat_perm<int, float>(
                n_rows, row_ptr, col, (float *)val, p_row_ptr, p_col,
                (float *)p_val, perm, inv_perm);
        else
            smax.utils->apply_mat_perm<int, double>(
                n_rows, row_ptr, col, (double *)val, p_row_ptr, p_col,
                (double *)p_val, perm, inv_perm);
        return 0;
    });
}

int ref_apply_vec_perm(int vbits, int n, void *vec, void *vec_perm,
                       int *perm) {
    return guarded([&] {
        SMAX::Interface smax;
        if (vbits == 32)
            smax.utils->apply_vec_perm<float>(n, (float *)vec,
                                              (float *)vec_perm, perm);
        else
            smax.utils->apply_vec_perm<double>(n, (double *)vec,
                                               (double *)vec_perm, perm);
        return 0;
    });
}

// ------------------------------------------------------ solver applications --
// The loops of the reference's iterative-solver programs,
// examples/applications/jacobi/jacobi.cpp:14-58 and
// gauss_seidel/gauss_seidel.cpp:13-50, on a caller's matrix (the programs fix
// a 10x10 Poisson problem), driven through the reference's kernels the way the
// programs drive them: run() on CPU SpMV / SpTRSV kernels once per step, the
// vector arithmetic on the host as their helpers do it (subtract_vectors with
// an OpenMP loop, normalize_x and infty_vec_norm serial,
// applications_common.hpp:113-133, jacobi/utils.hpp:38-50).  FP64, as the
// programs.  hist receives up to hist_cap residuals and *n_checks their count;
// the return value is the seconds spent after the first residual, or -1.
namespace {

double app_norm(const double *v, uint64_t n) {
    double m = 0.0;
    for (uint64_t i = 0; i < n; ++i) {
        const double a = (v[i] >= 0) ? v[i] : -1 * v[i];
        if (a > m)
            m = a;
    }
    return m;
}

void app_subtract(double *out, const double *a, const double *b, uint64_t n) {
#pragma omp parallel for
    for (long long i = 0; i < (long long)n; ++i)
        out[i] = a[i] - 1.0 * b[i];
}

struct AppLog {
    double *hist;
    int cap;
    int count = 0;
    void add(double v) {
        if (count < cap)
            hist[count] = v;
        ++count;
    }
};

} // namespace

double ref_jacobi(uint64_t n, uint64_t nnz, const int *col, int *row_ptr, const double *val, const double *b,
                  double *x, double tol, int max_iters, int check_length, int *n_iters, double *final_norm,
                  double *hist, int hist_cap, int *n_checks) {
    double t = -1.0;
    int rc = guarded([&] {
        // peel_diag_crs (jacobi/utils.hpp:7-36) on a copy of the matrix
        std::vector<int> pc(col, col + nnz);
        std::vector<double> pv(val, val + nnz), D(n);
        for (uint64_t r = 0; r < n; ++r) {
            const int s = row_ptr[r], e = row_ptr[r + 1] - 1;
            int dj = -1;
            for (int j = s; j <= e; ++j)
                if ((uint64_t)pc[j] == r)
                    dj = j;
            if (dj < 0)
                throw std::runtime_error("No diag!");
            D[r] = pv[dj];
            if (std::abs(D[r]) < 1e-16)
                throw std::runtime_error("Zero diag!");
            if (dj != e) {
                std::swap(pc[dj], pc[e]);
                std::swap(pv[dj], pv[e]);
            }
        }
        std::vector<double> x_new(x, x + n), x_old(x, x + n), tmp(n), residual(n);
        SMAX::Interface smax;
        smax.register_kernel("tmp <- Ax", SMAX::KernelType::SPMV, SMAX::PlatformType::CPU);
        smax.kernel("tmp <- Ax")->register_A(n, n, nnz, pc.data(), row_ptr, pv.data());
        smax.kernel("tmp <- Ax")->register_B(n, x_new.data());
        smax.kernel("tmp <- Ax")->register_C(n, tmp.data());
        smax.register_kernel("x_new <- Ax_old", SMAX::KernelType::SPMV, SMAX::PlatformType::CPU);
        smax.kernel("x_new <- Ax_old")->register_A(n, n, nnz, pc.data(), row_ptr, pv.data());
        smax.kernel("x_new <- Ax_old")->register_B(n, x_old.data());
        smax.kernel("x_new <- Ax_old")->register_C(n, x_new.data());
        double *xo = x_old.data(), *xn = x_new.data();
        AppLog log{hist, hist_cap};
        auto check = [&] {
            smax.kernel("tmp <- Ax")->run();
            app_subtract(residual.data(), b, tmp.data(), n);
            return app_norm(residual.data(), n);
        };
        double norm = check();
        log.add(norm);
        int it = 0;
        const double t0 = now_s();
        while (norm > tol && it < max_iters) {
            smax.kernel("x_new <- Ax_old")->run();
            for (uint64_t i = 0; i < n; ++i) {
                const double diag_contrib = D[i] * xo[i];
                const double offdiag_sum = xn[i] - diag_contrib;
                xn[i] = (b[i] - offdiag_sum) / D[i];
            }
            smax.kernel("x_new <- Ax_old")->swap_operands();
            std::swap(xo, xn);
            ++it;
            if (it % check_length == 0) {
                norm = check();
                log.add(norm);
            }
        }
        t = now_s() - t0;
        std::memcpy(x, xo, sizeof(double) * n);
        *n_iters = it;
        *final_norm = norm;
        *n_checks = log.count;
        return 0;
    });
    return rc == 0 ? t : -1.0;
}

double ref_gauss_seidel(uint64_t n, uint64_t nnz, const int *col, const int *row_ptr, const double *val,
                        const double *b, double *x, double tol, int max_iters, int check_length, int *n_iters,
                        double *final_norm, double *hist, int hist_cap, int *n_checks) {
    double t = -1.0;
    int rc = guarded([&] {
        // extract_D_L_U (examples/examples_common.hpp:283-398): col <= row to
        // D+L, the rest to U, in-row order kept
        std::vector<int> arp(row_ptr, row_ptr + n + 1), acol(col, col + nnz);
        std::vector<double> aval(val, val + nnz);
        std::vector<int> lrp(n + 1, 0), urp(n + 1, 0), lcol, ucol;
        std::vector<double> lval, uval;
        for (uint64_t r = 0; r < n; ++r) {
            for (int j = arp[r]; j < arp[r + 1]; ++j) {
                if ((uint64_t)acol[j] <= r) {
                    lcol.push_back(acol[j]);
                    lval.push_back(aval[j]);
                } else {
                    ucol.push_back(acol[j]);
                    uval.push_back(aval[j]);
                }
            }
            lrp[r + 1] = (int)lcol.size();
            urp[r + 1] = (int)ucol.size();
        }
        std::vector<double> xv(x, x + n), tmp(n), residual(n);
        SMAX::Interface smax;
        smax.register_kernel("tmp <- Ax", SMAX::KernelType::SPMV, SMAX::PlatformType::CPU);
        smax.kernel("tmp <- Ax")->register_A(n, n, nnz, acol.data(), arp.data(), aval.data());
        smax.kernel("tmp <- Ax")->register_B(n, xv.data());
        smax.kernel("tmp <- Ax")->register_C(n, tmp.data());
        smax.register_kernel("tmp <- Ux", SMAX::KernelType::SPMV, SMAX::PlatformType::CPU);
        smax.kernel("tmp <- Ux")->register_A(n, n, (uint64_t)ucol.size(), ucol.data(), urp.data(), uval.data());
        smax.kernel("tmp <- Ux")->register_B(n, xv.data());
        smax.kernel("tmp <- Ux")->register_C(n, tmp.data());
        smax.register_kernel("solve", SMAX::KernelType::SPTRSV);
        smax.kernel("solve")->register_A(n, n, (uint64_t)lcol.size(), lcol.data(), lrp.data(), lval.data());
        smax.kernel("solve")->register_B(n, xv.data());
        smax.kernel("solve")->register_C(n, tmp.data());
        AppLog log{hist, hist_cap};
        auto check = [&] {
            smax.kernel("tmp <- Ax")->run();
            app_subtract(residual.data(), b, tmp.data(), n);
            return app_norm(residual.data(), n);
        };
        double norm = check();
        log.add(norm);
        int it = 0;
        const double t0 = now_s();
        while (norm > tol && it < max_iters) {
            smax.kernel("tmp <- Ux")->run();
            app_subtract(tmp.data(), b, tmp.data(), n);
            smax.kernel("solve")->run();
            ++it;
            if (it % check_length == 0) {
                norm = check();
                log.add(norm);
            }
        }
        t = now_s() - t0;
        std::memcpy(x, xv.data(), sizeof(double) * n);
        *n_iters = it;
        *final_norm = norm;
        *n_checks = log.count;
        return 0;
    });
    return rc == 0 ? t : -1.0;
}

// ------------------------------------------------------ Matrix Market reader --
// The examples' reader, COOMatrix::read_from_mtx without fast_matrix_market
// (examples/matrix_structs.hpp:52-180), then CRSMatrix::convert_coo_to_crs
// (:338-387), FP64.  The arrays are new[] (ref_free_int / ref_free_val).
int ref_read_mtx(const char *path, uint64_t *n_rows, uint64_t *n_cols, uint64_t *nnz, int **row_ptr, int **col,
                 double **val) {
    return guarded([&] {
        COOMatrix coo;
        coo.read_from_mtx(path);
        CRSMatrix<int, double> crs;
        crs.convert_coo_to_crs(&coo);
        *n_rows = crs.n_rows;
        *n_cols = crs.n_cols;
        *nnz = crs.nnz;
        *row_ptr = crs.row_ptr;
        *col = crs.col;
        *val = crs.val;
        crs.row_ptr = nullptr;
        crs.col = nullptr;
        crs.val = nullptr;
        return 0;
    });
}

} // extern "C"
