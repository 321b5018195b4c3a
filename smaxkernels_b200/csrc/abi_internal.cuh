// abi_internal.cuh -- helpers shared by the translation units that implement
// the kernel-object part of the C ABI (abi.cu, adjoint_abi.cu, refine.cu,
// autotune.cu).
#pragma once

#include "kernel_obj.cuh"

namespace smax {

// rows * k of a level below which it joins a single-CTA merged run
constexpr int kDefaultLevelMerge = 4096;

void require(bool c, int code, const char *msg);
smax_kernel_s *K(smax_kernel k);
// synchronises the kernel's stream and turns a device-reported error into an Error
void read_status(smax_kernel_s *k);
DevStatus *dstatus(smax_kernel_s *k);
bool is_tri(const smax_kernel_s *k);
// builds (or reuses) the level schedule of a triangular solve
void tri_plan(smax_kernel_s *k);
// device addresses of the registered B and C (+ element offsets)
const void *dev_b(smax_kernel_s *k, uint64_t off);
void *dev_c(smax_kernel_s *k, uint64_t off);
// the level-merge threshold in effect for the kernel's solve mode
inline int tri_merge_rows(const smax_kernel_s *k) {
    return k->solve_mode == SMAX_SOLVE_PER_LEVEL ? 0 : (k->level_merge >= 0 ? k->level_merge : kDefaultLevelMerge);
}

// the launches of one apply of an initialized kernel (SpMV, SpMM, SpTRSV,
// SpTRSM), without the stopwatch events
void apply_core(smax_kernel_s *k, uint64_t b_off, uint64_t c_off);
// builds the plans of both CRS SpMV kernels for the device copy of A
void build_crs_plans(smax_kernel_s *k);

// FP32 solve refined with FP64 residuals (refine.cu); B = right-hand side,
// X = solution, both FP64 device arrays of n_rows
void refine_solve(smax_kernel_s *k, const double *B, double *X);

}  // namespace smax
