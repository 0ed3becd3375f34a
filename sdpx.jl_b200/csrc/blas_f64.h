// Host launchers for the FP64 tile kernels (blas_f64.cu).
#pragma once
#include <algorithm>
#include <cmath>

#include "common.cuh"

namespace sdpx {

// C = alpha·A·B + beta·C over the K range selected by `mode` (KRange).
// a_kcontig / b_kcontig state which index of each operand is contiguous.
void gemm_f64(const Opnd& A, bool a_kcontig, const Opnd& B, bool b_kcontig, const OutDesc& C,
              double alpha, double beta, int mode, bool big, cudaStream_t st);

// Up to kGemmGroups independent products C_g = alpha_g·A_g·B_g + beta_g·C_g
// (K range mode_g each, the same operand contiguity for all) in one launch:
// the tiles of every product in one grid, each tile computed exactly as
// gemm_f64 computes it (the same tile shape is chosen by the same rule).
constexpr int kGemmGroups = 8;
struct GemmGroups {
  int n = 0;
  Opnd A[kGemmGroups], B[kGemmGroups];
  OutDesc C[kGemmGroups];
  double alpha[kGemmGroups], beta[kGemmGroups];
  int mode[kGemmGroups];
};
void gemm_f64_grouped(const GemmGroups& g, bool a_kcontig, bool b_kcontig, cudaStream_t st);

// T ← T·L in place, L lower triangular with explicit zeros above the diagonal.
void trmm_right_lower_inplace_f64(const Opnd& T, const Opnd& L, const OutDesc& C, cudaStream_t st);

struct SyrkPlan {
  int bm = 128;
  int ntri = 0, nchunk = 0, kchunk = 0;
  size_t partial_doubles = 0;
};
SyrkPlan plan_syrk_f64(int m, long long K, int sm_count);
// Lower tiles of S(m×m, ld lds) = P̂ᵀP̂ (+ beta·S), P̂ given as a K-contiguous operand.
void syrk_lower_f64(const Opnd& P, const SyrkPlan& plan, double* partial, double* S, long long lds,
                    int m, double beta, cudaStream_t st);

// Allocation-free S = PᵀP (lower tiles then mirrored by the caller), split-K
// scratch in a fixed device array; throws std::invalid_argument when m > 2048.
void syrk_lower_f64_noalloc(const double* P, long long K, int m, double* S, cudaStream_t st);
size_t gram_noalloc_capacity_doubles();

}  // namespace sdpx
