// Double-double (Float64x2) kernels over the stacked layout: the operator
// passes 𝒜·v and 𝒜ᵀ·z, k×k block products of every dense block, and the
// elementwise and block-structured operations the extended-precision
// residuals need.  A double-double array is a pair (hi, lo) of double arrays
// of the same shape; a NULL lo reads as zero (a double operand).
#pragma once
#include <cuda_runtime.h>

namespace sdpx {

// out = 𝒜·v (K rows); v has m entries; partials ph/pl hold chunks·K each.
void dd_gemv_n(const double* A, long long K, int m, const double* vh, const double* vl,
               double* ph, double* pl, int chunks, double* oh, double* ol, cudaStream_t st);
// out_i = Σ_r 𝒜[r, i]·z_r (m entries).
void dd_gemv_t(const double* A, long long K, int m, const double* zh, const double* zl,
               double* oh, double* ol, cudaStream_t st);
// C_b = A_b·B_b for every dense block b (k_b×k_b column-major at offset doff[b]).
void dd_gemm_blocks(const long long* doff, const int* dk, int nb, int kmax, const double* Ah,
                    const double* Al, const double* Bh, const double* Bl, double* Ch, double* Cl,
                    cudaStream_t st);
// C = sa·A + sb·B elementwise (n entries; B may be NULL).
void dd_axpby(long long n, double sa, const double* ah, const double* al, double sb,
              const double* bh, const double* bl, double* ch, double* cl, cudaStream_t st);
// out[0], out[1] = ⟨a, b⟩ in double-double (device); null low halves read as 0.
void dd_dot(long long n, const double* ah, const double* al, const double* bh, const double* bl,
            double* out, cudaStream_t st);
// C_b = I − A_b per dense block.
void dd_eye_minus_blocks(const long long* doff, const int* dk, int nb, int kmax, const double* ah,
                         const double* al, double* ch, double* cl, cudaStream_t st);
// C_b = (A_b + A_bᵀ)/2 per dense block (C distinct from A).
void dd_sym_blocks(const long long* doff, const int* dk, int nb, int kmax, const double* ah,
                   const double* al, double* ch, double* cl, cudaStream_t st);
// 1×1 group rows [od, od + nd): C = 1 / X and C = A ⊙ B.
void dd_diag_recip(int nd, long long od, const double* xh, const double* xl, double* ch,
                   double* cl, cudaStream_t st);
void dd_diag_mul(int nd, long long od, const double* ah, const double* al, const double* bh,
                 const double* bl, double* ch, double* cl, cudaStream_t st);

}  // namespace sdpx
