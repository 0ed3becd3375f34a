// Device passes of the cold-path result certificate (certificate.cu).
#pragma once
#include "common.cuh"

namespace sdpx {

// Primal block backward errors over the stacked rows of A (K×m):
//   R_r = Σ_i A[r,i]·x_i − X_r − C_r,
//   nominal_r = |C_r| + Σ_i |A[r,i]|,  realized_r = |X_r| + |C_r| + Σ_i |A[r,i]|·|x_i|;
// writes |R_r|, |R_r|/(nominal+realized) and |R_r|/realized (0/0 → 0, r/0 → ∞).
// part: 3·chunks·K scratch.
void cert_primal_rows(const double* A, long long K, int m, const double* x, const double* X,
                      const double* C, double* part, int chunks, double* absR, double* mixed,
                      double* strict, cudaStream_t st);

// Dual backward errors per variable i:
//   v_i = c_i − Σ_r A[r,i]·Y_r − Σ_j B[i,j]·y_j, nominal_i = |c_i| + Σ_r |A[r,i]| + Σ_j |B[i,j]|,
//   realized_i = |c_i| + Σ_r |A[r,i]|·|Y_r| + Σ_j |B[i,j]|·|y_j|
// (the B terms only for n > 0 equality rows, B m×n column-major).
void cert_dual_cols(const double* A, long long K, int m, const double* Y, const double* c,
                    double* absv, double* mixed, double* strict, cudaStream_t st,
                    const double* B = nullptr, int n = 0, const double* y = nullptr);

// Equality backward errors per row j of Bᵀx = b: |Σ_i B[i,j]x_i − b_j| and its
// mixed / strict componentwise ratios with nominal |b_j| + Σ|B| and realized
// |b_j| + Σ|B|·|x|.
void cert_equality_rows(const double* B, int m, int n, const double* x, const double* b,
                        double* absr, double* mixed, double* strict, cudaStream_t st);

// out[0] += Σ a·b (single CTA, fixed order within the launch); out[1] += count of
// non-finite entries of a (as a double).
void cert_dot(long long n, const double* a, const double* b, double* out, cudaStream_t st);

// Per dense block b (stacked offset off[b], order k[b]) of M: out[3b] = number of
// non-finite entries, out[3b+1] = max |M|, out[3b+2] = max |M_rc − M_cr|.
void cert_block_stats(const long long* off, const int* k, int nb, const double* M, double* out,
                      cudaStream_t st);

// S_b = (M_b + M_bᵀ)/2 + shift[b]·I into the same offsets of S.
void cert_sym_shift(const long long* off, const int* k, int nb, int kmax, const double* M,
                    const double* shift, double* S, cudaStream_t st);

}  // namespace sdpx
