// Kernels of the equality block of the KKT system (n > 0 equality rows
// Bᵀx = b, B m×n column-major): column normalisation of B̃ = L_S⁻¹B, the exact
// duplicate-column test, the column-pivoted Householder QR of the
// rank-revealing fallback and the small triangular solves with either factor.
#pragma once
#include <cuda_runtime.h>

namespace sdpx {

// B̃[:, j] *= s_j with s_j = 1/‖B̃[:, j]‖∞ (1 for a zero column or an
// overflowing reciprocal), s written to scale[j].
void eq_normalize_columns(int m, int n, double* Bt, double* scale, cudaStream_t st);

// Position-sensitive 64-bit fingerprint of every column (signed zeros equal):
// equal columns have equal fingerprints.
void eq_column_fingerprints(int m, int n, const double* Bt, unsigned long long* fp,
                            cudaStream_t st);
// equal[q] = 1 when columns pairs[2q] and pairs[2q+1] agree entry by entry
// (== on doubles: −0 equals +0, NaN equals nothing).
void eq_columns_equal(int m, const double* Bt, const int* pairs, int npairs, int* equal,
                      cudaStream_t st);

// In-place column-pivoted Householder QR of A (m×n, ld lda) by one CTA:
// column norms recomputed exactly at every step, the first largest column
// becomes the pivot.  perm[j] = source column of position j, rdiag[j] = R_jj;
// R is left in the upper triangle.  Work O(m·n²); meant for the rank-deficient
// fallback.
void eq_qr_pivoted(int m, int n, double* A, int lda, int* perm, double* rdiag, double* colnorm,
                   cudaStream_t st);

// out = M⁻ᵀM⁻¹-solve on the leading rank×rank block: z = rhs[perm[0:rank]],
// M z' = z (forward), Mᵀ z'' = z' (backward), out[perm[i]] = z''[i] for
// i < rank and 0 for the dependent positions.  M is lower triangular: the
// Cholesky factor (upper = 0, ld n) or Rᵀ of the QR (upper = 1: M(r, c) is
// read as R(c, r) of the packed factor, ld lda).  One CTA; z is scratch (n).
void eq_small_solve(int n, int rank, const double* T, int ldt, int upper, const int* perm,
                    const double* rhs, double* out, double* z, cudaStream_t st);

// q[i] = scale[i]·p[i] − q[i].
void eq_scaled_rhs(int n, const double* scale, const double* p, double* q, cudaStream_t st);
// v[i] *= scale[i].
void eq_scale_vec(int n, const double* scale, double* v, cudaStream_t st);
// B[i + j·m] /= s[i] (equilibration of the equality rows).
void eq_scale_rows(int m, int n, double* B, const double* s, cudaStream_t st);
// out[0] = Σ a[i]·b[i] (one CTA, fixed order).
void eq_dot(int n, const double* a, const double* b, double* out, cudaStream_t st);
// perm[i] = i.
void eq_iota(int n, int* perm, cudaStream_t st);

}  // namespace sdpx
