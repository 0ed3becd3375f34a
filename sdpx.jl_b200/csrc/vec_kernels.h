// Host launchers of the memory-bound kernels (vec_kernels.cu).
#pragma once
#include <algorithm>

#include "common.cuh"

namespace sdpx {

struct TrialDesc {
  const double* X;
  const double* dX;
  double* out;
  double t;
  int k;
};
void make_trials_list(const TrialDesc* d_list, int n, int kmax, cudaStream_t st);

void gemv_n(const double* A, long long K, int m, const double* x, double* out, double* part,
            int chunks, cudaStream_t st);
void gemv_t(const double* A, long long K, int m, const double* z, double alpha, const double* base,
            double beta, double* out, cudaStream_t st);
// The same products as compensated (Dot2) sums rounded once, for the
// residuals: out = 𝒜x − X − C (X, C may be null; part holds 2·chunks·K
// doubles) and out = alpha·𝒜ᵀz + beta·base.
void gemv_n_acc(const double* A, long long K, int m, const double* x, const double* X,
                const double* C, double* out, double* part, int chunks, cudaStream_t st);
void gemv_n_sym_acc(const double* Ap, long long Kt, int m, const double* x, const long long* lo,
                    const long long* up, const double* X, const double* C, double* out,
                    double* part, int chunks, cudaStream_t st);
void gemv_t_acc(const double* A, long long K, int m, const double* z, double alpha,
                const double* base, double beta, double* out, cudaStream_t st);
// Lower-triangle copy of the constraint matrix (Kt kept rows per column):
// pack_rows gathers it, gemv_n_sym writes Ap·x to both stacked positions
// lo[q] and up[q] of every kept row, fold_sym folds a stacked vector onto the
// kept rows (z[lo] + z[up] off the diagonal) for Apᵀ·zf = 𝒜ᵀz.
void pack_rows(const double* A, long long K, int m, const long long* rows, long long Kt, double* Ap,
               cudaStream_t st);
void gemv_n_sym(const double* Ap, long long Kt, int m, const double* x, const long long* lo,
                const long long* up, double* out, double* part, int chunks, cudaStream_t st);
void fold_sym(long long Kt, const double* z, const long long* lo, const long long* up, double* zf,
              cudaStream_t st);
void axpbypcz(long long n, double a, const double* x, double b, const double* y, double c,
              const double* z, double* out, cudaStream_t st);
void combine(long long n, double* x, double t, const double* d, cudaStream_t st);
void scale(long long n, double* x, double f, cudaStream_t st);
void absmax(long long n, const double* x, double* out, cudaStream_t st);
void seg_dot(const long long* d_off, const long long* d_len, int nseg, int parts, const double* x,
             const double* dx, double tx, const double* y, const double* dy, double ty, double* part,
             double* out, cudaStream_t st);
void block_trace(const long long* d_off, const int* d_k, int nseg, const double* M, double* out,
                 cudaStream_t st);
void add_diag(const long long* d_off, const int* d_k, int nseg, int kmax, double* M,
              const double* d_shifts, double uniform, cudaStream_t st);
void symmetrize(const long long* d_off, const int* d_k, int nseg, int kmax, double* M,
                cudaStream_t st);
void gershgorin(const long long* d_off, const int* d_k, int nseg, int kmax, const double* M,
                double* d_cand, const long long* d_cand_off, double* d_scale, int* d_nonfinite,
                cudaStream_t st);
void diag_residual_R(int nd, long long od, const double* X, const double* Y, const double* mu_user,
                     const int* user, int use_affine, double* R, cudaStream_t st);
void diag_factor(int nd, long long od, const double* X, const double* Y, double* LX, double* MY,
                 int* fail, cudaStream_t st);
void diag_rhs_Z(int nd, long long od, const double* P, const double* Y, const double* R,
                const double* LX, double* Z, cudaStream_t st);
void diag_dY(int nd, long long od, const double* R, const double* dX, const double* Y,
             const double* LX, double* dY, cudaStream_t st);
void diag_corrector_R(int nd, long long od, const double* X, const double* Y, const double* dX,
                      const double* dY, const double* target_user, const int* user, double* R,
                      cudaStream_t st);
void diag_panel(long long K, int m, int nd, long long od, const double* A, const double* LX,
                const double* MY, double* Pc, cudaStream_t st);
void diag_trial(int nd, long long od, const double* X, const double* dX, const double* d_t, int nc,
                int margin, int* d_fail, cudaStream_t st);
void diag_ftb(int nd, long long od, const double* X, const double* dX, double* d_out,
              cudaStream_t st);
void make_trials(const long long* d_off, const int* d_k, const long long* d_trial_off, int nseg,
                 int kmax, const double* X, const double* dX, const double* d_t, int nc,
                 double* trials, cudaStream_t st);
void gather(long long n, const long long* map, const double* src, double* dst, cudaStream_t st);
void scatter(long long n, const long long* map, const double* src, double* dst, cudaStream_t st);
void mirror_lower(int m, double* S, cudaStream_t st);
void copy_reg(int m, const double* S, double* Sf, double reg, cudaStream_t st);
void symv_full(int m, const double* S, const double* x, double alpha, const double* b, double beta,
               double* y, cudaStream_t st);
void ruiz_rowmax_dense(const double* A, long long K, int m, long long off, int k, double* rn,
                       cudaStream_t st);
void ruiz_rowmax_diag(const double* A, long long K, int m, long long od, int nd, double* rn,
                      cudaStream_t st);
void ruiz_congruence_dense(double* A, long long K, int m, long long off, int k, const double* e,
                           cudaStream_t st);
void ruiz_congruence_diag(double* A, long long K, int m, long long od, int nd, const double* e,
                          cudaStream_t st);
void colmax(const double* A, long long K, int m, double* out, cudaStream_t st);
void scale_cols(double* A, long long K, int m, const double* s, cudaStream_t st);

}  // namespace sdpx
