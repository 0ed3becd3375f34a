// Device side of the batched small-SDP engine (batch.cu): one CTA per
// instance per phase, every instance one PSD block of order k ≤ 64 with m ≤ 256
// constraints.  Instance matrices live in HBM at per-instance offsets; the
// k×k work of a phase runs in shared memory.  The arithmetic of each phase is
// the single-instance path's (the same Newton-step stages of src/step.jl and
// src/kernels/threaded.jl restated for one block): residuals and block factors,
// the Schur panel P̂_j = L_X⁻¹A_jL_Y and S = P̂P̂ᵀ, the Schur Cholesky with
// the reference's regularisation retries, the right-hand sides, the direction
// blocks, the fraction-to-boundary bisection, refinement residuals, the
// backtracking line search with its Cholesky margin and the update.
#pragma once
#include <cuda_runtime.h>

#include "common.cuh"

namespace sdpx {
namespace batch {

constexpr int kMaxK = 64;
constexpr int kMaxM = 256;
constexpr int kThreads = 256;

// Per-instance layout (element offsets into the pooled arrays).
struct Inst {
  int k, m;
  long long kk_off;   // k² arrays: X, Y, C, P, R, LX, LY, W, dX, dY, Z, Xb, Yb
  long long m_off;    // m arrays: c, x, dx, d, r, rho, xb, dxb
  long long mm_off;   // m² arrays: S, LS
  long long a_off;    // m·k² arrays: A (rows vec(A_j)), the Schur panel P̂
};

struct Pool {
  const Inst* inst;
  const double* A;
  double* Ph;
  const double* C;
  const double* c;
  double *X, *Y, *P, *R, *LX, *LY, *W, *dX, *dY, *Z, *Xb, *Yb;
  double *x, *dx, *d, *r, *rho, *xb, *dxb;
  double *S, *LS;
  long long kq;  // stride of one k×k matrix slot in shared memory (kmax² of the pool)
};

// |v| with NaN read as +inf, so a poisoned value never passes a max-norm test.
__device__ __forceinline__ double abs_nan_inf(double v) {
  const double a = fabs(v);
  return (a == a) ? a : 1.0 / 0.0;
}

// ------------------------------------------------------------ reductions --
__device__ inline double cta_sum(double v, double* red) { return block_sum(v, red); }
__device__ inline double cta_max(double v, double* red) { return block_max(v, red); }

// ------------------------------------------------------ small factorisations
// In-place lower Cholesky of the k×k column-major M (shared memory), the
// unblocked right-looking algorithm (LAPACK potf2's operation order per column).
// Returns false at the first pivot that is not > 0 (or NaN); the upper
// triangle is left as it was.  Writes min/max |L_jj| to *dmin/*dmax on success.
__device__ bool cta_chol(double* M, int k, double* sflag, double* dmin, double* dmax) {
  for (int j = 0; j < k; ++j) {
    if (threadIdx.x == 0) {
      const double d = M[j + j * k];
      sflag[0] = d;
      sflag[1] = (d > 0.0) ? sqrt(d) : 0.0;
    }
    __syncthreads();
    const double piv = sflag[0];
    if (!(piv > 0.0)) return false;
    const double ljj = sflag[1];
    const double inv = 1.0 / ljj;
    for (int i = j + 1 + threadIdx.x; i < k; i += blockDim.x) M[i + j * k] *= inv;
    if (threadIdx.x == 0) M[j + j * k] = ljj;
    __syncthreads();
    const int rem = k - j - 1;
    for (int e = threadIdx.x; e < rem * rem; e += blockDim.x) {
      const int ii = j + 1 + e % rem, ll = j + 1 + e / rem;
      if (ii >= ll) M[ii + ll * k] -= M[ii + j * k] * M[ll + j * k];
    }
    __syncthreads();
  }
  if (dmin) {
    if (threadIdx.x == 0) {
      double mn = fabs(M[0]), mx = mn;
      for (int j = 1; j < k; ++j) {
        mn = fmin(mn, fabs(M[j + j * k]));
        mx = fmax(mx, fabs(M[j + j * k]));
      }
      sflag[0] = mn;
      sflag[1] = mx;
    }
    __syncthreads();
    *dmin = sflag[0];
    *dmax = sflag[1];
    __syncthreads();
  }
  return true;
}

// W = L⁻¹ (lower, k×k): one thread per column, forward substitution.
__device__ void cta_trinv(const double* L, double* W, int k) {
  for (int e = threadIdx.x; e < k * k; e += blockDim.x) W[e] = 0.0;
  __syncthreads();
  for (int c = threadIdx.x; c < k; c += blockDim.x) {
    W[c + c * k] = 1.0 / L[c + c * k];
    for (int r = c + 1; r < k; ++r) {
      double s = 0.0;
      for (int p = c; p < r; ++p) s += L[r + p * k] * W[p + c * k];
      W[r + c * k] = -s / L[r + r * k];
    }
  }
  __syncthreads();
}

// C = op(A)·B for k×k column-major operands; ta: A transposed.
__device__ void cta_gemm(const double* A, bool ta, const double* B, double* C, int k) {
  for (int e = threadIdx.x; e < k * k; e += blockDim.x) {
    const int r = e % k, c = e / k;
    double s = 0.0;
    if (ta)
      for (int p = 0; p < k; ++p) s += A[p + r * k] * B[p + c * k];
    else
      for (int p = 0; p < k; ++p) s += A[r + p * k] * B[p + c * k];
    C[e] = s;
  }
  __syncthreads();
}

// PD test of M = X + t·dX (copied into scratch) with the Cholesky margin
// min|L_jj| > ratio·max|L_jj| when ratio > 0 (`trial_has_cholesky_margin!`,
// src/kernels/generic.jl:318-340; ratio 0: `trial_isposdef`).
__device__ bool cta_trial(const double* X, const double* dX, double t, int k, double ratio,
                          double* M, double* sflag) {
  for (int e = threadIdx.x; e < k * k; e += blockDim.x) M[e] = X[e] + t * dX[e];
  __syncthreads();
  double mn = 0.0, mx = 0.0;
  const bool ok = cta_chol(M, k, sflag, ratio > 0.0 ? &mn : nullptr, &mx);
  __syncthreads();
  if (!ok) return false;
  if (!(ratio > 0.0)) return true;
  return isfinite(mn) && isfinite(mx) && mx > 0.0 && mn > ratio * mx;
}

// `fraction_to_boundary_bound!` for k ≥ 3 (src/kernels/generic.jl:350-422):
// 1 when the full step keeps X + dX positive definite, else the lower end of
// a bisection of at most 64 steps.
__device__ double cta_ftb(const double* X, const double* dX, int k, double* M, double* sflag) {
  if (cta_trial(X, dX, 1.0, k, 0.0, M, sflag)) return 1.0;
  double lo = 0.0, hi = 1.0;
  for (int it = 0; it < 64; ++it) {
    const double mid = (lo + hi) / 2.0;
    // Once [lo, hi] holds no double strictly inside, every further midpoint is
    // hi (a failing point) or lo > 0 (a passing one): lo no longer changes.
    if (mid == hi || (mid == lo && lo > 0.0)) break;
    if (cta_trial(X, dX, mid, k, 0.0, M, sflag)) lo = mid;
    else hi = mid;
  }
  return lo;
}

}  // namespace batch
}  // namespace sdpx
