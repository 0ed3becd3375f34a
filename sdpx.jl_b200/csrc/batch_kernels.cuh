// Device side of the batched small-SDP engine (batch.cu): one CTA per
// instance per phase, every instance one PSD block of order k ≤ 64 with m ≤ 256
// constraints.  Instance matrices live in HBM at per-instance offsets; the
// k×k work of a phase runs in shared memory.  The arithmetic of each phase is
// the single-instance path's (the same Newton-step stages of src/step.jl and
// src/kernels/threaded.jl restated for one block): residuals and block factors,
// the Schur panel P̂_j = L_X⁻¹A_jL_Y and S = P̂P̂ᵀ, the Schur Cholesky with
// the reference's regularisation retries, the right-hand sides, the direction
// blocks, the fraction-to-boundary bisection, refinement residuals, the
// backtracking line search with its Cholesky margin and the update.  The
// step-length trials run eight at a time, one warp each.
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
  long long kp;  // stride of one packed lower-triangle slot (kmax(kmax+1)/2)
  // Float64x2 mode: low halves of the double-double arrays (hi halves are the
  // FP64 arrays above), X⁻¹ in double-double and the low half of the panel.
  double *Pl, *Rl, *Zl, *dl, *rl, *dxl, *dxbl, *rhol, *Sl, *LSl, *Xih, *Xil, *Gl;
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

// ------------------------------------------ concurrent trials, one per warp
// The step-length phases test several step lengths of one instance at once:
// the CTA stages the lower triangles of X and dX in shared memory (packed,
// column-major: column j starts at pk_off(j, k)), and each warp factors its own
// trial matrix M = X + t·dX in its own packed slot with warp barriers only.
// Per element the operations and their order are those of cta_chol (pivot,
// scale by 1/L_jj, rank-one update column by column), so a trial's outcome is
// the same.
constexpr int kTrialWarps = kThreads / 32;

__device__ __forceinline__ int pk_off(int j, int k) { return j * k - (j * (j - 1)) / 2; }

// Packed lower triangles of the k×k column-major X and dX (global) into Xp,
// dXp (shared); called by the whole CTA.
__device__ void cta_load_packed(const double* X, const double* dX, int k, double* Xp,
                                double* dXp) {
  __syncthreads();  // the previous side's trials are done with Xp, dXp
  for (int e = threadIdx.x; e < k * k; e += blockDim.x) {
    const int i = e % k, j = e / k;
    if (i >= j) {
      const int p = pk_off(j, k) + i - j;
      Xp[p] = X[e];
      dXp[p] = dX[e];
    }
  }
  __syncthreads();
}

// Next packed position 32 further down the trailing triangle: row i of
// column c, columns holding rows c..k-1.
__device__ __forceinline__ void pk_advance(int& c, int& i, int k) {
  i += 32;
  while (i >= k && c < k - 1) {
    i = i - k + c + 1;
    ++c;
  }
}

// Is Xp + t·dXp positive definite (and, for ratio > 0, min|L_jj| > ratio·max|L_jj|)?
// Called by all 32 lanes of a warp.
__device__ bool warp_trial(const double* __restrict__ Xp, const double* __restrict__ dXp,
                           double t, int k, double ratio, double* __restrict__ slot) {
  const int lane = threadIdx.x & 31;
  const int n = k * (k + 1) / 2;
#pragma unroll 4
  for (int p = lane; p < n; p += 32) slot[p] = Xp[p] + t * dXp[p];
  __syncwarp();
  double mn = 0.0, mx = 0.0;
  for (int j = 0; j < k; ++j) {
    const int oj = pk_off(j, k) - j;  // slot[oj + i] = M(i, j)
    const double d = slot[oj + j];
    if (!(d > 0.0)) return false;  // every lane read the same pivot
    const double ljj = sqrt(d);
    const double inv = 1.0 / ljj;
    mn = j == 0 ? ljj : fmin(mn, ljj);
    mx = j == 0 ? ljj : fmax(mx, ljj);
    __syncwarp();  // the pivot is read before lane 0 overwrites it
    for (int i = j + 1 + lane; i < k; i += 32) slot[oj + i] *= inv;
    if (lane == 0) slot[oj + j] = ljj;
    __syncwarp();
    // M(i, c) −= L(i, j)·L(c, j) over the trailing triangle c ≥ j+1, i ≥ c:
    // lanes walk its packed positions 32 apart, four independent updates in
    // flight per lane (their targets are distinct and column j is read only).
    const int r = k - j - 1;
    const int T = r * (r + 1) / 2;
    int c = j + 1, i = j + 1 + lane;
    while (i >= k && c < k - 1) {
      i = i - k + c + 1;
      ++c;
    }
    for (int q = lane; q < T; q += 128) {
      int cc[4], ii[4];
      cc[0] = c;
      ii[0] = i;
#pragma unroll
      for (int u = 1; u < 4; ++u) {
        pk_advance(c, i, k);
        cc[u] = c;
        ii[u] = i;
      }
      pk_advance(c, i, k);
      double tv[4], a[4], b[4];
#pragma unroll
      for (int u = 0; u < 4; ++u)
        if (q + 32 * u < T) {
          tv[u] = slot[pk_off(cc[u], k) - cc[u] + ii[u]];
          a[u] = slot[oj + ii[u]];
          b[u] = slot[oj + cc[u]];
        }
#pragma unroll
      for (int u = 0; u < 4; ++u)
        if (q + 32 * u < T) slot[pk_off(cc[u], k) - cc[u] + ii[u]] = tv[u] - a[u] * b[u];
    }
    __syncwarp();
  }
  if (!(ratio > 0.0)) return true;
  return isfinite(mn) && isfinite(mx) && mx > 0.0 && mn > ratio * mx;
}

// `fraction_to_boundary_bound!` (src/kernels/generic.jl:350-422) with the
// bisection evaluated as a tree: each round tests the 7 midpoints of the next
// three bisection steps at once (warps 0..6; warp 7 tests the full step in
// the first round) and walks the tree, so the result is the sequential
// bisection's: 1 if X + dX is positive definite, else the lower end after at
// most 64 steps, stopping once [lo, hi] holds no double strictly inside.
// Called by the whole CTA (kThreads threads); sm: 2 + kTrialWarps packed
// slots of stride kp (X, dX, the trials); flags: kTrialWarps ints in shared
// memory.
__device__ double cta_ftb_tree(const double* X, const double* dX, int k, double* sm,
                               long long kp, int* flags) {
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  double* Xp = sm;
  double* dXp = sm + kp;
  double* slot = sm + (2 + w) * kp;
  cta_load_packed(X, dX, k, Xp, dXp);
  double lo = 0.0, hi = 1.0;
  int done = 0;
  bool first = true;
  while (true) {
    const int depth = min(3, 64 - done);
    const int npts = (1 << depth) - 1;
    double los[7], his[7], pts[7];
    los[0] = lo;
    his[0] = hi;
#pragma unroll
    for (int n = 0; n < 7; ++n) {
      if (n >= npts) break;
      pts[n] = (los[n] + his[n]) / 2.0;
      const int l2 = 2 * n + 1, r2 = 2 * n + 2;
      if (l2 < npts) los[l2] = los[n], his[l2] = pts[n];
      if (r2 < npts) los[r2] = pts[n], his[r2] = his[n];
    }
    if (w < npts) {
      const bool ok = warp_trial(Xp, dXp, pts[w], k, 0.0, slot);
      if (lane == 0) flags[w] = ok ? 1 : 0;
    } else if (first && w == kTrialWarps - 1) {
      const bool ok = warp_trial(Xp, dXp, 1.0, k, 0.0, slot);
      if (lane == 0) flags[w] = ok ? 1 : 0;
    }
    __syncthreads();
    int f[kTrialWarps];
#pragma unroll
    for (int n = 0; n < kTrialWarps; ++n) f[n] = flags[n];
    __syncthreads();  // every thread has its copy before the next round writes
    if (first) {
      first = false;
      if (f[kTrialWarps - 1]) return 1.0;
    }
    int node = 0;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      if (node >= npts) break;
      if (f[node]) {
        lo = pts[node];
        node = 2 * node + 2;
      } else {
        hi = pts[node];
        node = 2 * node + 1;
      }
      ++done;
    }
    const double mid = (lo + hi) / 2.0;
    if (done >= 64 || mid == hi || (mid == lo && lo > 0.0)) return lo;
  }
}

// Backtracking (src/kernels/threaded.jl:1751-1818): the first t of 1, γ, γ², …
// whose trial passes (Cholesky and, for ratio > 0, the diagonal-ratio margin),
// or the first t below min_step; kTrialWarps candidates per round, one per
// warp.  Called by the whole CTA.  γ ∈ (0, 1) reaches min_step > 0 long
// before the round guard, which bounds the loop for any other input.  sm and
// flags as for cta_ftb_tree.
__device__ double cta_backtrack(const double* X, const double* dX, int k, double gamma,
                                double min_step, double ratio, double* sm, long long kp,
                                int* flags) {
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  double* Xp = sm;
  double* dXp = sm + kp;
  double* slot = sm + (2 + w) * kp;
  cta_load_packed(X, dX, k, Xp, dXp);
  double t_next = 1.0;
  for (int round = 0; round < 512; ++round) {
    double cand[kTrialWarps];
    int nc = 0;
    double tt = t_next;
#pragma unroll
    for (int j = 0; j < kTrialWarps; ++j) {
      if (nc > 0 && cand[nc - 1] < min_step) break;
      cand[j] = tt;
      nc = j + 1;
      tt *= gamma;
    }
    double mine = 0.0;
#pragma unroll
    for (int j = 0; j < kTrialWarps; ++j)
      if (j == w) mine = cand[j];
    if (w < nc) {
      const bool ok = warp_trial(Xp, dXp, mine, k, ratio, slot);
      if (lane == 0) flags[w] = ok ? 1 : 0;
    }
    __syncthreads();
    int f[kTrialWarps];
#pragma unroll
    for (int n = 0; n < kTrialWarps; ++n) f[n] = flags[n];
    __syncthreads();
#pragma unroll
    for (int j = 0; j < kTrialWarps; ++j)
      if (j < nc && (f[j] || cand[j] < min_step)) return cand[j];
    t_next = cand[nc - 1] * gamma;
  }
  return t_next;
}

}  // namespace batch
}  // namespace sdpx
