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
  double* T;  // k×k scratch per work item of the DMMA Schur path (T_j = W·A_j)
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

// C = op(A)·B for k×k column-major operands (shared or global memory) on the
// FP64 tensor cores: each warp takes 8×8 output tiles in turn and runs the
// m8n8k4 DMMA over k in steps of 4 (loads past k read 0).  ta: A transposed.
// C must not alias A or B.  Ends with a CTA barrier.
__device__ void cta_gemm_dmma(const double* A, bool ta, const double* B, double* C, int k) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  const int g = lane >> 2, t = lane & 3;
  const int nb = (k + 7) / 8;
  for (int tile = warp; tile < nb * nb; tile += nw) {
    const int i0 = (tile % nb) * 8, j0 = (tile / nb) * 8;
    const int r = i0 + g, cB = j0 + g;
    double c0 = 0.0, c1 = 0.0;
    for (int kk = 0; kk < k; kk += 4) {
      const int p = kk + t;
      const bool okp = p < k;
      const double a = (okp && r < k) ? (ta ? A[p + r * k] : A[r + p * k]) : 0.0;
      const double b = (okp && cB < k) ? B[p + cB * k] : 0.0;
      dmma_8x8x4(c0, c1, a, b);
    }
    const int cc = j0 + 2 * t;
    if (r < k) {
      if (cc < k) C[r + cc * k] = c0;
      if (cc + 1 < k) C[r + (cc + 1) * k] = c1;
    }
  }
  __syncthreads();
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

// ------------------------------------- fraction to the boundary by eigenvalue
// X + t·dX = L(I + t·G)Lᵀ with G = L⁻¹·dX·L⁻ᵀ, so X + t·dX stays positive
// definite for t < t* = −1/λ_min(G) (every t when λ_min ≥ 0).  The bound is
// 1 when 1 + λ_min(G) > 0 (the full step stays interior), else t*: the value
// the bisection of `fraction_to_boundary_bound!` approaches from below, up to
// the rounding of its Cholesky tests.  λ_min comes from a Householder
// tridiagonalisation of G and a Sturm-count multisection of the tridiagonal
// matrix (one shift per thread per round).

namespace eigdetail {
// Number of eigenvalues of the symmetric tridiagonal (a, b) below x (the
// negative pivots of the LDLᵀ recurrence of T − x·I, zero pivots nudged).
__device__ __forceinline__ int sturm_count(const double* a, const double* b, int n, double x,
                                           double tiny) {
  int neg = 0;
  double q = a[0] - x;
  if (q == 0.0) q = -tiny;
  if (q < 0.0) ++neg;
  for (int i = 1; i < n; ++i) {
    q = (a[i] - x) - b[i - 1] * b[i - 1] / q;
    if (q == 0.0) q = -tiny;
    if (q < 0.0) ++neg;
  }
  return neg;
}
}  // namespace eigdetail

// λ_min of the symmetric k×k G (shared memory, overwritten); v, w: k doubles
// each, ab: 2k doubles (shared).  Called by the whole CTA.
__device__ double cta_lambda_min(double* G, int k, double* v, double* w, double* ab,
                                 double* red) {
  // Householder tridiagonalisation: column j's subdiagonal part is reduced
  // to α·e₁ by H = I − β·v·vᵀ applied on both sides of the trailing block.
  for (int j = 0; j + 2 < k; ++j) {
    const int n = k - j - 1, o = j + 1;
    double s = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
      const double x = G[(o + i) + j * k];
      v[i] = x;
      s += x * x;
    }
    s = block_sum(s, red);
    const double norm = sqrt(s);
    const double x0 = G[o + j * k];
    const double alpha = x0 > 0.0 ? -norm : norm;
    if (norm == 0.0) continue;  // column already reduced (uniform)
    if (threadIdx.x == 0) v[0] = x0 - alpha;
    __syncthreads();
    double vv = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) vv += v[i] * v[i];
    vv = block_sum(vv, red);
    if (!(vv > 0.0)) continue;
    const double beta = 2.0 / vv;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {  // p = β·A·v
      double t = 0.0;
      for (int c = 0; c < n; ++c) t += G[(o + i) + (o + c) * k] * v[c];
      w[i] = beta * t;
    }
    __syncthreads();
    double pv = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) pv += w[i] * v[i];
    pv = block_sum(pv, red);
    const double K = 0.5 * beta * pv;
    for (int i = threadIdx.x; i < n; i += blockDim.x) w[i] -= K * v[i];  // w = p − K·v
    __syncthreads();
    for (int e = threadIdx.x; e < n * n; e += blockDim.x) {  // A −= v·wᵀ + w·vᵀ
      const int r = e % n, c = e / n;
      G[(o + r) + (o + c) * k] -= v[r] * w[c] + w[r] * v[c];
    }
    if (threadIdx.x == 0) G[o + j * k] = alpha;
    __syncthreads();
  }
  double* a = ab;
  double* b = ab + k;
  for (int i = threadIdx.x; i < k; i += blockDim.x) {
    a[i] = G[i + i * k];
    if (i + 1 < k) b[i] = G[(i + 1) + i * k];
  }
  __syncthreads();
  // Gershgorin interval, then multisection: each thread counts at one shift
  double lo = 0.0, hi = 0.0, bmax = 0.0;
  if (threadIdx.x == 0) {
    lo = a[0], hi = a[0];
    for (int i = 0; i < k; ++i) {
      const double r = (i > 0 ? fabs(b[i - 1]) : 0.0) + (i + 1 < k ? fabs(b[i]) : 0.0);
      lo = fmin(lo, a[i] - r);
      hi = fmax(hi, a[i] + r);
      if (i + 1 < k) bmax = fmax(bmax, fabs(b[i]));
    }
    red[0] = lo;
    red[1] = hi;
    red[2] = fmax(bmax, fmax(fabs(lo), fabs(hi)));
  }
  __syncthreads();
  lo = red[0];
  hi = red[1];
  const double tiny = 2.2250738585072014e-308 * fmax(1.0, red[2] * red[2]);  // pivot floor
  __syncthreads();
  __shared__ int cnt[kThreads];
  for (int round = 0; round < 12; ++round) {
    const double step = (hi - lo) / (blockDim.x + 1);
    if (!(step > 0.0) || hi - lo <= 4.0 * 2.220446049250313e-16 * fmax(fabs(lo), fabs(hi)))
      break;
    const double x = lo + (threadIdx.x + 1) * step;
    cnt[threadIdx.x] = eigdetail::sturm_count(a, b, k, x, tiny);
    __syncthreads();
    // smallest eigenvalue ∈ (last shift with count 0, first shift with count ≥ 1]
    int first = blockDim.x;
    for (int t = 0; t < (int)blockDim.x; ++t)
      if (cnt[t] > 0) {
        first = t;
        break;
      }
    const double nlo = first == 0 ? lo : lo + first * step;
    const double nhi = first == (int)blockDim.x ? hi : lo + (first + 1) * step;
    __syncthreads();
    lo = nlo;
    hi = nhi;
  }
  return 0.5 * (lo + hi);
}

// Fraction-to-boundary bound of M along dM from the factor L of M (lower,
// global): W = L⁻¹ (given, or computed when Winv is null), G = W·dM·Wᵀ.
// S0, S1, S2: three k×k shared slots; small: 4k + 32 doubles of shared scratch.
__device__ double cta_ftb_eig(const double* L, const double* Wg, const double* dM, int k,
                              double* S0, double* S1, double* S2, double* small, double* red) {
  const int kk = k * k;
  if (Wg) {
    for (int e = threadIdx.x; e < kk; e += blockDim.x) S0[e] = Wg[e];
  } else {
    for (int e = threadIdx.x; e < kk; e += blockDim.x) {
      const int r = e % k, c = e / k;
      S2[e] = r >= c ? L[e] : 0.0;
    }
    __syncthreads();
    cta_trinv(S2, S0, k);
  }
  for (int e = threadIdx.x; e < kk; e += blockDim.x) S1[e] = dM[e];
  __syncthreads();
  for (int e = threadIdx.x; e < kk; e += blockDim.x) {  // T = W·dM (W lower)
    const int r = e % k, c = e / k;
    double s = 0.0;
    for (int p = 0; p <= r; ++p) s += S0[r + p * k] * S1[p + c * k];
    S2[e] = s;
  }
  __syncthreads();
  for (int e = threadIdx.x; e < kk; e += blockDim.x) {  // G = T·Wᵀ
    const int r = e % k, c = e / k;
    double s = 0.0;
    for (int p = 0; p <= c; ++p) s += S2[r + p * k] * S0[c + p * k];
    S1[e] = s;
  }
  __syncthreads();
  for (int e = threadIdx.x; e < kk; e += blockDim.x) {  // symmetrise into S2
    const int r = e % k, c = e / k;
    S2[e] = 0.5 * (S1[e] + S1[c + r * k]);
  }
  __syncthreads();
  const double lmin = cta_lambda_min(S2, k, small, small + k, small + 2 * k, red);
  if (!(lmin == lmin)) return 0.0;  // non-finite direction: no step
  if (1.0 + lmin > 0.0) return 1.0;
  return -1.0 / lmin;
}

}  // namespace batch
}  // namespace sdpx
