// Batched small-SDP engine: many independent single-block dense SDPs solved
// in lockstep, one kernel per interior-point phase over every instance still
// running, the scalar decisions of each instance taken on the host by its own
// controller.
//
// The loop is the library's dense loop (driver_api.inc: SDPX's
// `_solve_sdp_core!` and `newton_step!`, src/solver/interior_point.jl:1742-2333,
// src/step.jl:643-1023) for the options this engine serves: the fixed start
// x = 0, X = ω_p·I, Y = ω_d·I (src/solver/interior_point.jl:1600-1612), no
// equilibration, FP64 arithmetic, the adaptive or fixed parameter strategy,
// backtracking line search (k ≥ 3), fixed or adaptive refinement, no equality
// rows.  Per pass and instance it takes the same stages with the same scalar
// rules — termination and stagnation, the Newton step, centering and restarts
// on a collapsed step, the best-iterate rule — so an instance's result is its
// single solve's up to rounding (summation orders differ).
//
// Work layout: one CTA per instance for every phase but the Schur assembly,
// whose panel P̂_j = L_X⁻¹A_jL_Y and SYRK S = P̂P̂ᵀ are split into work items
// of about `grain` FLOPs (an instance's constraints, resp. its lower SYRK
// tiles, in contiguous ranges), issued largest first.  The launch shape
// (threads, SYRK tile, grain) is chosen by sdpx_b200_batch_autotune.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <numeric>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

#include "../../include/sdpx_b200_batch.h"
#include "batch_kernels.cuh"
#include "dbuf.h"
#include "dd.cuh"
#include "gemm_f64.cuh"
#include "ipm_controller.h"

namespace sdpx {
namespace batch {
namespace {

// Scalars per launched CTA row exchanged with the host each phase (row = the
// instance's position in the launch's list).
enum In { kMu = 0, kUseAffine, kFactor, kTarget, kMode, kTX, kTY, kRatio, kGamma, kMinStep,
          kOmega, kBoundMode, kNIn };
enum Out { oPres = 0, oDres, oOk, oPmargin, oDmargin, oReg, oQual, oCompl, oAff, oAffFull, oTX,
           oTY, oRes, oRnorm, oPobj, oDobj, oFinite, oDa, oNOut };

#define INST_PROLOGUE                                    \
  const int id = act[blockIdx.x];                        \
  const Inst I = pool.inst[id];                          \
  const int k = I.k, m = I.m;                            \
  const long long kk = (long long)k * k;                 \
  [[maybe_unused]] const double* in = par + (long long)blockIdx.x * kNIn; \
  [[maybe_unused]] double* out = res + (long long)blockIdx.x * oNOut;     \
  (void)m;                                                                \
  (void)kk;

// B1: P = 𝒜x − X − C, d = c − 𝒜ᵀY, R = −XY (+μI unless affine); with kFactor
// also L_X = chol(X), L_Y = chol(Y), W = L_X⁻¹ and the Cholesky margins
// (`threaded_residuals!`, src/kernels/threaded.jl; `_cholesky_diagonal_quality`).
__global__ void __launch_bounds__(kThreads)
    k_b_residuals(Pool pool, const int* act, const double* par, double* res) {
  INST_PROLOGUE
  extern __shared__ __align__(16) double sm[];
  double* Xs = sm;
  double* Ys = Xs + pool.kq;
  __shared__ double red[32], sflag[4];
  const double* A = pool.A + I.a_off;
  double* P = pool.P + I.kk_off;
  const double* X = pool.X + I.kk_off;
  const double* Y = pool.Y + I.kk_off;
  const double* C = pool.C + I.kk_off;
  const double* x = pool.x + I.m_off;
  double pmax = 0.0;
  for (long long e = threadIdx.x; e < kk; e += blockDim.x) {
    double s = 0.0;
    for (int j = 0; j < m; ++j) s += x[j] * A[(long long)j * kk + e];
    const double v = s - X[e] - C[e];
    P[e] = v;
    pmax = fmax(pmax, abs_nan_inf(v));
    Xs[e] = X[e];
    Ys[e] = Y[e];
  }
  pmax = cta_max(pmax, red);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  double dmax = 0.0;
  for (int j = warp; j < m; j += nw) {  // d_j = c_j − ⟨A_j, Y⟩, one warp per j
    double s = 0.0;
    for (long long e = lane; e < kk; e += 32) s += A[(long long)j * kk + e] * Y[e];
    s = warp_sum(s);
    const double dv = pool.c[I.m_off + j] - s;
    if (lane == 0) pool.d[I.m_off + j] = dv;
    dmax = fmax(dmax, abs_nan_inf(dv));
  }
  dmax = cta_max(dmax, red);
  double* R = pool.R + I.kk_off;
  const double mu = in[kMu];
  const bool add_mu = in[kUseAffine] == 0.0;
  cta_gemm_dmma(Xs, false, Ys, R, k);  // R = X·Y (global), then −XY (+μI)
  for (long long e = threadIdx.x; e < kk; e += blockDim.x) {
    const int r = (int)(e % k), c = (int)(e / k);
    double s = -R[e];
    if (add_mu && r == c) s += mu;
    R[e] = s;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    out[oPres] = pmax;
    out[oDres] = dmax;
    out[oOk] = 1.0;
  }
  if (in[kFactor] == 0.0) return;
  double xmn = 0, xmx = 0, ymn = 0, ymx = 0;
  const bool okx = cta_chol(Xs, k, sflag, &xmn, &xmx);
  const bool oky = okx && cta_chol(Ys, k, sflag, &ymn, &ymx);
  if (threadIdx.x == 0) {
    auto q = [](double mn, double mx) {
      return (mx > 0 && isfinite(mx)) ? fmin(1.0, fmax(0.0, mn / mx)) : 0.0;
    };
    out[oOk] = (okx && oky) ? 1.0 : 0.0;
    out[oPmargin] = okx ? q(xmn, xmx) : 0.0;
    out[oDmargin] = oky ? q(ymn, ymx) : 0.0;
  }
  if (!(okx && oky)) return;
  double* LX = pool.LX + I.kk_off;
  double* LY = pool.LY + I.kk_off;
  for (long long e = threadIdx.x; e < kk; e += blockDim.x) {
    const int r = (int)(e % k), c = (int)(e / k);
    LX[e] = r >= c ? Xs[e] : 0.0;
    LY[e] = r >= c ? Ys[e] : 0.0;
  }
  __syncthreads();
  for (long long e = threadIdx.x; e < kk; e += blockDim.x) {
    const int r = (int)(e % k), c = (int)(e / k);
    Ys[e] = r >= c ? Xs[e] : 0.0;  // lower L_X
  }
  __syncthreads();
  cta_trinv(Ys, Xs, k);
  double* W = pool.W + I.kk_off;
  for (long long e = threadIdx.x; e < kk; e += blockDim.x) W[e] = Xs[e];
}

// B2a: the Schur panel P̂_j = W·A_j·L_Y (W = L_X⁻¹, both lower) for the
// constraints j ∈ [lo, hi) of one work item {row, lo, hi}.
__global__ void k_b_panel(Pool pool, const int* act, const int4* work) {
  const int4 wi = work[blockIdx.x];
  const Inst I = pool.inst[act[wi.x]];
  const int k = I.k;
  const long long kk = (long long)k * k;
  extern __shared__ __align__(16) double sm[];
  double* Ws = sm;
  double* Ls = Ws + pool.kq;
  double* As = Ls + pool.kq;
  double* Ts = As + pool.kq;
  for (long long e = threadIdx.x; e < kk; e += blockDim.x) {
    Ws[e] = pool.W[I.kk_off + e];
    Ls[e] = pool.LY[I.kk_off + e];
  }
  const double* A = pool.A + I.a_off;
  double* Ph = pool.Ph + I.a_off;
  for (int j = wi.y; j < wi.z; ++j) {
    for (long long e = threadIdx.x; e < kk; e += blockDim.x) As[e] = A[(long long)j * kk + e];
    __syncthreads();
    for (long long e = threadIdx.x; e < kk; e += blockDim.x) {  // T = W·A_j
      const int r = (int)(e % k), c = (int)(e / k);
      double s = 0.0;
      for (int p = 0; p <= r; ++p) s += Ws[r + p * k] * As[p + c * k];
      Ts[e] = s;
    }
    __syncthreads();
    for (long long e = threadIdx.x; e < kk; e += blockDim.x) {  // P̂_j = T·L_Y
      const int r = (int)(e % k), c = (int)(e / k);
      double s = 0.0;
      for (int q = c; q < k; ++q) s += Ts[r + q * k] * Ls[q + c * k];
      Ph[(long long)j * kk + e] = s;
    }
    __syncthreads();
  }
}

// Row of the lower-triangle tile with linear index q (q = ti(ti+1)/2 + tj).
__device__ __forceinline__ int tri_row(int q) {
  int ti = (int)((sqrt(8.0 * q + 1.0) - 1.0) * 0.5);
  while ((ti + 1) * (ti + 2) / 2 <= q) ++ti;
  while (ti * (ti + 1) / 2 > q) --ti;
  return ti;
}

// B2b: S = P̂P̂ᵀ (m×m, both triangles written) over the lower T×T tiles
// [lo, hi) of one work item; K = k² staged T at a time through shared memory,
// RA×RB outputs per thread.
template <int NT, int T>
__global__ void __launch_bounds__(NT) k_b_syrk(Pool pool, const int* act, const int4* work) {
  constexpr int OUT = T * T / NT;
  constexpr int RB = OUT >= 4 ? 2 : 1;
  constexpr int RA = OUT / RB;
  constexpr int TX = T / RB;  // threads along the tile's columns
  static_assert(RA * RB * NT == T * T, "tile / thread split");
  const int4 wi = work[blockIdx.x];
  const Inst I = pool.inst[act[wi.x]];
  const int m = I.m;
  const long long kk = (long long)I.k * I.k;
  __shared__ double At[T][T + 1], Bt[T][T + 1];
  const double* Ph = pool.Ph + I.a_off;
  double* S = pool.S + I.mm_off;
  const int ty = threadIdx.x / TX, tx = threadIdx.x % TX;
  for (int q = wi.y; q < wi.z; ++q) {
    const int ti = tri_row(q), tj = q - ti * (ti + 1) / 2;
    double acc[RA][RB];
#pragma unroll
    for (int a = 0; a < RA; ++a)
#pragma unroll
      for (int b = 0; b < RB; ++b) acc[a][b] = 0.0;
    for (long long k0 = 0; k0 < kk; k0 += T) {
      for (int e = threadIdx.x; e < T * T; e += NT) {
        const int rr = e / T, cc = e % T;
        const int gi = ti * T + rr, gj = tj * T + rr;
        const long long kc = k0 + cc;
        At[rr][cc] = (gi < m && kc < kk) ? Ph[(long long)gi * kk + kc] : 0.0;
        Bt[rr][cc] = (gj < m && kc < kk) ? Ph[(long long)gj * kk + kc] : 0.0;
      }
      __syncthreads();
#pragma unroll 8
      for (int p = 0; p < T; ++p) {
        double av[RA], bv[RB];
#pragma unroll
        for (int a = 0; a < RA; ++a) av[a] = At[ty * RA + a][p];
#pragma unroll
        for (int b = 0; b < RB; ++b) bv[b] = Bt[tx * RB + b][p];
#pragma unroll
        for (int a = 0; a < RA; ++a)
#pragma unroll
          for (int b = 0; b < RB; ++b) acc[a][b] += av[a] * bv[b];
      }
      __syncthreads();
    }
#pragma unroll
    for (int a = 0; a < RA; ++a)
#pragma unroll
      for (int b = 0; b < RB; ++b) {
        const int gi = ti * T + ty * RA + a, gj = tj * T + tx * RB + b;
        if (gi < m && gj < m && gi >= gj) {
          S[gi + (long long)gj * m] = acc[a][b];
          S[gj + (long long)gi * m] = acc[a][b];
        }
      }
  }
}

// ---- B2 on the FP64 tensor cores (DMMA m8n8k4 tiles of gemm_f64.cuh) -----
// Per instance P̂_j = W·A_j·L_Y (W = L_X⁻¹) for every constraint, then
// S = P̂·P̂ᵀ over the lower tiles (both triangles written); 4 warps per CTA,
// work items {row, first, end} as for the scalar kernels.  Each instance takes
// the tile that pads least: 32×32 for T·P̂ when k ≤ 32 and for the SYRK when
// m ≤ 64, else 64×64.
using DmmaCfgKN = F64Cfg<64, 64, 2, 2, false, true>;  // A MN-contiguous, B K-contiguous
using DmmaCfgKK = F64Cfg<64, 64, 2, 2, true, true>;   // both K-contiguous
using DmmaCfgKN32 = F64Cfg<32, 32, 2, 2, false, true>;  // 32×32 tiles for small instances
using DmmaCfgKK32 = F64Cfg<32, 32, 2, 2, true, true>;

// T and P̂ fused per constraint: work item {row, first j, end j}; T_j = W·A_j
// goes to this CTA's k×k scratch (pool.T + blockIdx.x·kq, reused for every j,
// so it stays in L2), then P̂_j = T_j·L_Y.
template <class Cfg>
__global__ void __launch_bounds__(Cfg::NT)
    k_b_dmma_tp(Pool pool, const int* act, const int4* work) {
  extern __shared__ __align__(16) double smem[];
  const int4 wi = work[blockIdx.x];
  const Inst I = pool.inst[act[wi.x]];
  const int k = I.k;
  const long long kk = (long long)k * k;
  double* T = pool.T + (long long)blockIdx.x * pool.kq;
  const Opnd Aw{pool.W + I.kk_off, k, 1, 0, 1 << 30, k, k};     // (r, p) at r + p·k
  const Opnd At{T, k, 1, 0, 1 << 30, k, k};                      // (r, q) at r + q·k
  const Opnd Bl{pool.LY + I.kk_off, 1, k, 0, 1 << 30, k, k};    // (q, c) at q + c·k
  for (int j = wi.y; j < wi.z; ++j) {
    const Opnd Bj{pool.A + I.a_off + (long long)j * kk, 1, k, 0, 1 << 30, k, k};  // (p, c)
    double acc[Cfg::FM][Cfg::FN][2];
    zero_acc<Cfg>(acc);
    f64_tile_mainloop<Cfg>(acc, Aw, Bj, 0, 0, 0, k, smem);
    for_each_acc<Cfg>(acc, [&](int r, int c, double v) {
      if (r < k && c < k) T[r + (long long)c * k] = v;
    });
    __syncthreads();
    zero_acc<Cfg>(acc);
    f64_tile_mainloop<Cfg>(acc, At, Bl, 0, 0, 0, k, smem);
    double* Pj = pool.Ph + I.a_off + (long long)j * kk;
    for_each_acc<Cfg>(acc, [&](int r, int c, double v) {
      if (r < k && c < k) Pj[r + (long long)c * k] = v;
    });
    __syncthreads();
  }
}

template <class Cfg>
__global__ void __launch_bounds__(Cfg::NT)
    k_b_dmma_syrk(Pool pool, const int* act, const int4* work) {
  extern __shared__ __align__(16) double smem[];
  const int4 wi = work[blockIdx.x];
  const Inst I = pool.inst[act[wi.x]];
  const int m = I.m;
  const int kk = I.k * I.k;
  // P̂ rows j: (j, e) at j·k² + e, for both operands (S = P̂·P̂ᵀ)
  const Opnd Pp{pool.Ph + I.a_off, 1, kk, 0, 1 << 30, m, kk};
  double* S = pool.S + I.mm_off;
  for (int q = wi.y; q < wi.z; ++q) {
    const int ti = tri_row(q), tj = q - ti * (ti + 1) / 2;
    double acc[Cfg::FM][Cfg::FN][2];
    zero_acc<Cfg>(acc);
    f64_tile_mainloop<Cfg>(acc, Pp, Pp, ti * Cfg::BM, tj * Cfg::BM, 0, kk, smem);
    for_each_acc<Cfg>(acc, [&](int r, int c, double v) {
      const int gi = ti * Cfg::BM + r, gj = tj * Cfg::BM + c;
      if (gi < m && gj < m && gi >= gj) {
        S[gi + (long long)gj * m] = v;
        S[gj + (long long)gi * m] = v;
      }
    });
  }
}

// Blocked lower Cholesky of the m×m column-major M in place (global memory,
// one CTA): 16-column panels factored column by column (pivot, scale, rank-1
// update inside the panel), then the trailing block updated by the panel as a
// rank-16 SYRK on DMMA m8n8k4 fragments (8×8 lower tiles, one per warp in
// turn).  False at the first pivot that is not > 0.
__device__ bool cta_chol_blocked(double* M, int m, double* sflag) {
  constexpr int NB = 16;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  const int g = lane >> 2, t = lane & 3;
  for (int jb = 0; jb < m; jb += NB) {
    const int je = min(m, jb + NB);
    for (int j = jb; j < je; ++j) {
      if (threadIdx.x == 0) {
        const double d = M[j + (long long)j * m];
        sflag[0] = d;
        sflag[1] = d > 0.0 ? sqrt(d) : 0.0;
      }
      __syncthreads();
      if (!(sflag[0] > 0.0)) return false;
      const double ljj = sflag[1];
      const double inv = 1.0 / ljj;
      for (int i = j + 1 + threadIdx.x; i < m; i += blockDim.x) M[i + (long long)j * m] *= inv;
      if (threadIdx.x == 0) M[j + (long long)j * m] = ljj;
      __syncthreads();
      const int nc = je - j - 1, rows = m - j - 1;  // panel columns right of j, all rows below j
      for (long long e = threadIdx.x; e < (long long)nc * rows; e += blockDim.x) {
        const int ii = j + 1 + (int)(e % rows), ll = j + 1 + (int)(e / rows);
        if (ii >= ll)
          M[ii + (long long)ll * m] -= M[ii + (long long)j * m] * M[ll + (long long)j * m];
      }
      __syncthreads();
    }
    // trailing block rows, cols ≥ je:  M −= L_panel · L_panelᵀ (lower 8×8 tiles)
    const int n = m - je;
    if (n <= 0) break;
    const int nb8 = (n + 7) / 8;
    const int ntile = nb8 * (nb8 + 1) / 2;
    for (int tile = warp; tile < ntile; tile += nw) {
      int ti = (int)((sqrt(8.0 * tile + 1.0) - 1.0) * 0.5);
      while ((ti + 1) * (ti + 2) / 2 <= tile) ++ti;
      while (ti * (ti + 1) / 2 > tile) --ti;
      const int tj = tile - ti * (ti + 1) / 2;
      const int r = je + ti * 8 + g, cB = je + tj * 8 + g;
      double c0 = 0.0, c1 = 0.0;
      for (int kk = jb; kk < je; kk += 4) {
        const int p = kk + t;
        const bool okp = p < je;
        const double a = (okp && r < m) ? M[r + (long long)p * m] : 0.0;
        const double b = (okp && cB < m) ? M[cB + (long long)p * m] : 0.0;
        dmma_8x8x4(c0, c1, a, b);
      }
      const int cc = je + tj * 8 + 2 * t;
      if (r < m) {
        if (cc < m && r >= cc) M[r + (long long)cc * m] -= c0;
        if (cc + 1 < m && r >= cc + 1) M[r + (long long)(cc + 1) * m] -= c1;
      }
    }
    __syncthreads();
  }
  return true;
}

// B3: Cholesky of S with ≤ 6 regularisation retries, S_ii += δ·max(|S_ii|, 1)
// with δ = √eps then ×10 (src/kkt.jl:1419-1445); quality = min/max |L_jj|.
__global__ void __launch_bounds__(kThreads)
    k_b_factor(Pool pool, const int* act, const double* par, double* res) {
  INST_PROLOGUE
  __shared__ double sflag[4];
  const double* S = pool.S + I.mm_off;
  double* L = pool.LS + I.mm_off;
  const long long mm = (long long)m * m;
  int attempts = 0;
  double reg = 0.0;
  bool ok = false;
  while (true) {
    for (long long e = threadIdx.x; e < mm; e += blockDim.x) {
      const int r = (int)(e % m), c = (int)(e / m);
      double v = r >= c ? S[e] : 0.0;
      if (r == c && attempts > 0) v += reg * fmax(fabs(S[e]), 1.0);
      L[e] = v;
    }
    __syncthreads();
    ok = cta_chol_blocked(L, m, sflag);
    __syncthreads();
    if (ok || attempts >= 6) break;
    ++attempts;
    reg = attempts == 1 ? 1.4901161193847656e-08 : reg * 10.0;
  }
  if (threadIdx.x == 0) {
    out[oOk] = ok ? 1.0 : 0.0;
    out[oReg] = attempts;
    double q = 0.0;
    if (ok) {
      double mn = fabs(L[0]), mx = mn;
      for (int j = 1; j < m; ++j) {
        mn = fmin(mn, fabs(L[j + (long long)j * m]));
        mx = fmax(mx, fabs(L[j + (long long)j * m]));
      }
      q = (mx > 0 && isfinite(mx)) ? fmin(1.0, fmax(0.0, mn / mx)) : 0.0;
    }
    out[oQual] = q;
  }
}

// v ← S⁻¹v with the lower factor L (m×m, global), v in shared memory.
__device__ void cta_cholsolve(const double* L, int m, double* v, double* red) {
  for (int j = 0; j < m; ++j) {  // forward: L y = v, column-oriented
    __syncthreads();
    const double yj = v[j] / L[j + (long long)j * m];
    __syncthreads();
    if (threadIdx.x == 0) v[j] = yj;
    for (int i = j + 1 + threadIdx.x; i < m; i += blockDim.x) v[i] -= L[i + (long long)j * m] * yj;
  }
  for (int j = m - 1; j >= 0; --j) {  // backward: Lᵀ z = y, one dot per row
    __syncthreads();
    double s = 0.0;
    for (int i = j + 1 + threadIdx.x; i < m; i += blockDim.x) s += L[i + (long long)j * m] * v[i];
    s = block_sum(s, red);
    if (threadIdx.x == 0) v[j] = (v[j] - s) / L[j + (long long)j * m];
  }
  __syncthreads();
}

// B4: right-hand side r = −(d + ⟨A_j, X⁻¹(PY − R)⟩) (`rhs_from_R`); kMode 1
// first forms the corrector R = kTarget·I − XY − dX·dY.
__global__ void __launch_bounds__(kThreads)
    k_b_rhs(Pool pool, const int* act, const double* par, double* res) {
  INST_PROLOGUE
  extern __shared__ __align__(16) double sm[];
  double* M1 = sm;
  double* M2 = M1 + pool.kq;
  double* M3 = M2 + pool.kq;
  double* R = pool.R + I.kk_off;
  const double* X = pool.X + I.kk_off;
  const double* Y = pool.Y + I.kk_off;
  for (long long e = threadIdx.x; e < kk; e += blockDim.x) {
    M1[e] = X[e];
    M2[e] = Y[e];
  }
  __syncthreads();
  if (in[kMode] == 1.0) {  // R = target·I − X·Y − dX·dY
    cta_gemm_dmma(M1, false, M2, M3, k);                                    // X·Y
    cta_gemm_dmma(pool.dX + I.kk_off, false, pool.dY + I.kk_off, M1, k);  // dX·dY
    for (long long e = threadIdx.x; e < kk; e += blockDim.x) {
      const int r = (int)(e % k), c = (int)(e / k);
      double v = -M3[e] - M1[e];
      if (r == c) v += in[kTarget];
      R[e] = v;
    }
    __syncthreads();
  }
  // Z = P·Y − R, then X⁻¹Z = Wᵀ·W·Z
  const double* P = pool.P + I.kk_off;
  cta_gemm_dmma(P, false, M2, M3, k);  // P·Y
  for (long long e = threadIdx.x; e < kk; e += blockDim.x) M1[e] = M3[e] - R[e];
  for (long long e = threadIdx.x; e < kk; e += blockDim.x) M3[e] = pool.W[I.kk_off + e];
  __syncthreads();
  cta_gemm_dmma(M3, false, M1, M2, k);  // W·(PY − R)
  cta_gemm_dmma(M3, true, M2, M1, k);   // X⁻¹(PY − R) = Wᵀ·W·(PY − R)
  const double* A = pool.A + I.a_off;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  for (int j = warp; j < m; j += nw) {
    double s = 0.0;
    for (long long e = lane; e < kk; e += 32) s += A[(long long)j * kk + e] * M1[e];
    s = warp_sum(s);
    if (lane == 0) pool.r[I.m_off + j] = -(pool.d[I.m_off + j] + s);
  }
}

// B5: kMode 0: dx = S⁻¹r; kMode 1 (a refinement correction): dxb = dx,
// dx += S⁻¹ρ (`_apply_kkt_correction!`, src/kkt.jl:3762-3780).
__global__ void __launch_bounds__(kThreads)
    k_b_solve(Pool pool, const int* act, const double* par, double* res) {
  INST_PROLOGUE
  __shared__ double v[kMaxM];
  __shared__ double red[32];
  const bool corr = in[kMode] == 1.0;
  const double* src = corr ? pool.rho + I.m_off : pool.r + I.m_off;
  for (int i = threadIdx.x; i < m; i += blockDim.x) v[i] = src[i];
  cta_cholsolve(pool.LS + I.mm_off, m, v, red);
  double* dx = pool.dx + I.m_off;
  for (int i = threadIdx.x; i < m; i += blockDim.x) {
    if (corr) {
      pool.dxb[I.m_off + i] = dx[i];
      dx[i] += v[i];
    } else {
      dx[i] = v[i];
    }
  }
}

// B6: dX = mat(Σ dx_j A_j) + P, dY = sym(X⁻¹(R − dX·Y)) (`direction_blocks`).
__global__ void __launch_bounds__(kThreads)
    k_b_dirblocks(Pool pool, const int* act, const double* par, double* res) {
  INST_PROLOGUE
  extern __shared__ __align__(16) double sm[];
  double* M1 = sm;
  double* M2 = M1 + pool.kq;
  double* M3 = M2 + pool.kq;
  const double* A = pool.A + I.a_off;
  const double* dx = pool.dx + I.m_off;
  double* dX = pool.dX + I.kk_off;
  const double* P = pool.P + I.kk_off;
  for (long long e = threadIdx.x; e < kk; e += blockDim.x) {
    double s = 0.0;
    for (int j = 0; j < m; ++j) s += dx[j] * A[(long long)j * kk + e];
    const double v = s + P[e];
    dX[e] = v;
    M1[e] = v;
    M2[e] = pool.Y[I.kk_off + e];
    M3[e] = pool.W[I.kk_off + e];
  }
  __syncthreads();
  const double* R = pool.R + I.kk_off;
  double* Z = pool.Z + I.kk_off;
  cta_gemm_dmma(M1, false, M2, Z, k);  // dX·Y (global scratch)
  for (long long e = threadIdx.x; e < kk; e += blockDim.x) M1[e] = R[e] - Z[e];
  __syncthreads();
  cta_gemm_dmma(M3, false, M1, M2, k);
  cta_gemm_dmma(M3, true, M2, M1, k);
  double* dY = pool.dY + I.kk_off;
  for (long long e = threadIdx.x; e < kk; e += blockDim.x) {
    const int r = (int)(e % k), c = (int)(e / k);
    dY[e] = 0.5 * (M1[e] + M1[c + r * k]);
  }
}

// B7: affine diagnostics: with kMode 1 the fraction-to-boundary bounds of X
// and Y along dX, dY (`fraction_to_boundary_bound!`, eight trials at a time),
// ⟨X, Y⟩, ⟨X + tX·dX, Y + tY·dY⟩ and ⟨X + dX, Y + dY⟩.
__global__ void __launch_bounds__(kThreads)
    k_b_affine(Pool pool, const int* act, const double* par, double* res) {
  INST_PROLOGUE
  extern __shared__ __align__(16) double sm[];
  __shared__ double red[32];
  __shared__ int flags[kTrialWarps];
  __shared__ double small[4 * kMaxK];
  double tX = 1.0, tY = 1.0;
  if (in[kMode] == 1.0) {
    double bX, bY;
    if (in[kBoundMode] == 1.0) {  // t* = −1/λ_min(L⁻¹·dM·L⁻ᵀ) from the block factors of B1
      double* S0 = sm;
      double* S1 = S0 + pool.kq;
      double* S2 = S1 + pool.kq;
      bX = cta_ftb_eig(nullptr, pool.W + I.kk_off, pool.dX + I.kk_off, k, S0, S1, S2, small, red);
      __syncthreads();
      bY = cta_ftb_eig(pool.LY + I.kk_off, nullptr, pool.dY + I.kk_off, k, S0, S1, S2, small, red);
    } else {
      bX = cta_ftb_tree(pool.X + I.kk_off, pool.dX + I.kk_off, k, sm, pool.kp, flags);
      bY = cta_ftb_tree(pool.Y + I.kk_off, pool.dY + I.kk_off, k, sm, pool.kp, flags);
    }
    tX = bX < 1.0 ? bX : 1.0;
    tY = bY < 1.0 ? bY : 1.0;
  }
  double cs = 0.0, as = 0.0, af = 0.0;
  for (long long e = threadIdx.x; e < kk; e += blockDim.x) {
    const double X = pool.X[I.kk_off + e], Y = pool.Y[I.kk_off + e];
    const double dX = pool.dX[I.kk_off + e], dY = pool.dY[I.kk_off + e];
    cs += X * Y;
    as += (X + tX * dX) * (Y + tY * dY);
    af += (X + dX) * (Y + dY);
  }
  cs = cta_sum(cs, red);
  as = cta_sum(as, red);
  af = cta_sum(af, red);
  if (threadIdx.x == 0) {
    out[oCompl] = cs;
    out[oAff] = as;
    out[oAffFull] = af;
    out[oTX] = tX;
    out[oTY] = tY;
  }
}

// B8: ρ = r − S·dx (S stored full), ‖ρ‖∞ and ‖r‖∞; one warp per row.
__global__ void __launch_bounds__(kThreads)
    k_b_resid(Pool pool, const int* act, const double* par, double* res) {
  INST_PROLOGUE
  __shared__ double red[32];
  const double* S = pool.S + I.mm_off;
  const double* dx = pool.dx + I.m_off;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  double rm = 0.0, rn = 0.0;
  for (int i = warp; i < m; i += nw) {
    double s = 0.0;
    for (int j = lane; j < m; j += 32) s += S[j + (long long)i * m] * dx[j];
    s = warp_sum(s);
    const double rv = pool.r[I.m_off + i];
    const double v = rv - s;
    if (lane == 0) pool.rho[I.m_off + i] = v;
    rm = fmax(rm, abs_nan_inf(v));
    rn = fmax(rn, abs_nan_inf(rv));
  }
  rm = cta_max(rm, red);
  rn = cta_max(rn, red);
  if (threadIdx.x == 0) {
    out[oRes] = rm;
    out[oRnorm] = rn;
  }
}

// B9: dx ← dxb (a refinement correction that did not reduce the residual).
__global__ void k_b_rollback(Pool pool, const int* act, const double* par, double* res) {
  INST_PROLOGUE
  for (int i = threadIdx.x; i < m; i += blockDim.x) pool.dx[I.m_off + i] = pool.dxb[I.m_off + i];
}

// B10: backtracking line search per side: the first t of 1, γ, γ², … for
// which M + t·dM has a Cholesky factor with min|L_jj| > kRatio·max|L_jj|, or
// the first t below kMinStep (src/kernels/threaded.jl:1751-1818); eight
// candidates at a time.
__global__ void __launch_bounds__(kThreads)
    k_b_linesearch(Pool pool, const int* act, const double* par, double* res) {
  INST_PROLOGUE
  extern __shared__ __align__(16) double sm[];
  __shared__ int flags[kTrialWarps];
  const double gamma = in[kGamma], min_step = in[kMinStep], ratio = in[kRatio];
  const double tX = cta_backtrack(pool.X + I.kk_off, pool.dX + I.kk_off, k, gamma, min_step,
                                  ratio, sm, pool.kp, flags);
  const double tY = cta_backtrack(pool.Y + I.kk_off, pool.dY + I.kk_off, k, gamma, min_step,
                                  ratio, sm, pool.kp, flags);
  if (threadIdx.x == 0) {
    out[oTX] = tX;
    out[oTY] = tY;
  }
}

// B11: X += tX·dX, Y += tY·dY, x += tX·dx; ⟨X, Y⟩, finiteness of the
// iterate, the accepted dual residual d ← (1 − tY)d − tY·ρ and its norm
// (src/solver/interior_point.jl:2228-2290), objectives cᵀx and ⟨C, Y⟩.
__global__ void __launch_bounds__(kThreads)
    k_b_update(Pool pool, const int* act, const double* par, double* res) {
  INST_PROLOGUE
  __shared__ double red[32];
  const double tX = in[kTX], tY = in[kTY];
  double cs = 0.0, fin = 0.0, dobj = 0.0;
  for (long long e = threadIdx.x; e < kk; e += blockDim.x) {
    const double X = pool.X[I.kk_off + e] + tX * pool.dX[I.kk_off + e];
    const double Y = pool.Y[I.kk_off + e] + tY * pool.dY[I.kk_off + e];
    pool.X[I.kk_off + e] = X;
    pool.Y[I.kk_off + e] = Y;
    cs += X * Y;
    fin = fmax(fin, fmax(abs_nan_inf(X), abs_nan_inf(Y)));
    dobj += pool.C[I.kk_off + e] * Y;
  }
  double dmax = 0.0, pobj = 0.0;
  for (int i = threadIdx.x; i < m; i += blockDim.x) {
    const double xv = pool.x[I.m_off + i] + tX * pool.dx[I.m_off + i];
    pool.x[I.m_off + i] = xv;
    fin = fmax(fin, abs_nan_inf(xv));
    pobj += pool.c[I.m_off + i] * xv;
    const double dv = (1.0 - tY) * pool.d[I.m_off + i] - tY * pool.rho[I.m_off + i];
    pool.d[I.m_off + i] = dv;
    dmax = fmax(dmax, abs_nan_inf(dv));
  }
  cs = cta_sum(cs, red);
  fin = cta_max(fin, red);
  dmax = cta_max(dmax, red);
  pobj = cta_sum(pobj, red);
  dobj = cta_sum(dobj, red);
  if (threadIdx.x == 0) {
    out[oCompl] = cs;
    out[oFinite] = isfinite(fin) ? 1.0 : 0.0;
    out[oDa] = dmax;
    out[oPobj] = pobj;
    out[oDobj] = dobj;
  }
}

// B12: ⟨X, Y⟩ and the objectives cᵀx, ⟨C, Y⟩ of the current iterate.
__global__ void __launch_bounds__(kThreads)
    k_b_state(Pool pool, const int* act, const double* par, double* res) {
  INST_PROLOGUE
  __shared__ double red[32];
  double cs = 0.0, dobj = 0.0, pobj = 0.0;
  for (long long e = threadIdx.x; e < kk; e += blockDim.x) {
    cs += pool.X[I.kk_off + e] * pool.Y[I.kk_off + e];
    dobj += pool.C[I.kk_off + e] * pool.Y[I.kk_off + e];
  }
  for (int i = threadIdx.x; i < m; i += blockDim.x) pobj += pool.c[I.m_off + i] * pool.x[I.m_off + i];
  cs = cta_sum(cs, red);
  dobj = cta_sum(dobj, red);
  pobj = cta_sum(pobj, red);
  if (threadIdx.x == 0) {
    out[oCompl] = cs;
    out[oPobj] = pobj;
    out[oDobj] = dobj;
  }
}

// B13: kMode 0 fixed start (x = 0, X = kTX·I, Y = kTY·I), 1 save the best
// iterate, 2 restore it, 3 X *= kOmega, 4 Y *= kOmega, 5 rebuild the slack
// X = mat(𝒜x) − C.
__global__ void k_b_elementwise(Pool pool, const int* act, const double* par, double* res) {
  INST_PROLOGUE
  const int mode = (int)in[kMode];
  double* X = pool.X + I.kk_off;
  double* Y = pool.Y + I.kk_off;
  if (mode == 5) {
    const double* A = pool.A + I.a_off;
    for (long long e = threadIdx.x; e < kk; e += blockDim.x) {
      double s = 0.0;
      for (int j = 0; j < m; ++j) s += pool.x[I.m_off + j] * A[(long long)j * kk + e];
      X[e] = s - pool.C[I.kk_off + e];
    }
    return;
  }
  for (long long e = threadIdx.x; e < kk; e += blockDim.x) {
    const int r = (int)(e % k), c = (int)(e / k);
    switch (mode) {
      case 0:
        X[e] = r == c ? in[kTX] : 0.0;
        Y[e] = r == c ? in[kTY] : 0.0;
        break;
      case 1:
        pool.Xb[I.kk_off + e] = X[e];
        pool.Yb[I.kk_off + e] = Y[e];
        break;
      case 2:
        X[e] = pool.Xb[I.kk_off + e];
        Y[e] = pool.Yb[I.kk_off + e];
        break;
      case 3: X[e] *= in[kOmega]; break;
      case 4: Y[e] *= in[kOmega]; break;
      default: break;
    }
  }
  for (int i = threadIdx.x; i < m; i += blockDim.x) {
    if (mode == 0) pool.x[I.m_off + i] = 0.0;
    if (mode == 1) pool.xb[I.m_off + i] = pool.x[I.m_off + i];
    if (mode == 2) pool.x[I.m_off + i] = pool.xb[I.m_off + i];
  }
}

// B14: ‖𝒜x − X − C‖∞ and ‖c − 𝒜ᵀY‖∞ of the current iterate.
__global__ void __launch_bounds__(kThreads)
    k_b_solres(Pool pool, const int* act, const double* par, double* res) {
  INST_PROLOGUE
  __shared__ double red[32];
  const double* A = pool.A + I.a_off;
  double pm = 0.0;
  for (long long e = threadIdx.x; e < kk; e += blockDim.x) {
    double s = 0.0;
    for (int j = 0; j < m; ++j) s += pool.x[I.m_off + j] * A[(long long)j * kk + e];
    pm = fmax(pm, abs_nan_inf(s - pool.X[I.kk_off + e] - pool.C[I.kk_off + e]));
  }
  pm = cta_max(pm, red);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  double dm = 0.0;
  for (int j = warp; j < m; j += nw) {
    double s = 0.0;
    for (long long e = lane; e < kk; e += 32) s += A[(long long)j * kk + e] * pool.Y[I.kk_off + e];
    s = warp_sum(s);
    dm = fmax(dm, abs_nan_inf(pool.c[I.m_off + j] - s));
  }
  dm = cta_max(dm, red);
  if (threadIdx.x == 0) {
    out[oPres] = pm;
    out[oDres] = dm;
  }
}

// ---------------------------------------------------------------------------
// Batched result certificate (SDPX's `result_certificate`, src/validation.jl:
// 948-1115, optimality kind, n = 0) of every instance's device-resident
// solution (x, X, Y): one CTA per instance, one row of kCertOut doubles each.
enum CertOut { cPobj = 0, cDobj, cPaff, cDaff, cCompl, cPbMixed, cPbStrict, cDbMixed, cDbStrict,
               cBadX, cBadY, cXsym, cXallowed, cXok, cXrequired, cXresolved, cYsym, cYallowed,
               cYok, cYrequired, cYresolved, kCertOut };

// |r| / scale with 0/0 = 0 and r/0 = inf (`_componentwise_ratio`,
// src/validation.jl:506-513); NaN reads as inf.
__device__ __forceinline__ double cert_ratio(double r, double scale) {
  const double a = abs_nan_inf(r);
  if (scale == 0.0) return a == 0.0 ? 0.0 : 1.0 / 0.0;
  const double q = a / scale;
  return q == q ? q : 1.0 / 0.0;
}

// `_block_psd_certificate` (src/validation.jl:765-904) for one k×k block,
// k ≥ 3: symmetry defect, Cholesky of the symmetrised copy, then of the copy
// shifted by the allowed amount; for k ≤ 4 the shift is resolved by doubling
// and 48 bisection steps.  Writes sym, allowed, ok, required, resolved to
// o[0..4] (thread 0); returns the number of non-finite entries.
__device__ double cta_psd_certificate(const double* M, int k, double tol, double* S, double* red,
                                      double* sflag, double* o) {
  const int kk = k * k;
  double bad = 0.0, mx = 0.0, sym = 0.0;
  for (int e = threadIdx.x; e < kk; e += blockDim.x) {
    const int r = e % k, c = e / k;
    const double v = M[e];
    if (!isfinite(v)) bad += 1.0;
    mx = fmax(mx, fabs(v));
    if (r < c) sym = fmax(sym, fabs(v - M[c + r * k]));
  }
  bad = cta_sum(bad, red);
  mx = cta_max(mx, red);
  sym = cta_max(sym, red);
  const double scale = fmax(mx, 1.0);
  const double allowed = fmax(tol, 128.0 * 2.220446049250313e-16) * scale;
  double ok = 0.0, required = allowed, resolved = 0.0;
  auto shifted = [&](double shift) {
    __syncthreads();
    for (int e = threadIdx.x; e < kk; e += blockDim.x) {
      const int r = e % k, c = e / k;
      double v = (M[e] + M[c + r * k]) / 2.0;
      if (r == c) v += shift;
      S[e] = v;
    }
    __syncthreads();
    return cta_chol(S, k, sflag, nullptr, nullptr);
  };
  if (bad == 0.0) {
    if (shifted(0.0)) {
      ok = sym <= allowed ? 1.0 : 0.0;
      required = 0.0;
      resolved = 1.0;
    } else {
      const bool allowed_ok = shifted(allowed);
      ok = (allowed_ok && sym <= allowed) ? 1.0 : 0.0;
      if (k <= 4) {
        double lower = 0.0, upper = allowed;
        bool res = allowed_ok;
        if (!res) {
          lower = upper;
          for (int it = 0; it < 64; ++it) {
            const double cand = upper + upper;
            if (!isfinite(cand)) break;
            upper = cand;
            if (shifted(upper)) {
              res = true;
              break;
            }
            lower = upper;
          }
        }
        if (res)
          for (int it = 0; it < 48; ++it) {
            const double mid = (lower + upper) / 2.0;
            if (shifted(mid)) upper = mid;
            else lower = mid;
          }
        required = upper;
        resolved = res ? 1.0 : 0.0;
      }
    }
  }
  if (threadIdx.x == 0) {
    o[0] = sym;
    o[1] = allowed;
    o[2] = ok;
    o[3] = required;
    o[4] = resolved;
  }
  __syncthreads();
  return bad;
}

__global__ void __launch_bounds__(kThreads)
    k_b_certificate(Pool pool, double tol_p, double tol_d, double* cert) {
  const Inst I = pool.inst[blockIdx.x];
  const int k = I.k, m = I.m;
  const long long kk = (long long)k * k;
  extern __shared__ __align__(16) double sm[];
  __shared__ double red[32], sflag[4];
  double* out = cert + (long long)blockIdx.x * kCertOut;
  const double* A = pool.A + I.a_off;
  const double* X = pool.X + I.kk_off;
  const double* Y = pool.Y + I.kk_off;
  const double* C = pool.C + I.kk_off;
  const double* x = pool.x + I.m_off;
  const double* c = pool.c + I.m_off;
  // primal rows: R = (𝒜x − X) − C with its componentwise scales
  double paff = 0.0, pbm = 0.0, pbs = 0.0, dobj = 0.0, compl_ = 0.0, badx = 0.0;
  for (long long r = threadIdx.x; r < kk; r += blockDim.x) {
    double sv = 0.0, sn = 0.0, sr = 0.0;
    for (int i = 0; i < m; ++i) {
      const double a = A[(long long)i * kk + r];
      sv += a * x[i];
      sn += fabs(a);
      sr += fabs(a) * fabs(x[i]);
    }
    const double R = (sv - X[r]) - C[r];
    const double nominal = fabs(C[r]) + sn;
    const double realized = (fabs(X[r]) + fabs(C[r])) + sr;
    paff = fmax(paff, abs_nan_inf(R));
    pbm = fmax(pbm, cert_ratio(R, nominal + realized));
    pbs = fmax(pbs, cert_ratio(R, realized));
    dobj += C[r] * Y[r];
    compl_ += X[r] * Y[r];
  }
  // dual columns: v_i = c_i − ⟨A_i, Y⟩, one warp per i
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  double daff = 0.0, dbm = 0.0, dbs = 0.0, pobj = 0.0;
  for (int i = warp; i < m; i += nw) {
    double sv = 0.0, sn = 0.0, sr = 0.0;
    for (long long r = lane; r < kk; r += 32) {
      const double a = A[(long long)i * kk + r];
      sv += a * Y[r];
      sn += fabs(a);
      sr += fabs(a) * fabs(Y[r]);
    }
    sv = warp_sum(sv);
    sn = warp_sum(sn);
    sr = warp_sum(sr);
    const double v = c[i] - sv;
    daff = fmax(daff, abs_nan_inf(v));
    dbm = fmax(dbm, cert_ratio(v, fabs(c[i]) + sn + fabs(c[i]) + sr));
    dbs = fmax(dbs, cert_ratio(v, fabs(c[i]) + sr));
  }
  for (int i = threadIdx.x; i < m; i += blockDim.x) {
    pobj += c[i] * x[i];
    if (!isfinite(x[i])) badx += 1.0;
  }
  paff = cta_max(paff, red);
  pbm = cta_max(pbm, red);
  pbs = cta_max(pbs, red);
  daff = cta_max(daff, red);
  dbm = cta_max(dbm, red);
  dbs = cta_max(dbs, red);
  dobj = cta_sum(dobj, red);
  compl_ = cta_sum(compl_, red);
  pobj = cta_sum(pobj, red);
  badx = cta_sum(badx, red);
  const double bX = cta_psd_certificate(X, k, tol_p, sm, red, sflag, out + cXsym);
  const double bY = cta_psd_certificate(Y, k, tol_d, sm, red, sflag, out + cYsym);
  if (threadIdx.x == 0) {
    out[cPobj] = pobj;
    out[cDobj] = dobj;
    out[cPaff] = paff;
    out[cDaff] = daff;
    out[cCompl] = compl_;
    out[cPbMixed] = pbm;
    out[cPbStrict] = pbs;
    out[cDbMixed] = dbm;
    out[cDbStrict] = dbs;
    out[cBadX] = badx + bX;
    out[cBadY] = bY;
  }
}

#include "batch_dd.cuh"

using PhaseKernel = void (*)(Pool, const int*, const double*, double*);
using WorkKernel = void (*)(Pool, const int*, const int4*);

}  // namespace

WorkKernel syrk_kernel(int threads, int tile) {
  if (tile == 16 && threads == 128) return k_b_syrk<128, 16>;
  if (tile == 16 && threads == 256) return k_b_syrk<256, 16>;
  if (tile == 32 && threads == 128) return k_b_syrk<128, 32>;
  if (tile == 32 && threads == 256) return k_b_syrk<256, 32>;
  if (tile == 32 && threads == 512) return k_b_syrk<512, 32>;
  return nullptr;
}

// ---------------------------------------------------------------------------
// Host side.

struct Pinned {
  void* p = nullptr;
  size_t bytes = 0;
  void ensure(size_t b) {
    if (b <= bytes) return;
    if (p) cudaFreeHost(p);
    p = nullptr;
    SDPX_CUDA(cudaHostAlloc(&p, b, cudaHostAllocDefault));
    bytes = b;
  }
  void release() {
    if (p) cudaFreeHost(p);
    p = nullptr;
    bytes = 0;
  }
  ~Pinned() { release(); }
};

// The loop state of one instance (CoreLoop of driver_api.inc, one block).
struct Run {
  ipm::Controller ctl;
  ipm::Stagnation stag;
  double mu = 0;
  int iter = 0, restarts = 0, centering = 0, attempts = 0;
  double pObj = 0, dObj = 0, p_res = INFINITY, d_res = INFINITY;
  double scale_p = 1, scale_d = 1;
  double best_merit = INFINITY, initial_merit = INFINITY, current_compl = 0;
  bool have_best = false;
  double best_pObj = 0, best_dObj = 0, best_p = 0, best_d = 0;
  int best_iter = 0;
  int status = 0;
  std::string message;
  bool restore = false;
  // per-pass scratch
  bool term_ok = false, gap_ok = false, stagnated = false;
  double gap_rel = 0;
  double sp_res = 0, sd_res = 0, bpr = 0, pm = 1, dm = 1, fq = 0;
  int att = 0;
  bool adaptive = false;
  double beta0 = 0.1;
  double cmpl = 0, aff = 0, aff_full = 0, mu_pd = 0, mu_aff = 0, quality = 0, atX = 1, atY = 1;
  ipm::Params params;
  double rtol = 0, abstol = 0, residual = 0, rnorm = 0;
  int rcap = 0, steps = 0;
  bool refining = false, consistent = true;
  double tX = 1, tY = 1;
};

struct Engine {
  dcache::ReleaseScope release_scope;  // first member: destroyed last
  int dev = 0;
  cudaStream_t st = nullptr;
  int N = 0, kmax = 0, mmax = 0;
  std::vector<Inst> inst;
  std::vector<double> scale_p, scale_d;
  DBuf<Inst> d_inst;
  DBuf<double> A, Ph, C, c, X, Y, P, R, LX, LY, W, dX, dY, Z, Xb, Yb;
  DBuf<double> x, dx, d, r, rho, xb, dxb, S, LS;
  DBuf<double> Pl, Rl, Zl, Xih, Xil, dl, rl, dxl, dxbl, rhol, Sl, LSl, Gl;  // Float64x2 mode
  long long kk_tot = 0, m_tot = 0, mm_tot = 0, a_tot = 0;
  bool dd = false;  // the current optimize runs the Float64x2 Newton system
  DBuf<int> d_act;
  DBuf<int4> d_work;
  DBuf<double> d_par, d_res;
  Pinned h_act, h_par, h_res, h_work;
  Pinned h_stage[2];          // upload staging (create only)
  cudaEvent_t ev_stage[2] = {nullptr, nullptr};
  Pool pool{};
  int schur_threads = 256, schur_tile = 32;
  // Affine fraction-to-boundary bounds: 0 the bisection of Cholesky trials
  // (eight at a time), 1 the eigenvalue bound −1/λ_min(L⁻¹·dM·L⁻ᵀ).
  int bound_mode = 1;
  double grain = 4.0e6;
  std::vector<Run> runs;
  std::string err;
  cudaEvent_t ev[2] = {nullptr, nullptr};
  // counters of the last optimize
  long long passes = 0, launches = 0, inst_iters = 0;
  double t_loop = 0, t_schur = 0, t_factor = 0, t_step = 0, schur_flops = 0;
  bool solved = false;

  ~Engine() {
    if (st) cudaStreamSynchronize(st);
    release_scope.begin();
    for (auto& e : ev)
      if (e) cudaEventDestroy(e);
    for (auto& e : ev_stage)
      if (e) cudaEventDestroy(e);
    if (st) cudaStreamDestroy(st);
  }

  size_t smem_bytes(int mats) const { return (size_t)mats * (size_t)pool.kq * sizeof(double); }
  // Packed lower triangles of X, dX and kTrialWarps trial slots (the step-length phases).
  size_t smem_trials() const {
    return (size_t)(2 + kTrialWarps) * (size_t)pool.kp * sizeof(double);
  }

  void create(const sdpx_b200_batch_problem* prob, int device) {
    if (!prob || prob->count <= 0) throw std::invalid_argument("empty batch");
    if (!prob->block_order || !prob->m || !prob->Av || !prob->C || !prob->c)
      throw std::invalid_argument("NULL array in the batch problem");
    N = prob->count;
    inst.resize(N);
    scale_p.assign(N, 1.0);
    scale_d.assign(N, 1.0);
    for (int i = 0; i < N; ++i) {
      const int k = prob->block_order[i], m = prob->m[i];
      if (k < 3 || k > kMaxK)
        throw std::invalid_argument("instance " + std::to_string(i) + ": block order " +
                                    std::to_string(k) + " outside [3, 64]");
      if (m < 1 || m > kMaxM)
        throw std::invalid_argument("instance " + std::to_string(i) + ": m = " +
                                    std::to_string(m) + " outside [1, 256]");
      if (!prob->Av[i] || !prob->C[i] || !prob->c[i])
        throw std::invalid_argument("instance " + std::to_string(i) + ": NULL data");
      Inst& I = inst[i];
      I.k = k;
      I.m = m;
      I.kk_off = kk_tot;
      I.m_off = m_tot;
      I.mm_off = mm_tot;
      I.a_off = a_tot;
      kk_tot += (long long)k * k;
      m_tot += m;
      mm_tot += (long long)m * m;
      a_tot += (long long)k * k * m;
      kmax = std::max(kmax, k);
      mmax = std::max(mmax, m);
    }
    dev = device;  // sizes checked first: usage errors need no device
    SDPX_CUDA(cudaSetDevice(dev));
    SDPX_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    for (auto& e : ev) SDPX_CUDA(cudaEventCreate(&e));
    for (auto& e : ev_stage) SDPX_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    d_inst.alloc(N);
    A.alloc(a_tot);
    Ph.alloc(a_tot);
    for (DBuf<double>* b : {&C, &X, &Y, &P, &R, &LX, &LY, &W, &dX, &dY, &Z, &Xb, &Yb})
      b->alloc(kk_tot);
    for (DBuf<double>* b : {&c, &x, &dx, &d, &r, &rho, &xb, &dxb}) b->alloc(m_tot);
    S.alloc(mm_tot);
    LS.alloc(mm_tot);
    SDPX_CUDA(cudaMemcpyAsync(d_inst.p, inst.data(), N * sizeof(Inst), cudaMemcpyHostToDevice, st));
    upload_pooled(A.p, prob->Av, [&](int i) { return (long long)inst[i].k * inst[i].k * inst[i].m; });
    upload_pooled(C.p, prob->C, [&](int i) { return (long long)inst[i].k * inst[i].k; });
    upload_pooled(c.p, prob->c, [&](int i) { return (long long)inst[i].m; });
    h_stage[0].release();  // the engine keeps no pinned staging after the upload
    h_stage[1].release();
    for (int i = 0; i < N; ++i) {
      const Inst& I = inst[i];
      const long long kk = (long long)I.k * I.k;
      double mc = 0, mcc = 0;  // scale_p = 1 + ‖C‖max, scale_d = 1 + ‖c‖∞ (`data_norms`)
      for (long long e = 0; e < kk; ++e) mc = std::max(mc, std::fabs(prob->C[i][e]));
      for (int j = 0; j < I.m; ++j) mcc = std::max(mcc, std::fabs(prob->c[i][j]));
      scale_p[i] = 1.0 + mc;
      scale_d[i] = 1.0 + mcc;
    }
    {  // instances ranked by an estimate of their per-iteration work
      std::vector<int> order(N);
      std::iota(order.begin(), order.end(), 0);
      auto w = [&](int i) {
        const double k = inst[i].k, m = inst[i].m;
        return 4.0 * k * k * k + 4.0 * m * k * k + m * m * k * k / 64.0 + m * m * m / 3.0;
      };
      std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return w(a) > w(b); });
      work_rank.assign(N, 0);
      for (int r = 0; r < N; ++r) work_rank[order[r]] = r;
    }
    d_act.alloc(N);
    d_par.alloc((size_t)N * kNIn);
    d_res.alloc((size_t)N * oNOut);
    h_act.ensure(N * sizeof(int));
    h_par.ensure((size_t)N * kNIn * sizeof(double));
    h_res.ensure((size_t)N * oNOut * sizeof(double));
    pool.inst = d_inst.p;
    pool.A = A.p;
    pool.Ph = Ph.p;
    pool.C = C.p;
    pool.c = c.p;
    pool.X = X.p, pool.Y = Y.p, pool.P = P.p, pool.R = R.p, pool.LX = LX.p, pool.LY = LY.p;
    pool.W = W.p, pool.dX = dX.p, pool.dY = dY.p, pool.Z = Z.p, pool.Xb = Xb.p, pool.Yb = Yb.p;
    pool.x = x.p, pool.dx = dx.p, pool.d = d.p, pool.r = r.p, pool.rho = rho.p;
    pool.xb = xb.p, pool.dxb = dxb.p, pool.S = S.p, pool.LS = LS.p;
    pool.kq = (long long)kmax * kmax;
    pool.kp = (long long)kmax * (kmax + 1) / 2;
    for (PhaseKernel kf : {k_b_residuals, k_b_rhs, k_b_dirblocks})
      SDPX_CUDA(cudaFuncSetAttribute(kf, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)smem_bytes(3)));
    for (PhaseKernel kf : {k_b_affine, k_b_linesearch})
      SDPX_CUDA(cudaFuncSetAttribute(kf, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)std::max(smem_trials(), smem_bytes(3))));
    SDPX_CUDA(cudaFuncSetAttribute(k_b_panel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)smem_bytes(4)));
    SDPX_CUDA(cudaStreamSynchronize(st));
  }

  // Float64x2 arrays, allocated by the first Float64x2 solve.
  void ensure_dd() {
    if (Gl.p) return;
    for (DBuf<double>* b : {&Pl, &Rl, &Zl, &Xih, &Xil}) b->alloc(kk_tot);
    for (DBuf<double>* b : {&dl, &rl, &dxl, &dxbl, &rhol}) b->alloc(m_tot);
    Sl.alloc(mm_tot);
    LSl.alloc(mm_tot);
    Gl.alloc(a_tot);
    for (DBuf<double>* b : {&dxl, &dxbl}) b->zero(st);
    pool.Pl = Pl.p, pool.Rl = Rl.p, pool.Zl = Zl.p, pool.Xih = Xih.p, pool.Xil = Xil.p;
    pool.dl = dl.p, pool.rl = rl.p, pool.dxl = dxl.p, pool.dxbl = dxbl.p, pool.rhol = rhol.p;
    pool.Sl = Sl.p, pool.LSl = LSl.p, pool.Gl = Gl.p;
    for (PhaseKernel kf : {k_dd_resid, k_dd_xinv, k_dd_rhs, k_dd_dirblocks})
      SDPX_CUDA(cudaFuncSetAttribute(kf, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)smem_bytes(5)));
    SDPX_CUDA(cudaFuncSetAttribute(k_dd_schur, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)smem_bytes(5)));
    SDPX_CUDA(cudaStreamSynchronize(st));
  }

  // ------------------------------------------------------- phase launches --
  // One launch of `kf` over the instances `ids` (one CTA each); `fill` writes
  // each row's inputs.  With `read`, waits and returns the output rows.
  template <class Fill>
  const double* phase(PhaseKernel kf, const std::vector<int>& ids, size_t smem, Fill fill,
                      bool read) {
    const int n = (int)ids.size();
    if (n == 0) return nullptr;
    // The staging buffers are reused by every launch: the copies queued from
    // them by the previous one must have run first.
    SDPX_CUDA(cudaStreamSynchronize(st));
    // CTAs in decreasing order of the instance's work (largest first, so the
    // last wave of a phase holds small instances); rows map back to `ids`.
    lpt.resize(n);
    std::iota(lpt.begin(), lpt.end(), 0);
    std::stable_sort(lpt.begin(), lpt.end(),
                     [&](int a, int b) { return work_rank[ids[a]] < work_rank[ids[b]]; });
    int* ha = static_cast<int*>(h_act.p);
    double* hp = static_cast<double*>(h_par.p);
    std::memset(hp, 0, (size_t)n * kNIn * sizeof(double));
    for (int q = 0; q < n; ++q) {
      ha[q] = ids[lpt[q]];
      fill(ids[lpt[q]], hp + (size_t)q * kNIn);
    }
    SDPX_CUDA(cudaMemcpyAsync(d_act.p, ha, n * sizeof(int), cudaMemcpyHostToDevice, st));
    SDPX_CUDA(cudaMemcpyAsync(d_par.p, hp, (size_t)n * kNIn * sizeof(double),
                              cudaMemcpyHostToDevice, st));
    kf<<<n, kThreads, smem, st>>>(pool, d_act.p, d_par.p, d_res.p);
    SDPX_LAUNCH_CHECK();
    ++launches;
    if (!read) return nullptr;
    SDPX_CUDA(cudaMemcpyAsync(h_res.p, d_res.p, (size_t)n * oNOut * sizeof(double),
                              cudaMemcpyDeviceToHost, st));
    SDPX_CUDA(cudaStreamSynchronize(st));
    const double* launched = static_cast<const double*>(h_res.p);
    rows.resize((size_t)n * oNOut);
    for (int q = 0; q < n; ++q)
      std::memcpy(rows.data() + (size_t)lpt[q] * oNOut, launched + (size_t)q * oNOut,
                  oNOut * sizeof(double));
    return rows.data();
  }
  std::vector<int> lpt, work_rank;  // launch order; rank of each instance by work
  std::vector<double> rows;         // output rows in the caller's order
  const double* phase(PhaseKernel kf, const std::vector<int>& ids, size_t smem, bool read) {
    return phase(kf, ids, smem, [](int, double*) {}, read);
  }

  // The double-double Schur assembly over `ids`: work items of contiguous
  // constraint ranges (about 2·10⁶ double-double multiply-adds each), largest
  // instances first.
  void schur_dd(const std::vector<int>& ids) {
    const int n = (int)ids.size();
    if (n == 0) return;
    SDPX_CUDA(cudaStreamSynchronize(st));
    int* ha = static_cast<int*>(h_act.p);
    std::vector<int> order(n);
    std::iota(order.begin(), order.end(), 0);
    auto cost = [&](int q) {
      const Inst& I = inst[ids[q]];
      return (2.0 * I.k * I.k * I.k + (double)I.k * I.k * I.m) * I.m;
    };
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return cost(a) > cost(b); });
    std::vector<int4> items;
    for (int q = 0; q < n; ++q) ha[q] = ids[q];
    for (int q : order) {
      const Inst& I = inst[ids[q]];
      const int parts = std::max(1, std::min(I.m, (int)std::ceil(cost(q) / 2.0e6)));
      for (int p = 0; p < parts; ++p)
        items.push_back(make_int4(q, (int)((long long)I.m * p / parts),
                                  (int)((long long)I.m * (p + 1) / parts), 0));
      schur_flops += 20.0 * cost(q);
    }
    if (d_work.n < items.size()) d_work.alloc(items.size() + items.size() / 4);
    h_work.ensure(items.size() * sizeof(int4));
    std::copy(items.begin(), items.end(), static_cast<int4*>(h_work.p));
    SDPX_CUDA(cudaMemcpyAsync(d_act.p, ha, n * sizeof(int), cudaMemcpyHostToDevice, st));
    SDPX_CUDA(cudaMemcpyAsync(d_work.p, h_work.p, items.size() * sizeof(int4),
                              cudaMemcpyHostToDevice, st));
    SDPX_CUDA(cudaEventRecord(ev[0], st));
    k_dd_schur<<<(int)items.size(), kThreads, smem_bytes(5), st>>>(pool, d_act.p, d_work.p);
    SDPX_LAUNCH_CHECK();
    SDPX_CUDA(cudaEventRecord(ev[1], st));
    ++launches;
    SDPX_CUDA(cudaEventSynchronize(ev[1]));
    float ms = 0;
    SDPX_CUDA(cudaEventElapsedTime(&ms, ev[0], ev[1]));
    t_schur += ms * 1e-3;
  }

  // The Schur assembly on the FP64 tensor cores: three grouped DMMA products
  // (T = W·A, P̂ = T·L_Y, S = P̂P̂ᵀ), work items of about `g` flops, largest first.
  DBuf<double> Tbuf;  // one k×k scratch per fused T·P̂ work item
  bool dmma_attrs = false;
  void schur_dmma(const std::vector<int>& ids, double g) {
    const int n = (int)ids.size();
    if (n == 0) return;
    if (!dmma_attrs) {
      SDPX_CUDA(cudaFuncSetAttribute(k_b_dmma_tp<DmmaCfgKN>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)DmmaCfgKN::SMEM_BYTES));
      SDPX_CUDA(cudaFuncSetAttribute(k_b_dmma_syrk<DmmaCfgKK>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)DmmaCfgKK::SMEM_BYTES));
      dmma_attrs = true;
    }
    SDPX_CUDA(cudaStreamSynchronize(st));
    int* ha = static_cast<int*>(h_act.p);
    std::vector<int> order(n);
    std::iota(order.begin(), order.end(), 0);
    auto cost = [&](int q) {
      const Inst& I = inst[ids[q]];
      return 4.0 * I.k * I.k * I.k * I.m + (double)I.k * I.k * I.m * I.m;
    };
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return cost(a) > cost(b); });
    // Per instance the tile that pads least: 32 for T·P̂ when k ≤ 32 (one k×k
    // tile per constraint) and for the SYRK when m ≤ 64, else 64.
    std::vector<int4> tp64, tp32, sy64, sy32;
    auto split = [&](std::vector<int4>& w, int q, int units, double flops) {
      int parts = g > 0 ? (int)std::ceil(flops / g) : 1;
      parts = std::max(1, std::min(parts, units));
      for (int p = 0; p < parts; ++p)
        w.push_back(make_int4(q, (int)((long long)units * p / parts),
                              (int)((long long)units * (p + 1) / parts), 0));
    };
    for (int q = 0; q < n; ++q) ha[q] = ids[q];
    for (int q : order) {
      const Inst& I = inst[ids[q]];
      split(I.k <= 32 ? tp32 : tp64, q, I.m, 4.0 * I.k * I.k * I.k * I.m);
      const int T = I.m <= 64 ? 32 : 64;
      const int nt = (I.m + T - 1) / T, tri = nt * (nt + 1) / 2;
      split(T == 32 ? sy32 : sy64, q, tri, (double)I.k * I.k * I.m * I.m);
      schur_flops += 2.0 * I.k * I.k * I.k * I.m + (double)I.k * I.k * I.m * I.m;
    }
    const size_t ntp = tp64.size() + tp32.size();
    if (Tbuf.n < ntp * (size_t)pool.kq) {
      Tbuf.alloc(ntp * (size_t)pool.kq + ntp * (size_t)pool.kq / 4);
      pool.T = Tbuf.p;
    }
    const size_t nw = ntp + sy64.size() + sy32.size();
    if (d_work.n < nw) d_work.alloc(nw + nw / 4);
    h_work.ensure(nw * sizeof(int4));
    int4* hw = static_cast<int4*>(h_work.p);
    size_t o = 0;
    for (auto* w : {&tp64, &tp32, &sy64, &sy32}) {
      std::copy(w->begin(), w->end(), hw + o);
      o += w->size();
    }
    SDPX_CUDA(cudaMemcpyAsync(d_act.p, ha, n * sizeof(int), cudaMemcpyHostToDevice, st));
    SDPX_CUDA(cudaMemcpyAsync(d_work.p, hw, nw * sizeof(int4), cudaMemcpyHostToDevice, st));
    SDPX_CUDA(cudaEventRecord(ev[0], st));
    // The T·P̂ kernels index their scratch by blockIdx.x: the 32-tile launch
    // takes the slots after the 64-tile one's.
    Pool p32 = pool;
    p32.T = pool.T + (long long)tp64.size() * pool.kq;
    const int4* w = d_work.p;
    if (!tp64.empty()) {
      k_b_dmma_tp<DmmaCfgKN><<<(int)tp64.size(), DmmaCfgKN::NT, DmmaCfgKN::SMEM_BYTES, st>>>(
          pool, d_act.p, w);
      SDPX_LAUNCH_CHECK();
    }
    w += tp64.size();
    if (!tp32.empty()) {
      k_b_dmma_tp<DmmaCfgKN32><<<(int)tp32.size(), DmmaCfgKN32::NT, DmmaCfgKN32::SMEM_BYTES,
                                 st>>>(p32, d_act.p, w);
      SDPX_LAUNCH_CHECK();
    }
    w += tp32.size();
    if (!sy64.empty()) {
      k_b_dmma_syrk<DmmaCfgKK><<<(int)sy64.size(), DmmaCfgKK::NT, DmmaCfgKK::SMEM_BYTES, st>>>(
          pool, d_act.p, w);
      SDPX_LAUNCH_CHECK();
    }
    w += sy64.size();
    if (!sy32.empty()) {
      k_b_dmma_syrk<DmmaCfgKK32><<<(int)sy32.size(), DmmaCfgKK32::NT, DmmaCfgKK32::SMEM_BYTES,
                                   st>>>(pool, d_act.p, w);
      SDPX_LAUNCH_CHECK();
    }
    SDPX_CUDA(cudaEventRecord(ev[1], st));
    launches += (tp64.empty() ? 0 : 1) + (tp32.empty() ? 0 : 1) + (sy64.empty() ? 0 : 1) +
                (sy32.empty() ? 0 : 1);
    SDPX_CUDA(cudaEventSynchronize(ev[1]));
    float ms = 0;
    SDPX_CUDA(cudaEventElapsedTime(&ms, ev[0], ev[1]));
    t_schur += ms * 1e-3;
  }

  // The Schur assembly over `ids`: panel then SYRK work items, largest first
  // (tile 64: the DMMA products of schur_dmma).
  void schur(const std::vector<int>& ids, int threads, int tile, double g) {
    const int n = (int)ids.size();
    if (n == 0) return;
    if (tile == 64) {
      schur_dmma(ids, g);
      return;
    }
    WorkKernel syrk = syrk_kernel(threads, tile);
    if (!syrk) throw std::invalid_argument("unsupported Schur launch shape");
    SDPX_CUDA(cudaStreamSynchronize(st));
    int* ha = static_cast<int*>(h_act.p);
    std::vector<int> order(n);
    std::iota(order.begin(), order.end(), 0);
    auto cost = [&](int q) {
      const Inst& I = inst[ids[q]];
      return 2.0 * I.k * I.k * I.k * I.m + (double)I.k * I.k * I.m * I.m;
    };
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return cost(a) > cost(b); });
    std::vector<int4> panel, syr;
    for (int q = 0; q < n; ++q) ha[q] = ids[q];
    for (int q : order) {
      const Inst& I = inst[ids[q]];
      const double pf = 2.0 * I.k * I.k * I.k * I.m;
      const int nt = (I.m + tile - 1) / tile, ntiles = nt * (nt + 1) / 2;
      const double sf = (double)I.k * I.k * I.m * I.m;
      int pp = g > 0 ? (int)std::ceil(pf / g) : 1;
      int sp = g > 0 ? (int)std::ceil(sf / g) : 1;
      pp = std::max(1, std::min(pp, I.m));
      sp = std::max(1, std::min(sp, ntiles));
      for (int p = 0; p < pp; ++p)
        panel.push_back(make_int4(q, (int)((long long)I.m * p / pp),
                                  (int)((long long)I.m * (p + 1) / pp), 0));
      for (int p = 0; p < sp; ++p)
        syr.push_back(make_int4(q, (int)((long long)ntiles * p / sp),
                                (int)((long long)ntiles * (p + 1) / sp), 0));
      schur_flops += pf + sf;
    }
    const size_t nw = panel.size() + syr.size();
    if (d_work.n < nw) d_work.alloc(nw + nw / 4);
    h_work.ensure(nw * sizeof(int4));
    int4* hw = static_cast<int4*>(h_work.p);
    std::copy(panel.begin(), panel.end(), hw);
    std::copy(syr.begin(), syr.end(), hw + panel.size());
    SDPX_CUDA(cudaMemcpyAsync(d_act.p, ha, n * sizeof(int), cudaMemcpyHostToDevice, st));
    SDPX_CUDA(cudaMemcpyAsync(d_work.p, hw, nw * sizeof(int4), cudaMemcpyHostToDevice, st));
    SDPX_CUDA(cudaEventRecord(ev[0], st));
    k_b_panel<<<(int)panel.size(), threads, smem_bytes(4), st>>>(pool, d_act.p, d_work.p);
    SDPX_LAUNCH_CHECK();
    syrk<<<(int)syr.size(), threads, 0, st>>>(pool, d_act.p, d_work.p + panel.size());
    SDPX_LAUNCH_CHECK();
    SDPX_CUDA(cudaEventRecord(ev[1], st));
    launches += 2;
    SDPX_CUDA(cudaEventSynchronize(ev[1]));
    float ms = 0;
    SDPX_CUDA(cudaEventElapsedTime(&ms, ev[0], ev[1]));
    t_schur += ms * 1e-3;
  }

  // ---------------------------------------------------------------- loop --
  static double gap_rel_of(double p, double q) {
    return std::fabs(p - q) / std::max(1.0, (std::fabs(p) + std::fabs(q)) / 2);
  }

  // Loop exit and the best-iterate rule (CoreLoop::finish).
  void finish(const sdpx_b200_solve_options& o, Run& R, int st_code, const std::string& msg) {
    R.status = st_code;
    R.message = msg;
    if (st_code != SDPX_B200_STATUS_OPTIMAL && R.have_best) {
      const double gr = gap_rel_of(R.pObj, R.dObj);
      const double final_merit =
          ipm::merit_of(o, R.p_res, R.d_res, gr, R.current_compl, R.scale_p, R.scale_d,
                        std::max(std::fabs(R.pObj), std::fabs(R.dObj)));
      if (!std::isfinite(final_merit) || R.best_merit < final_merit / 2) {
        R.restore = true;
        R.pObj = R.best_pObj;
        R.dObj = R.best_dObj;
        R.p_res = R.best_p;
        R.d_res = R.best_d;
        R.message +=
            " Returned the best iterate found (iteration " + std::to_string(R.best_iter) + ").";
      }
    }
  }

  static void check_options(const sdpx_b200_solve_options& o) {
    if (o.parameter_policy != 1)
      throw std::invalid_argument("the batched engine runs the fixed start (parameter_policy = 1)");
    if (o.scaling != 1)
      throw std::invalid_argument("the batched engine runs without equilibration (scaling = 1)");
    if (o.precision != SDPX_B200_FP64 && o.precision != SDPX_B200_FLOAT64X2)
      throw std::invalid_argument(
          "the batched engine runs in FP64 or Float64x2 (precision = SDPX_B200_FP64 or "
          "SDPX_B200_FLOAT64X2)");
    if (o.step_rule == 2)
      throw std::invalid_argument("the batched engine runs the backtracking step rule");
  }

  void optimize(const sdpx_b200_solve_options& o, sdpx_b200_solve_result* results) {
    check_options(o);
    const auto t0 = std::chrono::steady_clock::now();
    auto elapsed = [&] {
      return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    };
    dd = o.precision == SDPX_B200_FLOAT64X2;
    if (dd) ensure_dd();
    // Kernels of the Newton system in the chosen arithmetic.
    const PhaseKernel K_factor = dd ? k_dd_factor : k_b_factor;
    const PhaseKernel K_rhs = dd ? k_dd_rhs : k_b_rhs;
    const PhaseKernel K_solve = dd ? k_dd_solve : k_b_solve;
    const PhaseKernel K_dir = dd ? k_dd_dirblocks : k_b_dirblocks;
    const PhaseKernel K_rho = dd ? k_dd_rho : k_b_resid;
    const PhaseKernel K_back = dd ? k_dd_rollback : k_b_rollback;
    const size_t smem_blk = dd ? smem_bytes(5) : smem_bytes(3);
    passes = launches = inst_iters = 0;
    t_schur = t_factor = t_step = schur_flops = 0;
    runs.assign(N, Run{});
    std::vector<int> all(N);
    std::iota(all.begin(), all.end(), 0);
    const double sqrt_eps = ipm::sqrt_eps();
    // begin (CoreLoop::begin with the fixed start, no equilibration)
    phase(k_b_elementwise, all, 0, [&](int, double* in) {
      in[kMode] = 0;
      in[kTX] = o.omega_p;
      in[kTY] = o.omega_d;
    }, false);
    const double* out = phase(k_b_state, all, 0, true);
    for (int q = 0; q < N; ++q) {
      Run& R = runs[all[q]];
      const Inst& I = inst[all[q]];
      const double* ro = out + (size_t)q * oNOut;
      R.mu = o.beta * ro[oCompl] / I.k;
      R.ctl.init(o);
      R.pObj = ro[oPobj];
      R.dObj = ro[oDobj];
      R.current_compl = ro[oCompl];
      R.stag.init(o.stall_iterations, o.stall_tolerance);
      R.scale_p = scale_p[all[q]];
      R.scale_d = scale_d[all[q]];
    }
    out = phase(k_b_residuals, all, smem_bytes(2), [&](int id, double* in) {
      in[kMu] = runs[id].mu;
      in[kUseAffine] = runs[id].ctl.strategy_adaptive() ? 1 : 0;
      in[kFactor] = 0;
    }, true);
    if (dd)  // the same residuals in double-double
      out = phase(k_dd_resid, all, smem_bytes(2), [&](int id, double* in) {
        in[kMu] = runs[id].mu;
        in[kUseAffine] = runs[id].ctl.strategy_adaptive() ? 1 : 0;
      }, true);
    for (int q = 0; q < N; ++q) {
      Run& R = runs[all[q]];
      R.p_res = out[(size_t)q * oNOut + oPres];
      R.d_res = out[(size_t)q * oNOut + oDres];
    }
    const double term_tol = o.eps_gap;
    const double adaptive_margin = o.parameter_strategy == 0 ? sqrt_eps : 0.0;

    std::vector<int> running = all;
    while (!running.empty()) {
      ++passes;
      // ---- termination tests (CoreLoop::step, top)
      std::vector<int> need;
      for (int id : running) {
        Run& R = runs[id];
        R.gap_rel = gap_rel_of(R.pObj, R.dObj);
        R.term_ok = R.p_res / R.scale_p <= o.eps_primal && R.d_res / R.scale_d <= o.eps_dual;
        R.gap_ok = R.gap_rel <= term_tol;
        if (R.term_ok && R.gap_ok) need.push_back(id);
      }
      out = dd ? phase(k_dd_resid, need, smem_bytes(2), [](int, double* in) { in[kMode] = 1; },
                       true)
               : phase(k_b_solres, need, 0, true);
      for (size_t q = 0; q < need.size(); ++q) {
        Run& R = runs[need[q]];
        R.p_res = out[q * oNOut + oPres];
        R.d_res = out[q * oNOut + oDres];
        R.term_ok = R.p_res / R.scale_p <= o.eps_primal && R.d_res / R.scale_d <= o.eps_dual;
      }
      std::vector<int> save, stepping;
      const bool out_of_time = elapsed() > o.max_time;
      for (int id : running) {
        Run& R = runs[id];
        const double merit = ipm::merit_of(o, R.p_res, R.d_res, R.gap_rel, R.current_compl,
                                           R.scale_p, R.scale_d,
                                           std::max(std::fabs(R.pObj), std::fabs(R.dObj)));
        const bool floor_reached =
            ipm::precision_floor(R.p_res, R.d_res, R.gap_rel, R.scale_p, R.scale_d);
        R.stagnated = R.stag.observe(merit, floor_reached, (long long)o.iter_max - R.iter);
        if (std::isfinite(merit) && !std::isfinite(R.initial_merit)) R.initial_merit = merit;
        if (std::isfinite(merit) && merit < R.best_merit) {
          R.best_merit = merit;
          save.push_back(id);
          R.have_best = true;
          R.best_pObj = R.pObj;
          R.best_dObj = R.dObj;
          R.best_p = R.p_res;
          R.best_d = R.d_res;
          R.best_iter = R.iter;
        }
        if (R.term_ok && R.gap_ok) finish(o, R, SDPX_B200_STATUS_OPTIMAL, "Optimal");
        else if (R.iter >= o.iter_max)
          finish(o, R, SDPX_B200_STATUS_ITER_LIMIT,
                 "Cannot reach optimality within " + std::to_string(o.iter_max) + " iterations.");
        else if (R.stagnated)
          finish(o, R,
                 R.stag.reason == 1 ? SDPX_B200_STATUS_INSUFFICIENT_PRECISION
                                    : SDPX_B200_STATUS_STALLED,
                 "Convergence stagnated.");
        else if (out_of_time)
          finish(o, R, SDPX_B200_STATUS_TIME_LIMIT, "Time limit exceeded.");
        else
          stepping.push_back(id);
      }
      phase(k_b_elementwise, save, 0, [](int, double* in) { in[kMode] = 1; }, false);

      // ---- newton_step (src/step.jl:643-1023)
      for (int id : stepping) {
        Run& R = runs[id];
        ++R.attempts;
        R.adaptive = R.ctl.strategy_adaptive();  // use_affine
        R.beta0 = R.ctl.beta;
      }
      out = phase(k_b_residuals, stepping, smem_bytes(2), [&](int id, double* in) {
        in[kMu] = runs[id].mu;
        in[kUseAffine] = runs[id].adaptive ? 1 : 0;
        in[kFactor] = 1;
      }, true);
      std::vector<int> ok1;
      for (size_t q = 0; q < stepping.size(); ++q) {
        Run& R = runs[stepping[q]];
        const double* ro = out + q * oNOut;
        R.sp_res = ro[oPres];
        R.sd_res = ro[oDres];
        R.bpr = ro[oPres];
        R.pm = ro[oPmargin];
        R.dm = ro[oDmargin];
        if (ro[oOk] == 0.0)
          finish(o, R, SDPX_B200_STATUS_NUMERICAL_BREAKDOWN,
                 "Cholesky factorization of X or Y failed (iterate left the interior)");
        else
          ok1.push_back(stepping[q]);
      }
      if (dd) {  // P, d, R and X⁻¹ in double-double
        out = phase(k_dd_resid, ok1, smem_bytes(2), [&](int id, double* in) {
          in[kMu] = runs[id].mu;
          in[kUseAffine] = runs[id].adaptive ? 1 : 0;
        }, true);
        for (size_t q = 0; q < ok1.size(); ++q) {
          Run& R = runs[ok1[q]];
          R.sp_res = R.bpr = out[q * oNOut + oPres];
          R.sd_res = out[q * oNOut + oDres];
        }
        phase(k_dd_xinv, ok1, smem_bytes(5), false);
        schur_dd(ok1);
      } else {
        schur(ok1, schur_threads, schur_tile, grain);
      }
      const auto tf0 = std::chrono::steady_clock::now();
      out = phase(K_factor, ok1, 0, true);
      t_factor += std::chrono::duration<double>(std::chrono::steady_clock::now() - tf0).count();
      std::vector<int> ok2;
      for (size_t q = 0; q < ok1.size(); ++q) {
        Run& R = runs[ok1[q]];
        const double* ro = out + q * oNOut;
        R.att = (int)ro[oReg];
        R.fq = ro[oQual];
        if (ro[oOk] == 0.0)
          finish(o, R, SDPX_B200_STATUS_NUMERICAL_BREAKDOWN,
                 "Schur complement not positive definite after " + std::to_string(R.att) +
                     " regularization attempt(s)");
        else
          ok2.push_back(ok1[q]);
      }
      // predictor
      phase(K_rhs, ok2, smem_blk, [](int, double* in) { in[kMode] = 0; }, false);
      phase(K_solve, ok2, 0, [](int, double* in) { in[kMode] = 0; }, false);
      phase(K_dir, ok2, smem_blk, false);
      const auto tl0 = std::chrono::steady_clock::now();
      out = phase(k_b_affine, ok2, bound_mode == 1 ? smem_bytes(3) : smem_trials(),
                  [&](int id, double* in) {
        const Run& R = runs[id];
        in[kMode] = (R.adaptive && !R.ctl.fallback) ? 1 : 0;
        in[kBoundMode] = bound_mode;
      }, true);
      t_step += std::chrono::duration<double>(std::chrono::steady_clock::now() - tl0).count();
      for (size_t q = 0; q < ok2.size(); ++q) {
        const int id = ok2[q];
        Run& R = runs[id];
        const Inst& I = inst[id];
        const double* ro = out + q * oNOut;
        const bool adaptive = R.adaptive && !R.ctl.fallback;
        R.cmpl = ro[oCompl];
        R.aff = ro[oAff];
        R.aff_full = ro[oAffFull];
        R.atX = ro[oTX];
        R.atY = ro[oTY];
        const double den = (double)std::max(I.k, 1);
        R.mu_pd = R.cmpl / den;
        R.mu_aff = std::max(0.0, R.aff / den);
        if (adaptive)
          R.quality = R.mu_pd > 0 ? std::min(std::max(R.mu_aff / R.mu_pd, 0.0), 2.0) : 1.0;
        else
          R.quality = R.cmpl > 0 ? std::min(std::max(R.aff / R.cmpl, 0.0), 2.0) : 1.0;
        const auto& hist = R.ctl.history;
        const double prev_tX = hist.empty() ? 1.0 : hist.back().primal_step;
        const double prev_tY = hist.empty() ? 1.0 : hist.back().dual_step;
        const long long prev_bt = hist.empty() ? 0 : hist.back().backtracking_count;
        const int prev_ref = hist.empty() ? 0 : hist.back().refinement_count;
        const double cur_feas = std::max(R.sp_res / std::max(R.scale_p, 1.0),
                                         R.sd_res / std::max(R.scale_d, 1.0));
        double prev_achieved = 1.0;
        if (!hist.empty()) {
          const auto& row = hist.back();
          const double prev_feas =
              std::max(row.primal_residual / std::max(R.scale_p, 1.0),
                       std::max(row.dual_residual / std::max(R.scale_d, 1.0), ipm::kEpsD));
          prev_achieved = cur_feas / prev_feas;
        }
        ipm::Diag dg;
        dg.iteration = R.iter + 1;
        dg.primal_residual = R.sp_res / std::max(R.scale_p, 1.0);
        dg.dual_residual = R.sd_res / std::max(R.scale_d, 1.0);
        dg.relative_gap = R.gap_rel;
        dg.mu = R.mu_pd;
        dg.mu_aff = R.mu_aff;
        dg.affine_primal_step = R.atX;
        dg.affine_dual_step = R.atY;
        dg.previous_primal_step = prev_tX;
        dg.previous_dual_step = prev_tY;
        dg.backtracking_count = prev_bt;
        dg.regularization = ipm::relative_regularization(R.att);
        dg.refinement_count = prev_ref;
        dg.factorization_quality = R.fq;
        dg.achieved_residual_reduction = prev_achieved;
        dg.primal_psd_margin = R.pm;
        dg.dual_psd_margin = R.dm;
        dg.precision_floor =
            ipm::precision_floor(R.sp_res, R.sd_res, R.gap_rel, R.scale_p, R.scale_d);
        R.params = R.ctl.select(dg);
        if (adaptive && !R.params.fallback) {
          R.rtol = R.params.refinement_tolerance;
          R.rcap = R.params.refinement_max_count;
        } else {
          R.rtol = o.refine_tol;
          R.rcap = o.refine_max_steps;
        }
        R.adaptive = adaptive;  // as evaluated before the controller's selection
      }
      // corrector
      phase(K_rhs, ok2, smem_blk, [&](int id, double* in) {
        const Run& R = runs[id];
        const Inst& I = inst[id];
        in[kMode] = 1;
        if (R.adaptive && !R.params.fallback) {
          // Mehrotra: σ·μ (the uniform and block-local targets agree for one block)
          in[kTarget] = R.params.sigma * R.mu_pd;
        } else {  // `rhs_corrector_fixed` with ⟨X + dX, Y + dY⟩
          const double rl = R.aff_full / R.mu / I.k;
          const double gl = std::max(rl < 1 ? rl * rl : rl, R.beta0);
          in[kTarget] = gl * R.mu;
        }
      }, false);
      phase(K_solve, ok2, 0, [](int, double* in) { in[kMode] = 0; }, false);
      out = phase(K_rho, ok2, 0, true);
      std::vector<int> refining;
      for (size_t q = 0; q < ok2.size(); ++q) {
        Run& R = runs[ok2[q]];
        R.residual = out[q * oNOut + oRes];
        R.rnorm = out[q * oNOut + oRnorm];
        R.steps = 0;
        R.consistent = true;
        const double rel = R.rtol > 0 ? R.rtol : ipm::kRefineUlps * ipm::kEpsD;
        R.abstol = rel * std::max(R.rnorm, 1.0);
        R.refining = o.refine_policy == 0 ? o.refine_steps > 0 : R.rcap > 0;
        if (R.refining) refining.push_back(ok2[q]);
      }
      // refinement rounds (Handle::refine, FP64 branch)
      while (true) {
        std::vector<int> round;
        for (int id : refining) {
          Run& R = runs[id];
          if (!R.refining) continue;
          const bool more = o.refine_policy == 0 ? R.steps < o.refine_steps
                                                 : (R.steps < R.rcap && R.residual > R.abstol);
          if (more) round.push_back(id);
          else R.refining = false;
        }
        if (round.empty()) break;
        phase(K_solve, round, 0, [](int, double* in) { in[kMode] = 1; }, false);
        out = phase(K_rho, round, 0, true);
        std::vector<int> back;
        for (size_t q = 0; q < round.size(); ++q) {
          Run& R = runs[round[q]];
          const double corr = out[q * oNOut + oRes];
          if (!std::isfinite(corr) || corr > R.residual) {
            back.push_back(round[q]);
            R.consistent = false;
            R.refining = false;
            continue;
          }
          ++R.steps;
          const bool small = corr > R.residual * 0.5;
          R.residual = corr;
          if (o.refine_policy != 0 && small) R.refining = false;
        }
        phase(K_back, back, 0, false);
        out = phase(K_rho, back, 0, true);  // ρ of the restored direction
        for (size_t q = 0; q < back.size(); ++q) runs[back[q]].residual = out[q * oNOut + oRes];
      }
      std::vector<int> ok3;
      for (int id : ok2) {
        Run& R = runs[id];
        const double dir_tol =
            std::max(sqrt_eps, std::max(o.eps_primal, o.eps_dual)) * std::max(R.rnorm, 1.0);
        if (!std::isfinite(R.residual) || R.residual > dir_tol)
          finish(o, R, SDPX_B200_STATUS_NUMERICAL_BREAKDOWN,
                 "final structured KKT direction residual exceeded the accepted tolerance");
        else
          ok3.push_back(id);
      }
      phase(K_dir, ok3, smem_blk, false);
      for (int id : ok3) {  // the step succeeded: its residuals become the loop's
        Run& R = runs[id];
        R.p_res = R.sp_res;
        R.d_res = R.sd_res;
      }
      const auto tl1 = std::chrono::steady_clock::now();
      out = phase(k_b_linesearch, ok3, smem_trials(), [&](int id, double* in) {
        const Run& R = runs[id];
        in[kGamma] = R.params.backtracking;
        in[kMinStep] = R.params.minimum_step;
        in[kRatio] = adaptive_margin;
      }, true);
      t_step += std::chrono::duration<double>(std::chrono::steady_clock::now() - tl1).count();
      std::vector<int> upd, centre, rescX, rescY;
      std::vector<char> restarted(N, 0);
      for (size_t q = 0; q < ok3.size(); ++q) {
        const int id = ok3[q];
        Run& R = runs[id];
        const ipm::Params& pr = R.params;
        R.tX = out[q * oNOut + oTX];
        R.tY = out[q * oNOut + oTY];
        const bool primal_feasible = R.p_res / R.scale_p <= o.eps_primal;
        const bool dual_feasible = R.d_res / R.scale_d <= o.eps_dual;
        bool x_stuck = R.tX < pr.minimum_step, y_stuck = R.tY < pr.minimum_step;
        if (x_stuck && primal_feasible && !y_stuck) {
          R.tX = 0.0;
          x_stuck = false;
        }
        if (y_stuck && dual_feasible && !x_stuck) {
          R.tY = 0.0;
          y_stuck = false;
        }
        if (!(x_stuck || y_stuck)) {
          upd.push_back(id);
          continue;
        }
        const double near_tol = 1000.0;
        const double gap_now = gap_rel_of(R.pObj, R.dObj);
        if (gap_now < near_tol * term_tol && R.p_res / R.scale_p < near_tol * o.eps_primal &&
            R.d_res / R.scale_d < near_tol * o.eps_dual) {
          finish(o, R, SDPX_B200_STATUS_STALLED,
                 "Step size collapsed near, but not within, the requested tolerance.");
          continue;
        }
        const bool made_progress = std::isfinite(R.initial_merit) &&
                                   R.best_merit < R.initial_merit * 1e-3 &&
                                   R.best_merit < ipm::kNearSolutionMerit;
        if (o.stall_iterations > 0 && made_progress) {
          finish(o, R, SDPX_B200_STATUS_INSUFFICIENT_PRECISION,
                 "Step size collapsed after the solve had already converged (precision "
                 "exhaustion).");
          continue;
        }
        if (R.centering < o.max_centering && R.ctl.beta < ipm::kCenteringBetaMax) {
          ++R.centering;
          R.ctl.beta = std::min(R.ctl.beta * ipm::kCenteringBetaStep, ipm::kCenteringBetaMax);
          centre.push_back(id);
          continue;
        }
        const bool rescale_X = x_stuck && !primal_feasible;
        const bool rescale_Y = y_stuck && !dual_feasible;
        if (o.restart && R.restarts < o.max_restarts && (rescale_X || rescale_Y)) {
          ++R.restarts;
          if (rescale_X) rescX.push_back(id);
          if (rescale_Y) rescY.push_back(id);
          restarted[id] = 1;
          centre.push_back(id);
          continue;
        }
        if (o.restart && R.restarts < o.max_restarts) {
          finish(o, R, SDPX_B200_STATUS_STALLED,
                 "Step size collapsed while both residuals were already within tolerance.");
          continue;
        }
        finish(o, R,
               R.restarts >= o.max_restarts ? SDPX_B200_STATUS_MAX_RESTARTS
                                            : SDPX_B200_STATUS_NUMERICAL_BREAKDOWN,
               "Step size collapsed.");
      }
      phase(k_b_elementwise, rescX, 0, [&](int id, double* in) {
        in[kMode] = 3;
        in[kOmega] = runs[id].params.restart_scale;
      }, false);
      phase(k_b_elementwise, rescY, 0, [&](int id, double* in) {
        in[kMode] = 4;
        in[kOmega] = runs[id].params.restart_scale;
      }, false);
      out = phase(k_b_state, centre, 0, true);  // μ from the block dots
      for (size_t q = 0; q < centre.size(); ++q) {
        Run& R = runs[centre[q]];
        const double dots = out[q * oNOut + oCompl];
        if (restarted[centre[q]]) R.current_compl = dots;
        R.mu = R.ctl.beta * dots / inst[centre[q]].k;
      }
      // update
      out = phase(k_b_update, upd, 0, [&](int id, double* in) {
        in[kTX] = runs[id].tX;
        in[kTY] = runs[id].tY;
      }, true);
      for (size_t q = 0; q < upd.size(); ++q) {
        const int id = upd[q];
        Run& R = runs[id];
        const Inst& I = inst[id];
        const double* ro = out + q * oNOut;
        if (ro[oFinite] == 0.0) {
          finish(o, R, SDPX_B200_STATUS_NUMERICAL_BREAKDOWN,
                 "non-finite primal or dual iterate detected");
          continue;
        }
        const double compl_after = ro[oCompl];
        const double p_after = std::fabs(1.0 - R.tX) * R.bpr;
        const double d_after = ro[oDa];
        const long long bt = ipm::estimate_backtracking(R.tX, R.params.backtracking, true) +
                             ipm::estimate_backtracking(R.tY, R.params.backtracking, true);
        R.ctl.record(R.iter + 1, R.cmpl, compl_after, R.p_res, R.d_res, R.tX, R.tY, p_after,
                     d_after, bt, R.steps, R.params);
        R.current_compl = compl_after;
        R.mu = R.ctl.beta * compl_after / std::max(I.k, 1);
        if (!std::isfinite(R.mu)) {
          finish(o, R, SDPX_B200_STATUS_NUMERICAL_BREAKDOWN,
                 "non-finite complementarity target detected");
          continue;
        }
        R.pObj = ro[oPobj];
        R.dObj = ro[oDobj];
        if (!(std::isfinite(R.pObj) && std::isfinite(R.dObj))) {
          finish(o, R, SDPX_B200_STATUS_NUMERICAL_BREAKDOWN,
                 "non-finite primal or dual objective detected");
          continue;
        }
        ++R.iter;
        ++inst_iters;
        R.p_res = p_after;
        R.d_res = d_after;
      }
      // restore the best iterate of the instances that ended in this pass
      std::vector<int> restore, still;
      for (int id : running) {
        Run& R = runs[id];
        if (R.status != 0) {
          if (R.restore) restore.push_back(id);
        } else {
          still.push_back(id);
        }
      }
      phase(k_b_elementwise, restore, 0, [](int, double* in) { in[kMode] = 2; }, false);
      running.swap(still);
    }
    // end: slack rebuilt from x, objectives and residuals on the data
    phase(k_b_elementwise, all, 0, [](int, double* in) { in[kMode] = 5; }, false);
    out = phase(k_b_state, all, 0, true);
    std::vector<double> po(N), dob(N);
    for (int q = 0; q < N; ++q) {
      po[q] = out[(size_t)q * oNOut + oPobj];
      dob[q] = out[(size_t)q * oNOut + oDobj];
    }
    out = dd ? phase(k_dd_resid, all, smem_bytes(2), [](int, double* in) { in[kMode] = 1; }, true)
             : phase(k_b_solres, all, 0, true);
    t_loop = elapsed();
    for (int i = 0; i < N; ++i) {
      const Run& R = runs[i];
      sdpx_b200_solve_result& rr = results[i];
      rr = sdpx_b200_solve_result{};
      rr.status = R.status;
      rr.iterations = R.iter;
      rr.restarts = R.restarts;
      rr.p_obj = po[i];
      rr.d_obj = dob[i];
      rr.p_res = out[(size_t)i * oNOut + oPres];
      rr.d_res = out[(size_t)i * oNOut + oDres];
      rr.seconds = t_loop;
      rr.fp64_iterations = R.attempts;
      std::snprintf(rr.message, sizeof(rr.message), "%s", R.message.c_str());
    }
    solved = true;
  }

  // Times every Schur launch shape on the current iterates (factored first).
  int autotune(const sdpx_b200_solve_options& o, double* table, int cap) {
    std::vector<int> all(N);
    std::iota(all.begin(), all.end(), 0);
    if (!solved) {
      phase(k_b_elementwise, all, 0, [&](int, double* in) {
        in[kMode] = 0;
        in[kTX] = o.omega_p;
        in[kTY] = o.omega_d;
      }, false);
    }
    const double* out =
        phase(k_b_residuals, all, smem_bytes(2), [](int, double* in) { in[kFactor] = 1; }, true);
    std::vector<int> ok;
    for (int q = 0; q < N; ++q)
      if (out[(size_t)q * oNOut + oOk] != 0.0) ok.push_back(q);
    if (ok.empty()) throw std::runtime_error("no instance has a positive definite iterate");
    struct Cand {
      int threads, tile;
      double grain;
    };
    std::vector<Cand> cands;
    const std::pair<int, int> shapes[] = {{128, 16}, {256, 16}, {128, 32},
                                          {256, 32}, {512, 32}, {128, 64}};
    for (double g : {0.0, 1.0e6, 4.0e6, 16.0e6})
      for (const auto& tt : shapes) cands.push_back({tt.first, tt.second, g});
    double best = INFINITY;
    Cand pick{schur_threads, schur_tile, grain};
    int row = 0;
    const double saved_flops = schur_flops, saved_t = t_schur;
    const long long saved_launches = launches;
    for (const Cand& cd : cands) {
      double ms_best = INFINITY;
      for (int rep = 0; rep < 3; ++rep) {
        const double before = t_schur;
        schur(ok, cd.threads, cd.tile, cd.grain);
        ms_best = std::min(ms_best, (t_schur - before) * 1e3);
      }
      if (table && row < cap) {
        table[4 * row + 0] = cd.threads;
        table[4 * row + 1] = cd.tile;
        table[4 * row + 2] = cd.grain;
        table[4 * row + 3] = ms_best;
      }
      ++row;
      if (ms_best < best) {
        best = ms_best;
        pick = cd;
      }
    }
    schur_flops = saved_flops;
    t_schur = saved_t;
    launches = saved_launches;
    schur_threads = pick.threads;
    schur_tile = pick.tile;
    grain = pick.grain;
    return row;
  }

  // Certificates of every instance's current solution (after optimize: the
  // returned iterate, original coordinates); one kernel, one read-back.
  DBuf<double> d_cert;
  Pinned h_cert;
  void certificate(double ep, double ed, double eg, int legacy,
                   sdpx_b200_certificate_result* results) {
    if (!solved)
      throw std::invalid_argument("no solution to certify: run sdpx_b200_batch_optimize or "
                                  "set every instance's solution first");
    if (d_cert.n < (size_t)N * kCertOut) d_cert.alloc((size_t)N * kCertOut);
    h_cert.ensure((size_t)N * kCertOut * sizeof(double));
    SDPX_CUDA(cudaFuncSetAttribute(k_b_certificate, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)smem_bytes(1)));
    k_b_certificate<<<N, kThreads, smem_bytes(1), st>>>(pool, std::max(ep, eg), std::max(ed, eg),
                                                       d_cert.p);
    SDPX_LAUNCH_CHECK();
    ++launches;
    SDPX_CUDA(cudaMemcpyAsync(h_cert.p, d_cert.p, (size_t)N * kCertOut * sizeof(double),
                              cudaMemcpyDeviceToHost, st));
    SDPX_CUDA(cudaStreamSynchronize(st));
    const double* all = static_cast<const double*>(h_cert.p);
    // `_psd_violation` (src/validation.jl:919-932) of one block
    auto violation = [](const double* o, double bad) {
      if (o[2] != 0.0) return 0.0;
      if (bad != 0.0) return (double)INFINITY;
      const double excess = std::max(0.0, o[0] - o[1]);
      return std::max(excess, o[4] != 0.0 ? o[3] : o[1]);
    };
    for (int i = 0; i < N; ++i) {
      const double* o = all + (size_t)i * kCertOut;
      sdpx_b200_certificate_result& r = results[i];
      r = sdpx_b200_certificate_result{};
      r.primal_objective = o[cPobj];
      r.dual_objective = o[cDobj];
      r.gap = o[cPobj] - o[cDobj];
      const double oscale = std::max(1.0, (std::fabs(o[cPobj]) + std::fabs(o[cDobj])) / 2.0);
      r.gap_relative = std::fabs(r.gap) / oscale;
      r.primal_affine_residual = o[cPaff];
      r.dual_affine_residual = o[cDaff];
      r.primal_cone_violation = violation(o + cXsym, o[cBadX]);
      r.dual_cone_violation = violation(o + cYsym, o[cBadY]);
      r.primal_residual = std::max(o[cPaff], r.primal_cone_violation);
      r.dual_residual = std::max(o[cDaff], r.dual_cone_violation);
      r.primal_residual_scaled = r.primal_residual / scale_p[i];
      r.dual_residual_scaled = r.dual_residual / scale_d[i];
      r.primal_block_backward_error = o[cPbMixed];
      r.primal_block_strict_backward_error = o[cPbStrict];
      r.dual_backward_error = o[cDbMixed];
      r.dual_strict_backward_error = o[cDbStrict];
      r.complementarity = o[cCompl];
      r.complementarity_relative = std::fabs(o[cCompl]) / oscale;
      r.primal_psd_failing_blocks = o[cXok] != 0.0 ? 0 : 1;
      r.dual_psd_failing_blocks = o[cYok] != 0.0 ? 0 : 1;
      const bool primal_finite = std::isfinite(r.primal_objective) &&
                                 std::isfinite(r.primal_residual) && o[cBadX] == 0.0;
      const bool dual_finite = std::isfinite(r.dual_objective) && std::isfinite(r.dual_residual) &&
                               o[cBadY] == 0.0;
      const bool finite = primal_finite && dual_finite && std::isfinite(r.gap_relative) &&
                          std::isfinite(r.complementarity);
      const bool gap_ok = legacy ? (0.0 <= r.gap && r.gap <= eg) : (r.gap_relative <= eg);
      int f = 0;
      if (!finite) f |= SDPX_B200_CERT_NONFINITE;
      if (!(r.primal_residual_scaled <= ep)) f |= SDPX_B200_CERT_PRIMAL_RESIDUAL;
      if (!(r.primal_block_backward_error <= ep)) f |= SDPX_B200_CERT_PRIMAL_BLOCK_BACKWARD_ERROR;
      if (!(r.dual_residual_scaled <= ed)) f |= SDPX_B200_CERT_DUAL_RESIDUAL;
      if (!(r.dual_backward_error <= ed)) f |= SDPX_B200_CERT_DUAL_BACKWARD_ERROR;
      if (!gap_ok) f |= SDPX_B200_CERT_DUALITY_GAP;
      if (r.primal_psd_failing_blocks) f |= SDPX_B200_CERT_PRIMAL_PSD;
      if (r.dual_psd_failing_blocks) f |= SDPX_B200_CERT_DUAL_PSD;
      r.failures = f;
      r.valid = f == 0 ? 1 : 0;
    }
  }

  // Replaces instance i's current iterate (x, X, Y; NULL keeps a part).
  std::vector<char> has_solution;
  void set_solution(int i, const double* hx, const double* hX, const double* hY) {
    if (i < 0 || i >= N) throw std::invalid_argument("instance index out of range");
    const Inst& I = inst[i];
    const long long kk = (long long)I.k * I.k;
    SDPX_CUDA(cudaStreamSynchronize(st));
    if (hx)
      SDPX_CUDA(cudaMemcpyAsync(x.p + I.m_off, hx, I.m * sizeof(double), cudaMemcpyHostToDevice,
                                st));
    if (hX)
      SDPX_CUDA(cudaMemcpyAsync(X.p + I.kk_off, hX, kk * sizeof(double), cudaMemcpyHostToDevice,
                                st));
    if (hY)
      SDPX_CUDA(cudaMemcpyAsync(Y.p + I.kk_off, hY, kk * sizeof(double), cudaMemcpyHostToDevice,
                                st));
    SDPX_CUDA(cudaStreamSynchronize(st));
    if (has_solution.empty()) has_solution.assign(N, 0);
    if (hx && hX && hY) has_solution[i] = 1;
    bool all = true;
    for (char h : has_solution) all = all && h;
    if (all) solved = true;
  }

  // Host → device copy of one pooled array whose instance segments lie in
  // input order (segment i of len(i) doubles from src[i]): consecutive
  // instances are packed by a few host threads into one of two 64 MB pinned
  // staging buffers, each buffer goes out as one asynchronous copy, and the
  // other buffer is filled meanwhile — instead of one pageable copy per
  // instance and array.
  template <class Len>
  void upload_pooled(double* dst, const double* const* src, Len len) {
    size_t total = 0;
    for (int q = 0; q < N; ++q) total += (size_t)len(q);
    // doubles per staging buffer: 64 MB, or the whole array when smaller
    const size_t kStage = std::min<size_t>((size_t)8 << 20, total);
    Pinned& b0 = h_stage[0];
    Pinned& b1 = h_stage[1];
    b0.ensure(kStage * sizeof(double));
    b1.ensure(kStage * sizeof(double));
    const unsigned nthr = std::max(1u, std::min(8u, std::thread::hardware_concurrency()));
    long long doff = 0;
    int i = 0, which = 0;
    bool pending[2] = {false, false};
    while (i < N) {
      // instances [i, j) that fit one buffer (a single instance always fits:
      // at most 64²·256 doubles)
      int j = i;
      size_t fill = 0;
      std::vector<size_t> at;
      while (j < N && fill + (size_t)len(j) <= kStage) {
        at.push_back(fill);
        fill += (size_t)len(j);
        ++j;
      }
      if (j == i) throw std::logic_error("upload_pooled: segment larger than the staging buffer");
      if (pending[which]) SDPX_CUDA(cudaEventSynchronize(ev_stage[which]));
      double* buf = static_cast<double*>((which ? b1 : b0).p);
      auto pack = [&](unsigned t) {
        for (int q = i + (int)t; q < j; q += (int)nthr)
          std::memcpy(buf + at[q - i], src[q], (size_t)len(q) * sizeof(double));
      };
      std::vector<std::thread> pool;
      for (unsigned t = 1; t < nthr && (int)t < j - i; ++t) pool.emplace_back(pack, t);
      pack(0);
      for (auto& th : pool) th.join();
      SDPX_CUDA(cudaMemcpyAsync(dst + doff, buf, fill * sizeof(double), cudaMemcpyHostToDevice, st));
      SDPX_CUDA(cudaEventRecord(ev_stage[which], st));
      pending[which] = true;
      doff += (long long)fill;
      which ^= 1;
      i = j;
    }
    SDPX_CUDA(cudaStreamSynchronize(st));  // the staging buffers are reused by the next array
  }

  // Every instance's x, X and Y in one read-back: the pooled arrays are laid
  // out in input order (x_i at Σ_{j<i} m_j, X_i and Y_i at Σ_{j<i} k_j²).
  void get_solutions(double* hx, double* hX, double* hY) {
    long long mt = 0, kt = 0;
    for (const Inst& I : inst) {
      mt += I.m;
      kt += (long long)I.k * I.k;
    }
    if (hx) SDPX_CUDA(cudaMemcpyAsync(hx, x.p, mt * sizeof(double), cudaMemcpyDeviceToHost, st));
    if (hX) SDPX_CUDA(cudaMemcpyAsync(hX, X.p, kt * sizeof(double), cudaMemcpyDeviceToHost, st));
    if (hY) SDPX_CUDA(cudaMemcpyAsync(hY, Y.p, kt * sizeof(double), cudaMemcpyDeviceToHost, st));
    SDPX_CUDA(cudaStreamSynchronize(st));
  }

  void get_solution(int i, double* hx, double* hX, double* hY) {
    if (i < 0 || i >= N) throw std::invalid_argument("instance index out of range");
    const Inst& I = inst[i];
    const long long kk = (long long)I.k * I.k;
    if (hx)
      SDPX_CUDA(cudaMemcpyAsync(hx, x.p + I.m_off, I.m * sizeof(double), cudaMemcpyDeviceToHost,
                                st));
    if (hX)
      SDPX_CUDA(cudaMemcpyAsync(hX, X.p + I.kk_off, kk * sizeof(double), cudaMemcpyDeviceToHost,
                                st));
    if (hY)
      SDPX_CUDA(cudaMemcpyAsync(hY, Y.p + I.kk_off, kk * sizeof(double), cudaMemcpyDeviceToHost,
                                st));
    SDPX_CUDA(cudaStreamSynchronize(st));
  }
};

}  // namespace batch
}  // namespace sdpx

struct sdpx_b200_batch {
  sdpx::batch::Engine e;
};

namespace {
thread_local std::string g_batch_create_error;
}

#define BGUARD(bb, body)                     \
  do {                                       \
    if (!(bb)) return -1;                    \
    try {                                    \
      SDPX_CUDA(cudaSetDevice((bb)->e.dev)); \
      body;                                  \
      return 0;                              \
    } catch (const std::exception& ex) {     \
      (bb)->e.err = ex.what();               \
      return -2;                             \
    } catch (...) {                          \
      (bb)->e.err = "unknown error";         \
      return -3;                             \
    }                                        \
  } while (0)

extern "C" {

int sdpx_b200_batch_create(const sdpx_b200_batch_problem* problem, int device,
                           sdpx_b200_batch** out) {
  if (!out) return -1;
  *out = nullptr;
  auto* b = new (std::nothrow) sdpx_b200_batch();
  if (!b) {
    g_batch_create_error = "out of host memory";
    return -1;
  }
  try {
    b->e.create(problem, device);
  } catch (const std::exception& ex) {
    g_batch_create_error = ex.what();
    delete b;
    return -2;
  }
  *out = b;
  return 0;
}

void sdpx_b200_batch_destroy(sdpx_b200_batch* b) {
  if (!b) return;
  cudaSetDevice(b->e.dev);
  delete b;
}

const char* sdpx_b200_batch_last_error(const sdpx_b200_batch* b) {
  return b ? b->e.err.c_str() : "NULL batch";
}

const char* sdpx_b200_batch_create_error(void) { return g_batch_create_error.c_str(); }

int sdpx_b200_batch_optimize(sdpx_b200_batch* b, const sdpx_b200_solve_options* opts,
                             sdpx_b200_solve_result* results) {
  if (b && (!opts || !results)) {
    b->e.err = "NULL options or results";
    return -1;
  }
  BGUARD(b, b->e.optimize(*opts, results));
}

int sdpx_b200_batch_certificate(sdpx_b200_batch* b, double eps_primal, double eps_dual,
                                double eps_gap, int32_t legacy_gap,
                                sdpx_b200_certificate_result* results) {
  if (b && !results) {
    b->e.err = "NULL results";
    return -1;
  }
  BGUARD(b, b->e.certificate(eps_primal, eps_dual, eps_gap, legacy_gap, results));
}

int sdpx_b200_batch_set_solution(sdpx_b200_batch* b, int32_t i, const double* x,
                                 const double* X, const double* Y) {
  BGUARD(b, b->e.set_solution(i, x, X, Y));
}

int sdpx_b200_batch_get_solution(sdpx_b200_batch* b, int32_t i, double* x, double* X, double* Y) {
  BGUARD(b, b->e.get_solution(i, x, X, Y));
}

int sdpx_b200_batch_get_solutions(sdpx_b200_batch* b, double* x, double* X, double* Y) {
  BGUARD(b, b->e.get_solutions(x, X, Y));
}

int sdpx_b200_batch_stats(sdpx_b200_batch* b, double* out8) {
  BGUARD(b, {
    if (!out8) throw std::invalid_argument("NULL output");
    out8[0] = (double)b->e.passes;
    out8[1] = (double)b->e.launches;
    out8[2] = b->e.t_loop;
    out8[3] = b->e.t_schur;
    out8[4] = b->e.t_factor;
    out8[5] = b->e.t_step;
    out8[6] = (double)b->e.inst_iters;
    out8[7] = b->e.schur_flops;
  });
}

int sdpx_b200_batch_set_step_bounds(sdpx_b200_batch* b, int32_t mode) {
  BGUARD(b, {
    if (mode != 0 && mode != 1) throw std::invalid_argument("step-bound mode must be 0 or 1");
    b->e.bound_mode = mode;
  });
}

int sdpx_b200_batch_set_schur_shape(sdpx_b200_batch* b, int32_t threads, int32_t tile,
                                    double grain) {
  BGUARD(b, {
    if (threads != 0) {
      if (!(tile == 64 && threads == 128) && !sdpx::batch::syrk_kernel(threads, tile))
        throw std::invalid_argument("unsupported Schur launch shape (threads, tile)");
      b->e.schur_threads = threads;
      b->e.schur_tile = tile;
    }
    b->e.grain = grain;
  });
}

int sdpx_b200_batch_autotune(sdpx_b200_batch* b, const sdpx_b200_solve_options* opts,
                             double* table, int32_t capacity, int32_t* count) {
  if (b && !opts) {
    b->e.err = "NULL options";
    return -1;
  }
  BGUARD(b, {
    const int n = b->e.autotune(*opts, table, capacity);
    if (count) *count = n;
  });
}

}  // extern "C"
