// Reduced normal system of SDPX's LP standard form and of Lorentz cones
// (include/sdpx_b200_normal.h).
//
// Layout.  B (n × m_eq, column-major, one column per equality) stays resident;
// the scaled operand B̂ has the same layout, so Q = B̂ᵀB̂ is one lower SYRK of
// the FP64 tile engine with the variables as the contraction index:
//   rows [0, n_lp)         B̂ = D^{-1/2} B           (LP, src/lp_solver.jl:1892-1915)
//   rows of cone k         B̂ = W_k⁻¹ B_k            (Lorentz, W_k symmetric, so
//                                                    B̂_kᵀB̂_k = B_kᵀ Hs_k⁻¹ B_k)
// Using W⁻¹ rather than the signed form Hs⁻¹ = (2Jw(Jw)ᵀ − J)/η² keeps the
// contraction a plain positive Gram matrix (no cancellation between a
// rank-one and a diagonal term).
//
// This translation unit is compiled with FMA contraction off (--fmad=false):
// the per-cone kernels then evaluate the reference's scalar recurrences with
// exactly its roundings (IEEE division and square root are correctly rounded),
// so NT scaling points, λ, η, the NT maps and the LP pack are bit-identical to
// a sequential IEEE evaluation in the reference's order.
#include <cuda_runtime.h>

#include <array>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/sdpx_b200_normal.h"
#include "ipm_controller.h"
#include "blas_f64.h"
#include "chol.h"
#include "dbuf.h"
#include "schur_bf16.h"
#include "vec_kernels.h"

namespace sdpx {
namespace {

// ------------------------------------------------------------ NT scaling --
// `_soc_tail_norm` (src/soc_lorentz_kernels.jl:21-34).
__device__ double tail_norm(const double* v, int n) {
  double scale = 0.0;
  for (int i = 1; i < n; ++i) scale = fmax(scale, fabs(v[i]));
  if (scale == 0.0) return scale;
  double ss = 0.0;
  for (int i = 1; i < n; ++i) {
    double y = v[i] / scale;
    ss += y * y;
  }
  return scale * sqrt(ss);
}

// `_soc_sqrt_determinant` (src/soc_lorentz_kernels.jl:42-62).
__device__ bool sqrt_determinant(const double* v, int n, double* out) {
  double scale = 0.0;
  for (int i = 0; i < n; ++i) {
    if (!isfinite(v[i])) return false;
    scale = fmax(scale, fabs(v[i]));
  }
  if (scale == 0.0) return false;
  double head = v[0];
  double tail = tail_norm(v, n);
  double margin = head - tail;
  if (!(margin > 0.0)) return false;
  double residual = (margin / scale) * (head / scale + tail / scale);
  if (!(residual > 0.0)) return false;
  double r = scale * sqrt(residual);
  *out = r;
  return isfinite(r) && r > 0.0;
}

// `_soc_nt_scaling!` (src/soc_lorentz_kernels.jl:72-185), one thread per cone.
// The normalised points a = s/√det s, b = z/√det z and the midpoint raw are
// recomputed where the reference reads its temporaries (the same division
// gives the same value).  Outputs are written only after every check passed.
__global__ void k_nt_scaling(int ncones, const long long* __restrict__ off,
                             const int* __restrict__ dim, const double* __restrict__ s,
                             const double* __restrict__ z, double* w, double* lam, double* eta_out,
                             double* eta2_out, int* ok_out) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= ncones) return;
  const int n = dim[c];
  const double* sc = s + off[c];
  const double* zc = z + off[c];
  double* wc = w + off[c];
  double* lc = lam + off[c];
  ok_out[c] = 0;
  eta_out[c] = 0.0;
  eta2_out[c] = 0.0;
  double ss = 0.0, zs = 0.0;
  bool sok = sqrt_determinant(sc, n, &ss);
  bool zok = sqrt_determinant(zc, n, &zs);
  if (!(sok && zok)) return;
  double eta = sqrt(ss) / sqrt(zs);
  double eta2 = eta * eta;
  if (!(isfinite(eta2) && eta2 > 0.0)) return;
#define A_(i) (sc[i] / ss)
#define B_(i) (zc[i] / zs)
  for (int i = 0; i < n; ++i) {
    double a = A_(i), b = B_(i);
    double raw = (i == 0) ? a + b : a - b;
    if (!(isfinite(a) && isfinite(b) && isfinite(raw))) return;
  }
  double mscale = 1.0;
  for (int i = 0; i < n; ++i) mscale = fmax(mscale, fmax(fabs(A_(i)), fabs(B_(i))));
  double inv_m = 1.0 / mscale;
  double cross = (A_(0) * inv_m) * (B_(0) * inv_m);
  for (int i = 1; i < n; ++i) cross += (A_(i) * inv_m) * (B_(i) * inv_m);
  double radicand = inv_m * inv_m + cross;
  if (!(isfinite(radicand) && radicand > 0.0)) return;
  double wscale = sqrt(2.0) * mscale * sqrt(radicand);
  if (!(isfinite(wscale) && wscale > 0.0)) return;
  double nts = 1.0;
  for (int i = 1; i < n; ++i) nts = fmax(nts, fabs((A_(i) - B_(i)) / wscale));
  double inv_t = 1.0 / nts;
  double hacc = inv_t * inv_t;
  for (int i = 1; i < n; ++i) {
    double val = ((A_(i) - B_(i)) / wscale) / nts;
    hacc += val * val;
  }
  double nhead = nts * sqrt(hacc);
  if (!(isfinite(nhead) && nhead > 0.0)) return;
  double gamma = wscale / 2.0;
  double lscale = fmax(fmax(1.0, fabs(A_(0))), fmax(fabs(B_(0)), fabs(gamma)));
  for (int i = 1; i < n; ++i) lscale = fmax(lscale, fmax(fabs(A_(i)), fabs(B_(i))));
  double inv_l = 1.0 / lscale;
  double aa_h = A_(0) * inv_l, bb_h = B_(0) * inv_l, gg = gamma * inv_l;
  double den = aa_h + bb_h + 2.0 * gg;
  if (!(isfinite(den) && den > 0.0)) return;
  double geo = sqrt(ss) * sqrt(zs);
  double lam_head = geo * gamma;
  if (!isfinite(lam_head)) return;
  for (int pass = 0; pass < 2; ++pass) {  // pass 0 checks, pass 1 commits
    for (int i = 1; i < n; ++i) {
      double aa = A_(i) * inv_l, bb = B_(i) * inv_l;
      double scaled = (gg + bb_h) * aa + (gg + aa_h) * bb;
      double val = geo * (scaled / den) * lscale;
      if (pass == 0) {
        if (!isfinite(val)) return;
      } else {
        lc[i] = val;
        wc[i] = (A_(i) - B_(i)) / wscale;
      }
    }
  }
#undef A_
#undef B_
  wc[0] = nhead;
  lc[0] = lam_head;
  eta_out[c] = eta;
  eta2_out[c] = eta2;
  ok_out[c] = 1;
}

// ------------------------------------------------------------- NT maps ----
// `_soc_nt_apply_w!` / `_soc_nt_apply_winv!` / `_soc_nt_apply_hs_inverse!`
// (src/soc_lorentz_kernels.jl:187-255) on the contiguous segment v[0..n)
// (a cone vector, or a cone's rows of one column of B).  which = 2 may add
// the result to `base` (out = base + Hs⁻¹v); W and W⁻¹ ignore it.
__device__ __forceinline__ void nt_map(int which, const double* wc, double eta, double eta2,
                                       const double* v, double* out, int n, const double* base) {
  const double head = v[0];
  if (which == 2) {
    double ld = wc[0] * head;
    for (int i = 1; i < n; ++i) ld -= wc[i] * v[i];
    double o0 = (2.0 * wc[0] * ld - head) / eta2;
    out[0] = base ? base[0] + o0 : o0;
    for (int i = 1; i < n; ++i) {
      double oi = (-2.0 * wc[i] * ld + v[i]) / eta2;
      out[i] = base ? base[i] + oi : oi;
    }
    return;
  }
  double dt = 0.0;
  for (int i = 1; i < n; ++i) dt += wc[i] * v[i];
  if (which == 0) {
    double corr = head + dt / (1.0 + wc[0]);
    out[0] = eta * (wc[0] * head + dt);
    for (int i = 1; i < n; ++i) out[i] = eta * (v[i] + corr * wc[i]);
  } else {
    double corr = -head + dt / (1.0 + wc[0]);
    out[0] = (wc[0] * head - dt) / eta;
    for (int i = 1; i < n; ++i) out[i] = (v[i] + corr * wc[i]) / eta;
  }
}

__global__ void k_nt_apply(int which, int ncones, const long long* __restrict__ off,
                           const int* __restrict__ dim, const double* __restrict__ w,
                           const double* __restrict__ eta, const double* __restrict__ eta2,
                           const double* __restrict__ v, double* __restrict__ out) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= ncones) return;
  nt_map(which, w + off[c], eta[c], eta2[c], v + off[c], out + off[c], dim[c], nullptr);
}

// --------------------------------------------------------------- LP pack --
__global__ void k_lp_pack(int n_lp, const double* __restrict__ weights, const int* __restrict__ row,
                          const double* __restrict__ coef, double reg, double* D, double* Dinv,
                          double* Dis) {
  int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n_lp) return;
  double c = coef[j];
  double d = weights[row[j]] * c * c + reg;
  double inv = 1.0 / d;
  D[j] = d;
  Dinv[j] = inv;
  Dis[j] = sqrt(inv);
}

// B̂[j, e] = D^{-1/2}_j · B[j, e] for the LP rows of every column.
__global__ void k_scale_lp(int n_lp, long long n, int m, const double* __restrict__ B,
                           const double* __restrict__ Dis, double* __restrict__ Bh) {
  const long long tot = (long long)n_lp * m;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < tot;
       e += (long long)gridDim.x * blockDim.x) {
    long long col = e / n_lp;
    int j = (int)(e - col * n_lp);
    long long idx = col * n + j;
    Bh[idx] = Dis[j] * B[idx];
  }
}

// B̂_k[:, e] = W_k⁻¹ B_k[:, e]: one thread per (cone, column), the cone's
// segment of column e walked sequentially (the W⁻¹ map's order).  Adjacent
// threads take adjacent columns of the same cone.
__global__ void k_scale_cones(int ncones, int m, long long n, long long cone_base,
                              const long long* __restrict__ off, const int* __restrict__ dim,
                              const double* __restrict__ w, const double* __restrict__ eta,
                              const double* __restrict__ B, double* __restrict__ Bh) {
  long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= (long long)ncones * m) return;
  int c = (int)(t / m);
  long long col = t - (long long)c * m;
  long long base = col * n + cone_base + off[c];
  nt_map(1, w + off[c], eta[c], 0.0, B + base, Bh + base, dim[c], nullptr);
}

// Q_ii += δ (Q holds the lower triangle from the SYRK); F = lower(Q), upper 0.
__global__ void k_shift_copy_lower(int m, double* Q, double reg, double* F) {
  const long long tot = (long long)m * m;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < tot;
       e += (long long)gridDim.x * blockDim.x) {
    int i = (int)(e % m), j = (int)(e / m);
    double v = 0.0;
    if (i > j) v = Q[e];
    if (i == j) {
      v = Q[e] + reg;
      Q[e] = v;
    }
    F[e] = v;
  }
}

// out = base + D⁻¹ v over all variables: LP entries by D⁻¹_j, cone k by Hs_k⁻¹
// (thread per LP entry, then one thread per cone).
__global__ void k_apply_dinv(int n_lp, const double* __restrict__ Dinv, int ncones,
                             long long cone_base, const long long* __restrict__ off,
                             const int* __restrict__ dim, const double* __restrict__ w,
                             const double* __restrict__ eta2, const double* __restrict__ v,
                             const double* __restrict__ base, double* __restrict__ out) {
  long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t < n_lp) {
    double o = Dinv[t] * v[t];
    out[t] = base ? base[t] + o : o;
    return;
  }
  long long c = t - n_lp;
  if (c >= ncones) return;
  long long o = cone_base + off[c];
  nt_map(2, w + off[c], 0.0, eta2[c], v + o, out + o, dim[c], base ? base + o : nullptr);
}

}  // namespace

// ============================================================================
struct NormalHandle {
  int dev = 0;
  cudaStream_t st = nullptr;
  int sms = 148;
  std::string err;
  int n_lp = 0, ncones = 0, m = 0, n_weights = 0;
  long long n = 0, nq = 0;  // variables, cone variables
  std::vector<long long> cone_off;
  std::vector<int> cone_dim;
  DBuf<long long> d_off;
  DBuf<int> d_dim, d_row, d_ok, d_info;
  DBuf<unsigned> coop_bar;  // grid-barrier state of the single-launch Cholesky
  DBuf<double> B, Bh, coef, weights, D, Dinv, Dis, w, lam, eta, eta2, s, z, v, out;
  DBuf<double> Q, F, Finv_diag, partial, rhs, t, red, work, u, gemv_part;
  DBuf<double> dmin, dmax;
  DBuf<MatDesc<double>> descs;
  SyrkPlan plan;
  int gemv_chunks = 8;
  bool have_scaling = false, have_factor = false, have_assembled = false;
  bool standard_rows = true;  // row_for_variable = identity, g = 1, one weight per LP variable
  // Split-BF16 assembly: three BF16 planes of B̂ (m rows of pitch Kp = n
  // rounded up to 64) and the tcgen05 SYRK of the Schur path.
  long long Kp = 0;
  DBuf<unsigned char> plane_buf[3];
  SplitSyrkPlan splan;
  DBuf<float> spartial;
  DBuf<int> serr;
  // Explicit inverse of the reduced factor for the refined (mixed) solves:
  // each solve is two GEMVs over L⁻¹ instead of 2·⌈m/64⌉ dependent launches.
  DBuf<double> Linv, Ltmp, Ldinv;
  bool have_inverse = false;
  void make_inverse() {
    if (Linv.n < (size_t)m * m) {
      Linv.alloc((size_t)m * m);
      Ltmp.alloc((size_t)m * m);
      Ldinv.alloc((size_t)ceil_div(std::max(m, 1), 64) * 64 * 64);
    }
    trinv_recursive_f64(F.p, m, Linv.p, Ldinv.p, Ltmp.p, st);
    have_inverse = true;
  }
  // v ← Q⁻¹v = L⁻ᵀ(L⁻¹v) with the explicit inverse (work: m).
  void solve_inverse(double* v) {
    gemv_n(Linv.p, m, m, v, work.p, gemv_part.p, gemv_chunks, st);
    gemv_t(Linv.p, m, m, work.p, 1.0, nullptr, 0.0, v, st);
  }
  cudaEvent_t ev[4] = {};
  double assemble_ms = 0.0, factor_ms = 0.0;

  void create(int n_lp_, int ncones_, const int* dims, int m_, const double* hB, const int* row,
              const double* hcoef, int n_weights_, int device) {
    if (n_lp_ < 0 || ncones_ < 0 || m_ < 0 || n_weights_ < 0)
      throw std::invalid_argument("negative size");
    if (ncones_ > 0 && !dims) throw std::invalid_argument("cone_dims is NULL");
    if (n_lp_ > 0 && (!row || !hcoef || n_weights_ <= 0))
      throw std::invalid_argument("LP variables need row_for_variable, diagonal_coefficient, weights");
    dev = device;
    SDPX_CUDA(cudaSetDevice(dev));
    SDPX_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    SDPX_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    for (auto& e : ev) SDPX_CUDA(cudaEventCreate(&e));
    n_lp = n_lp_;
    ncones = ncones_;
    m = m_;
    n_weights = n_weights_;
    long long o = 0;
    for (int c = 0; c < ncones; ++c) {
      if (dims[c] < 1) throw std::invalid_argument("cone dimension must be >= 1");
      cone_off.push_back(o);
      cone_dim.push_back(dims[c]);
      o += dims[c];
    }
    nq = o;
    n = n_lp + nq;
    for (int j = 0; j < n_lp; ++j)
      if (row[j] < 0 || row[j] >= n_weights)
        throw std::invalid_argument("row_for_variable out of range at variable " + std::to_string(j));
    standard_rows = n_weights == n_lp;
    for (int j = 0; j < n_lp && standard_rows; ++j) standard_rows = row[j] == j && hcoef[j] == 1.0;
    if (n > 0 && m > 0 && !hB) throw std::invalid_argument("B is NULL");
    B.alloc((size_t)n * m);
    Bh.alloc((size_t)n * m);
    if (n > 0 && m > 0) h2d(B.p, hB, sizeof(double) * n * m);
    d_off.alloc(ncones);
    d_dim.alloc(ncones);
    if (ncones) {
      h2d(d_off.p, cone_off.data(), sizeof(long long) * ncones);
      h2d(d_dim.p, cone_dim.data(), sizeof(int) * ncones);
    }
    d_row.alloc(n_lp);
    coef.alloc(n_lp);
    if (n_lp) {
      h2d(d_row.p, row, sizeof(int) * n_lp);
      h2d(coef.p, hcoef, sizeof(double) * n_lp);
    }
    weights.alloc(n_weights);
    for (auto* b : {&D, &Dinv, &Dis}) b->alloc(n_lp);
    for (auto* b : {&w, &lam, &s, &z, &v, &out}) b->alloc(nq);
    for (auto* b : {&eta, &eta2}) b->alloc(ncones);
    d_ok.alloc(ncones);
    Q.alloc((size_t)m * m);
    F.alloc((size_t)m * m);
    Finv_diag.alloc((size_t)ceil_div(std::max(m, 1), 64) * 64 * 64);
    rhs.alloc(n + m);
    t.alloc(n);
    u.alloc(n);
    red.alloc(m);
    work.alloc(m);
    gemv_chunks = std::max(1, std::min(16, m / 64));
    gemv_part.alloc((size_t)gemv_chunks * std::max<long long>(n, m));
    plan = plan_syrk_f64(std::max(m, 1), std::max<long long>(n, 1), sms);
    partial.alloc(plan.partial_doubles);
    d_info.alloc(1);
    dmin.alloc(1);
    dmax.alloc(1);
    descs.alloc(1);
    sync();
  }
  ~NormalHandle() {
    if (st) {
      cudaSetDevice(dev);
      cudaStreamSynchronize(st);
      for (auto& e : ev)
        if (e) cudaEventDestroy(e);
      cudaStreamDestroy(st);
    }
  }

  void h2d(void* d, const void* h, size_t bytes) {
    if (bytes) SDPX_CUDA(cudaMemcpyAsync(d, h, bytes, cudaMemcpyHostToDevice, st));
  }
  void d2h(void* h, const void* d, size_t bytes) {
    if (bytes) SDPX_CUDA(cudaMemcpyAsync(h, d, bytes, cudaMemcpyDeviceToHost, st));
  }
  void sync() { SDPX_CUDA(cudaStreamSynchronize(st)); }

  int nt_scaling(const double* hs, const double* hz, int* ok, double* hw, double* hlam,
                 double* heta, double* heta2) {
    have_scaling = false;
    if (ncones == 0) return 0;
    if (!hs || !hz) throw std::invalid_argument("s and z are required");
    h2d(s.p, hs, sizeof(double) * nq);
    h2d(z.p, hz, sizeof(double) * nq);
    k_nt_scaling<<<ceil_div(ncones, 128), 128, 0, st>>>(ncones, d_off.p, d_dim.p, s.p, z.p, w.p,
                                                         lam.p, eta.p, eta2.p, d_ok.p);
    SDPX_LAUNCH_CHECK();
    std::vector<int> okv(ncones);
    d2h(okv.data(), d_ok.p, sizeof(int) * ncones);
    if (hw) d2h(hw, w.p, sizeof(double) * nq);
    if (hlam) d2h(hlam, lam.p, sizeof(double) * nq);
    if (heta) d2h(heta, eta.p, sizeof(double) * ncones);
    if (heta2) d2h(heta2, eta2.p, sizeof(double) * ncones);
    sync();
    int bad = 0;
    for (int c = 0; c < ncones; ++c) {
      if (ok) ok[c] = okv[c];
      bad += okv[c] == 0;
    }
    have_scaling = bad == 0;
    have_factor = false;
    return bad ? 1 : 0;
  }

  void require_scaling() {
    if (ncones > 0 && !have_scaling)
      throw std::logic_error("no valid NT scaling held: call nt_scaling with interior points first");
  }

  void nt_apply(int which, const double* hv, double* hout) {
    if (which < 0 || which > 2) throw std::invalid_argument("which must be 0 (W), 1 (W^-1) or 2 (Hs^-1)");
    require_scaling();
    if (ncones == 0) return;
    h2d(v.p, hv, sizeof(double) * nq);
    k_nt_apply<<<ceil_div(ncones, 128), 128, 0, st>>>(which, ncones, d_off.p, d_dim.p, w.p, eta.p,
                                                       eta2.p, v.p, out.p);
    SDPX_LAUNCH_CHECK();
    d2h(hout, out.p, sizeof(double) * nq);
    sync();
  }

  void pack(const double* hweights, double reg) {
    if (n_lp == 0) return;
    if (!hweights) throw std::invalid_argument("weights is NULL");
    h2d(weights.p, hweights, sizeof(double) * n_weights);
    k_lp_pack<<<ceil_div(n_lp, 256), 256, 0, st>>>(n_lp, weights.p, d_row.p, coef.p, reg, D.p,
                                                    Dinv.p, Dis.p);
    SDPX_LAUNCH_CHECK();
  }

  // B̂ rows of the cones (independent of δ) — once per scaling.
  void scale_cones() {
    if (ncones == 0 || m == 0) return;
    long long threads = (long long)ncones * m;
    k_scale_cones<<<ceil_div(threads, 128), 128, 0, st>>>(ncones, m, n, n_lp, d_off.p, d_dim.p,
                                                          w.p, eta.p, B.p, Bh.p);
    SDPX_LAUNCH_CHECK();
  }

  // Q = B̂ᵀB̂ from three BF16 planes of B̂ on the tcgen05 split SYRK (FP32
  // tiles summed in FP64; ≈ 1e-6 relative), +δ and the lower copy into F.
  void assemble_split(double reg) {
    if (m == 0) return;
    scale_lp_rows();
    if (Kp == 0) {
      Kp = (std::max<long long>(n, 1) + 63) / 64 * 64;
      for (auto& b : plane_buf) b.alloc(sizeof(__nv_bfloat16) * (size_t)m * Kp);
      splan = plan_split_syrk(m, Kp, sms);
      spartial.alloc(splan.partial_floats);
      serr.alloc(1);
    }
    __nv_bfloat16* pl[3];
    for (int i = 0; i < 3; ++i) pl[i] = reinterpret_cast<__nv_bfloat16*>(plane_buf[i].p);
    split_rows_f64(Bh.p, n, m, n, Kp, pl, st);
    SDPX_CUDA(cudaMemsetAsync(serr.p, 0, sizeof(int), st));
    Plane2D P{{pl[0], pl[1], pl[2]}, m, Kp};
    split_syrk(P, m, (int)Kp, splan, spartial.p, Q.p, serr.p, st);
    int e = 0;
    d2h(&e, serr.p, sizeof(int));
    sync();
    if (e) throw CudaError("split normal-matrix SYRK: a bounded wait gave up");
    long long tot = (long long)m * m;
    k_shift_copy_lower<<<(int)std::min<long long>(ceil_div(tot, 256), (long long)sms * 16), 256, 0,
                         st>>>(m, Q.p, reg, F.p);
    SDPX_LAUNCH_CHECK();
    have_assembled = true;
  }

  // B̂ = D^{-1/2}B on the LP rows (the cone rows come from scale_cones).
  void scale_lp_rows() {
    if (n_lp > 0 && m > 0) {
      long long tot = (long long)n_lp * m;
      int grid = (int)std::min<long long>(ceil_div(tot, 256), (long long)sms * 16);
      k_scale_lp<<<grid, 256, 0, st>>>(n_lp, n, m, B.p, Dis.p, Bh.p);
      SDPX_LAUNCH_CHECK();
    }
  }

  // LP rows of B̂, SYRK, +δ on the diagonal, copy of lower(Q) into F.
  void assemble_lp_and_syrk(double reg) {
    if (m == 0) return;
    scale_lp_rows();
    if (n > 0) {
      Opnd P;
      P.base = Bh.p;
      P.kstride = 1;
      P.inner = 1 << 30;
      P.inner_stride = n;
      P.outer_stride = 0;
      P.mn_extent = m;
      P.k_extent = (int)n;
      syrk_lower_f64(P, plan, partial.p, Q.p, m, m, 0.0, st);
    } else {
      SDPX_CUDA(cudaMemsetAsync(Q.p, 0, sizeof(double) * (size_t)m * m, st));
    }
    long long tot = (long long)m * m;
    k_shift_copy_lower<<<(int)std::min<long long>(ceil_div(tot, 256), (long long)sms * 16), 256, 0,
                         st>>>(m, Q.p, reg, F.p);
    SDPX_LAUNCH_CHECK();
    have_assembled = true;
  }

  void assemble(const double* hweights, double reg) {
    require_scaling();
    have_factor = false;
    SDPX_CUDA(cudaEventRecord(ev[0], st));
    pack(hweights, reg);
    scale_cones();
    assemble_lp_and_syrk(reg);
    SDPX_CUDA(cudaEventRecord(ev[1], st));
    sync();
    float ms = 0.f;
    SDPX_CUDA(cudaEventElapsedTime(&ms, ev[0], ev[1]));
    assemble_ms = ms;
  }

  // Returns 0 on success, 1 when every attempt failed.
  int factorize(const double* hweights, double reg, int max_attempts, int* attempts,
                double* reg_used) {
    if (max_attempts < 1) throw std::invalid_argument("max_attempts must be >= 1");
    require_scaling();
    have_factor = false;
    double r = reg;
    int info = 1;
    int att = 0;
    float asm_ms = 0.f, fac_ms = 0.f;
    for (att = 1; att <= max_attempts; ++att) {
      SDPX_CUDA(cudaEventRecord(ev[0], st));
      pack(hweights, r);
      if (att == 1) scale_cones();
      assemble_lp_and_syrk(r);
      SDPX_CUDA(cudaEventRecord(ev[1], st));
      if (m == 0) {
        info = 0;
        break;
      }
      factor_F();
      SDPX_CUDA(cudaEventRecord(ev[2], st));
      d2h(&info, d_info.p, sizeof(int));
      sync();
      if (info < 0) throw CudaError("normal-matrix Cholesky: a grid barrier timed out");
      float a = 0.f, f = 0.f;
      SDPX_CUDA(cudaEventElapsedTime(&a, ev[0], ev[1]));
      SDPX_CUDA(cudaEventElapsedTime(&f, ev[1], ev[2]));
      asm_ms += a;
      fac_ms += f;
      if (info == 0 || att == max_attempts) break;
      r *= 10.0;
    }
    if (attempts) *attempts = att;
    if (reg_used) *reg_used = r;
    assemble_ms = asm_ms;
    factor_ms = fac_ms;
    if (info != 0) return 1;
    if (m > 0) factor_diag_inverses<double, 64>(F.p, m, m, Finv_diag.p, st);
    sync();
    have_factor = true;
    return 0;
  }

  // Cholesky of the reduced matrix F in place: one cooperative launch above the
  // whole-panel size, the batched panels below it (identical factors).
  void factor_F() {
    if (potrf_single_pays<double, 64>(m)) {
      if (coop_bar.n < 4) coop_bar.alloc(4);
      potrf_single<double, 64>(F.p, m, m, d_info.p, dmin.p, dmax.p,
                               reinterpret_cast<CoopBar*>(coop_bar.p), true, st);
      return;
    }
    MatDesc<double> md{F.p, m, m};
    h2d(descs.p, &md, sizeof(md));
    potrf_batched<double, 64>(descs.p, 1, m, d_info.p, dmin.p, dmax.p, st);
  }

  // One assembly + Cholesky attempt with LP weights already on the device
  // (one weight per LP variable): 0 on success, 1 when the factor failed.
  int factorize_dev(const double* dweights, double reg, bool split = false) {
    require_scaling();
    have_factor = false;
    have_inverse = false;
    if (n_lp) {
      k_lp_pack<<<ceil_div(n_lp, 256), 256, 0, st>>>(n_lp, dweights, d_row.p, coef.p, reg, D.p,
                                                      Dinv.p, Dis.p);
      SDPX_LAUNCH_CHECK();
    }
    scale_cones();
    if (split) assemble_split(reg);
    else assemble_lp_and_syrk(reg);
    if (m == 0) {
      have_factor = true;
      return 0;
    }
    factor_F();
    int info = 1;
    d2h(&info, d_info.p, sizeof(int));
    sync();
    if (info < 0) throw CudaError("normal-matrix Cholesky: a grid barrier timed out");
    if (info != 0) return 1;
    factor_diag_inverses<double, 64>(F.p, m, m, Finv_diag.p, st);
    if (split) make_inverse();
    have_factor = true;
    return 0;
  }

  void get_matrix(int which, double* hout) {
    if (which == 0) {
      if (!have_assembled) throw std::logic_error("no assembled matrix");
      if (m > 0) mirror_lower(m, Q.p, st);
      d2h(hout, Q.p, sizeof(double) * (size_t)m * m);
    } else {
      if (!have_factor) throw std::logic_error("no successful factor held");
      d2h(hout, F.p, sizeof(double) * (size_t)m * m);
    }
    sync();
  }

  // Device-resident solve on rhs (n + m) already in `rhs`.
  void solve_device() {
    const long long nthreads = n_lp + ncones;
    const int grid = std::max(1, ceil_div(nthreads, 128));
    // t = D⁻¹ rx
    if (n > 0) {
      k_apply_dinv<<<grid, 128, 0, st>>>(n_lp, Dinv.p, ncones, n_lp, d_off.p, d_dim.p, w.p, eta2.p,
                                         rhs.p, nullptr, t.p);
      SDPX_LAUNCH_CHECK();
    }
    if (m == 0) {
      if (n > 0) SDPX_CUDA(cudaMemcpyAsync(rhs.p, t.p, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
      return;
    }
    double* dy = rhs.p + n;
    // dy ← ry − Bᵀt, then Q⁻¹
    if (n > 0) gemv_t(B.p, n, m, t.p, -1.0, dy, 1.0, dy, st);
    cholesky_solve<double, 64>(F.p, m, m, Finv_diag.p, dy, work.p, st);
    if (n == 0) return;
    // dx = t + D⁻¹(B dy)
    gemv_n(B.p, n, m, dy, u.p, gemv_part.p, gemv_chunks, st);
    k_apply_dinv<<<grid, 128, 0, st>>>(n_lp, Dinv.p, ncones, n_lp, d_off.p, d_dim.p, w.p, eta2.p,
                                       u.p, t.p, rhs.p);
    SDPX_LAUNCH_CHECK();
  }

  int solve(double* hrhs) {
    if (!have_factor) return 1;
    h2d(rhs.p, hrhs, sizeof(double) * (n + m));
    solve_device();
    d2h(hrhs, rhs.p, sizeof(double) * (n + m));
    sync();
    return 0;
  }
};

}  // namespace sdpx

#include "cone_ipm.inc"

// ============================================================================
//                                   C ABI
// ============================================================================
struct sdpx_b200_normal {
  sdpx::NormalHandle h;
};

static thread_local std::string g_normal_create_error;

#define NGUARD(hh, body)                      \
  do {                                        \
    if (!(hh)) return -1;                     \
    try {                                     \
      SDPX_CUDA(cudaSetDevice((hh)->h.dev));  \
      body;                                   \
      return 0;                               \
    } catch (const std::exception& ex) {      \
      (hh)->h.err = ex.what();                \
      return -2;                              \
    } catch (...) {                           \
      (hh)->h.err = "unknown error";          \
      return -3;                              \
    }                                         \
  } while (0)

extern "C" {

int sdpx_b200_normal_create(int32_t n_lp, int32_t n_cones, const int32_t* cone_dims, int32_t m_eq,
                            const double* B, const int32_t* row_for_variable,
                            const double* diagonal_coefficient, int32_t n_weights, int device,
                            sdpx_b200_normal** out) {
  if (!out) return -1;
  *out = nullptr;
  auto* hh = new (std::nothrow) sdpx_b200_normal();
  if (!hh) return -4;
  try {
    hh->h.create(n_lp, n_cones, cone_dims, m_eq, B, row_for_variable, diagonal_coefficient,
                 n_weights, device);
  } catch (const std::exception& ex) {
    g_normal_create_error = ex.what();
    delete hh;
    return -2;
  }
  *out = hh;
  return 0;
}
void sdpx_b200_normal_destroy(sdpx_b200_normal* h) { delete h; }
const char* sdpx_b200_normal_last_error(const sdpx_b200_normal* h) {
  return h ? h->h.err.c_str() : "null handle";
}
const char* sdpx_b200_normal_create_error(void) { return g_normal_create_error.c_str(); }

int sdpx_b200_normal_nt_scaling(sdpx_b200_normal* h, const double* s, const double* z, int32_t* ok,
                                double* w, double* lambda, double* eta, double* eta_squared) {
  NGUARD(h, return h->h.nt_scaling(s, z, ok, w, lambda, eta, eta_squared));
}
int sdpx_b200_normal_nt_apply(sdpx_b200_normal* h, int32_t which, const double* v, double* out) {
  NGUARD(h, {
    h->h.nt_apply(which, v, out);
    return 0;
  });
}
int sdpx_b200_normal_pack(sdpx_b200_normal* h, const double* weights, double regularization,
                          double* D, double* inverse_diagonal, double* inverse_sqrt) {
  NGUARD(h, {
    auto& H = h->h;
    H.pack(weights, regularization);
    if (D) H.d2h(D, H.D.p, sizeof(double) * H.n_lp);
    if (inverse_diagonal) H.d2h(inverse_diagonal, H.Dinv.p, sizeof(double) * H.n_lp);
    if (inverse_sqrt) H.d2h(inverse_sqrt, H.Dis.p, sizeof(double) * H.n_lp);
    H.sync();
    return 0;
  });
}
int sdpx_b200_normal_assemble(sdpx_b200_normal* h, const double* weights, double regularization) {
  NGUARD(h, {
    h->h.assemble(weights, regularization);
    return 0;
  });
}
int sdpx_b200_normal_factorize(sdpx_b200_normal* h, const double* weights, double regularization,
                               int32_t max_attempts, int32_t* attempts,
                               double* regularization_used) {
  NGUARD(h, {
    int att = 0;
    int rc = h->h.factorize(weights, regularization, max_attempts, &att, regularization_used);
    if (attempts) *attempts = att;
    if (rc) h->h.err = "reduced normal matrix not positive definite after regularization retries";
    return rc;
  });
}
int sdpx_b200_normal_get_matrix(sdpx_b200_normal* h, int32_t which, double* out) {
  NGUARD(h, {
    if (!out) throw std::invalid_argument("out is NULL");
    h->h.get_matrix(which, out);
    return 0;
  });
}
int sdpx_b200_normal_solve(sdpx_b200_normal* h, double* rhs) {
  NGUARD(h, {
    if (!rhs) throw std::invalid_argument("rhs is NULL");
    int rc = h->h.solve(rhs);
    if (rc) h->h.err = "no successful factor held (factorize failed or was not called)";
    return rc;
  });
}
int sdpx_b200_normal_optimize(sdpx_b200_normal* h, const double* b, const double* c,
                              const sdpx_b200_solve_options* opts, sdpx_b200_solve_result* result,
                              double* x, double* y, double* z) {
  if (!h) return -1;
  try {
    SDPX_CUDA(cudaSetDevice(h->h.dev));
    if (!opts || !c || (h->h.m > 0 && !b)) throw std::invalid_argument("NULL b, c or options");
    if (!h->h.standard_rows)
      throw std::invalid_argument("the LP part must be standard form (identity rows, g = 1)");
    sdpx::ConeIPM ipm(h->h);
    ipm.run(b, c, *opts, result, x, y, z);
    return 0;
  } catch (const std::exception& ex) {
    h->h.err = ex.what();
    return -2;
  }
}
int sdpx_b200_normal_times(sdpx_b200_normal* h, double* assemble_ms, double* factor_ms) {
  NGUARD(h, {
    if (assemble_ms) *assemble_ms = h->h.assemble_ms;
    if (factor_ms) *factor_ms = h->h.factor_ms;
    return 0;
  });
}
int sdpx_b200_normal_get_stream(sdpx_b200_normal* h, void** stream) {
  NGUARD(h, {
    if (!stream) throw std::invalid_argument("stream is NULL");
    *stream = (void*)h->h.st;
    return 0;
  });
}

}  // extern "C"
