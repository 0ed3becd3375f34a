// Equality block of the KKT system: kernels behind equality.h.
//
// The algorithm is SDPX's dense route for n > 0 equality rows
// (src/kkt.jl:1466-1680 factor, :2570-2595 solve): B̃ = L_S⁻¹B with each
// column scaled to unit ∞-norm (`_normalize_equality_panel_columns!`,
// src/kkt.jl:281-304), Q = B̃ᵀB̃ by Cholesky with a diagonal rank test, and the
// column-pivoted QR of B̃ (`la_qr_factor!(…; pivoted=true)`,
// src/la_backend.jl:823-850, rank by `_equality_qr_factor_handle`,
// src/la_backend.jl:956-1024) when that test fails.  The GEMM and SYRK of the
// block run on the FP64 tile kernels; what lives here is the column-wise and
// the inherently sequential small work.
#include <algorithm>

#include "common.cuh"
#include "equality.h"

namespace sdpx {

namespace {

__global__ void k_eq_normalize(int m, double* __restrict__ Bt, double* __restrict__ scale) {
  __shared__ double red[32];
  const int j = blockIdx.x;
  double* col = Bt + (long long)j * m;
  double v = 0.0;
  for (int i = threadIdx.x; i < m; i += blockDim.x) v = fmax(v, fabs(col[i]));
  v = block_max(v, red);
  double s = (v == 0.0) ? 1.0 : 1.0 / v;
  if (!isfinite(s)) s = 1.0;
  if (threadIdx.x == 0) scale[j] = s;
  if (s != 1.0)
    for (int i = threadIdx.x; i < m; i += blockDim.x) col[i] *= s;
}

// 64-bit mixing of (value bits, row): splitmix64 finaliser.
__device__ __forceinline__ unsigned long long mix64(unsigned long long z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

__global__ void k_eq_fingerprint(int m, const double* __restrict__ Bt,
                                 unsigned long long* __restrict__ fp) {
  __shared__ unsigned long long red[32];
  const int j = blockIdx.x;
  const double* col = Bt + (long long)j * m;
  unsigned long long h = 0;
  for (int i = threadIdx.x; i < m; i += blockDim.x) {
    double v = col[i];
    if (v == 0.0) v = 0.0;  // −0 and +0 fingerprint alike
    h += mix64((unsigned long long)__double_as_longlong(v) ^ mix64((unsigned long long)i));
  }
  for (int o = 16; o > 0; o >>= 1) h += __shfl_xor_sync(0xffffffffu, h, o);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane == 0) red[w] = h;
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned long long t = 0;
    for (int q = 0; q < (int)(blockDim.x >> 5); ++q) t += red[q];
    fp[j] = t;
  }
}

__global__ void k_eq_cols_equal(int m, const double* __restrict__ Bt, const int* __restrict__ pairs,
                                int* __restrict__ equal) {
  __shared__ int diff;
  if (threadIdx.x == 0) diff = 0;
  __syncthreads();
  const double* a = Bt + (long long)pairs[2 * blockIdx.x] * m;
  const double* b = Bt + (long long)pairs[2 * blockIdx.x + 1] * m;
  int d = 0;
  for (int i = threadIdx.x; i < m; i += blockDim.x) d |= !(a[i] == b[i]);
  if (d) atomicOr(&diff, 1);
  __syncthreads();
  if (threadIdx.x == 0) equal[blockIdx.x] = diff ? 0 : 1;
}

constexpr int QR_THREADS = 1024;
constexpr int QR_WARPS = QR_THREADS / 32;

// One CTA.  Step j: squared norms of the trailing columns over rows j..m−1
// (a warp per column, fixed-order lane sums), the first largest becomes the
// pivot, the pivot column is swapped in, its Householder reflector
// (β = −sign(α)·hypot(α, ‖x‖), τ = (β − α)/β, v = x/(α − β), as LAPACK's
// dlarfg) overwrites it, and every trailing column c receives
// A[j:, c] −= τ·v·(vᵀA[j:, c]) (a warp per column).
__global__ void __launch_bounds__(QR_THREADS) k_eq_qr(int m, int n, double* __restrict__ A, int lda,
                                                      int* __restrict__ perm,
                                                      double* __restrict__ rdiag,
                                                      double* __restrict__ colnorm) {
  __shared__ double red[32];
  __shared__ int s_piv;
  __shared__ double s_tau;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int j = threadIdx.x; j < n; j += blockDim.x) perm[j] = j;
  __syncthreads();
  const int steps = min(m, n);
  for (int j = 0; j < steps; ++j) {
    for (int c = j + warp; c < n; c += QR_WARPS) {
      const double* col = A + (long long)c * lda;
      double s = 0.0;
      for (int i = j + lane; i < m; i += 32) s += col[i] * col[i];
      s = warp_sum(s);
      if (lane == 0) colnorm[c] = s;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      int p = j;
      double best = colnorm[j];
      for (int c = j + 1; c < n; ++c)
        if (colnorm[c] > best) best = colnorm[c], p = c;
      s_piv = p;
    }
    __syncthreads();
    const int p = s_piv;
    if (p != j) {
      double* cj = A + (long long)j * lda;
      double* cp = A + (long long)p * lda;
      for (int i = threadIdx.x; i < m; i += blockDim.x) {
        const double t = cj[i];
        cj[i] = cp[i];
        cp[i] = t;
      }
      if (threadIdx.x == 0) {
        const int t = perm[j];
        perm[j] = perm[p];
        perm[p] = t;
      }
    }
    __syncthreads();
    double* cj = A + (long long)j * lda;
    double xs = 0.0;
    for (int i = j + 1 + threadIdx.x; i < m; i += blockDim.x) xs += cj[i] * cj[i];
    xs = block_sum(xs, red);
    const double alpha = cj[j];
    const double xnorm = sqrt(xs);
    double beta = alpha, tau = 0.0, scal = 1.0;
    if (xnorm != 0.0) {
      beta = -copysign(hypot(alpha, xnorm), alpha);
      tau = (beta - alpha) / beta;
      scal = 1.0 / (alpha - beta);
    }
    __syncthreads();
    for (int i = j + 1 + threadIdx.x; i < m; i += blockDim.x) cj[i] *= scal;
    if (threadIdx.x == 0) {
      cj[j] = beta;
      rdiag[j] = beta;
      s_tau = tau;
    }
    __syncthreads();
    tau = s_tau;
    if (tau != 0.0) {
      for (int c = j + 1 + warp; c < n; c += QR_WARPS) {
        double* col = A + (long long)c * lda;
        double w = 0.0;
        for (int i = j + 1 + lane; i < m; i += 32) w += cj[i] * col[i];
        w = warp_sum(w);
        if (lane == 0) w += col[j];
        w = __shfl_sync(0xffffffffu, w, 0);
        const double tw = tau * w;
        if (lane == 0) col[j] -= tw;
        for (int i = j + 1 + lane; i < m; i += 32) col[i] -= tw * cj[i];
      }
    }
    __syncthreads();
  }
}

// M(r, c) of the lower-triangular solve operator.
__device__ __forceinline__ double tri_at(const double* T, int ldt, int upper, int r, int c) {
  return upper ? T[c + (long long)r * ldt] : T[r + (long long)c * ldt];
}

__global__ void k_eq_small_solve(int n, int rank, const double* __restrict__ T, int ldt, int upper,
                                 const int* __restrict__ perm, const double* __restrict__ rhs,
                                 double* __restrict__ out, double* __restrict__ z) {
  __shared__ double red[32];
  for (int i = threadIdx.x; i < rank; i += blockDim.x) z[i] = rhs[perm[i]];
  __syncthreads();
  for (int row = 0; row < rank; ++row) {
    double s = 0.0;
    for (int c = threadIdx.x; c < row; c += blockDim.x) s += tri_at(T, ldt, upper, row, c) * z[c];
    s = block_sum(s, red);
    if (threadIdx.x == 0) z[row] = (z[row] - s) / tri_at(T, ldt, upper, row, row);
    __syncthreads();
  }
  for (int row = rank - 1; row >= 0; --row) {
    double s = 0.0;
    for (int c = row + 1 + threadIdx.x; c < rank; c += blockDim.x)
      s += tri_at(T, ldt, upper, c, row) * z[c];
    s = block_sum(s, red);
    if (threadIdx.x == 0) z[row] = (z[row] - s) / tri_at(T, ldt, upper, row, row);
    __syncthreads();
  }
  for (int i = threadIdx.x; i < n; i += blockDim.x) out[perm[i]] = (i < rank) ? z[i] : 0.0;
}

__global__ void k_eq_scaled_rhs(int n, const double* __restrict__ scale,
                                const double* __restrict__ p, double* __restrict__ q) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) q[i] = scale[i] * p[i] - q[i];
}
__global__ void k_eq_scale_vec(int n, const double* __restrict__ scale, double* __restrict__ v) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) v[i] *= scale[i];
}
__global__ void k_eq_scale_rows(int m, long long total, double* __restrict__ B,
                                const double* __restrict__ s) {
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x)
    B[e] /= s[e % m];
}
__global__ void k_eq_dot(int n, const double* __restrict__ a, const double* __restrict__ b,
                         double* __restrict__ out) {
  __shared__ double red[32];
  double s = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) s += a[i] * b[i];
  s = block_sum(s, red);
  if (threadIdx.x == 0) out[0] = s;
}
__global__ void k_eq_iota(int n, int* perm) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) perm[i] = i;
}

}  // namespace

void eq_normalize_columns(int m, int n, double* Bt, double* scale, cudaStream_t st) {
  if (n <= 0) return;
  k_eq_normalize<<<n, 256, 0, st>>>(m, Bt, scale);
  SDPX_LAUNCH_CHECK();
}
void eq_column_fingerprints(int m, int n, const double* Bt, unsigned long long* fp,
                            cudaStream_t st) {
  if (n <= 0) return;
  k_eq_fingerprint<<<n, 256, 0, st>>>(m, Bt, fp);
  SDPX_LAUNCH_CHECK();
}
void eq_columns_equal(int m, const double* Bt, const int* pairs, int npairs, int* equal,
                      cudaStream_t st) {
  if (npairs <= 0) return;
  k_eq_cols_equal<<<npairs, 256, 0, st>>>(m, Bt, pairs, equal);
  SDPX_LAUNCH_CHECK();
}
void eq_qr_pivoted(int m, int n, double* A, int lda, int* perm, double* rdiag, double* colnorm,
                   cudaStream_t st) {
  if (n <= 0) return;
  k_eq_qr<<<1, QR_THREADS, 0, st>>>(m, n, A, lda, perm, rdiag, colnorm);
  SDPX_LAUNCH_CHECK();
}
void eq_small_solve(int n, int rank, const double* T, int ldt, int upper, const int* perm,
                    const double* rhs, double* out, double* z, cudaStream_t st) {
  if (n <= 0) return;
  k_eq_small_solve<<<1, 256, 0, st>>>(n, rank, T, ldt, upper, perm, rhs, out, z);
  SDPX_LAUNCH_CHECK();
}
void eq_scaled_rhs(int n, const double* scale, const double* p, double* q, cudaStream_t st) {
  if (n <= 0) return;
  k_eq_scaled_rhs<<<ceil_div(n, 256), 256, 0, st>>>(n, scale, p, q);
  SDPX_LAUNCH_CHECK();
}
void eq_scale_vec(int n, const double* scale, double* v, cudaStream_t st) {
  if (n <= 0) return;
  k_eq_scale_vec<<<ceil_div(n, 256), 256, 0, st>>>(n, scale, v);
  SDPX_LAUNCH_CHECK();
}
void eq_scale_rows(int m, int n, double* B, const double* s, cudaStream_t st) {
  const long long total = (long long)m * n;
  if (total <= 0) return;
  k_eq_scale_rows<<<std::min(ceil_div(total, 256), 4096), 256, 0, st>>>(m, total, B, s);
  SDPX_LAUNCH_CHECK();
}
void eq_dot(int n, const double* a, const double* b, double* out, cudaStream_t st) {
  k_eq_dot<<<1, 256, 0, st>>>(n, a, b, out);
  SDPX_LAUNCH_CHECK();
}
void eq_iota(int n, int* perm, cudaStream_t st) {
  if (n <= 0) return;
  k_eq_iota<<<ceil_div(n, 256), 256, 0, st>>>(n, perm);
  SDPX_LAUNCH_CHECK();
}

}  // namespace sdpx
