// Device passes of the cold-path result certificate (SDPX's
// `result_certificate`, src/validation.jl:948-1115): one streaming pass over
// the original constraint data per direction (rows for the primal block
// backward errors, columns for the dual ones), block statistics and the
// symmetrised, shifted copies the PSD checks factor.
#include <cuda_runtime.h>

#include "certificate.h"

namespace sdpx {
namespace {

__device__ __forceinline__ double cw_ratio(double r, double scale) {
  double a = fabs(r);
  if (scale == 0.0) return a == 0.0 ? 0.0 : (1.0 / 0.0);
  return a / scale;
}

__global__ void k_cert_rows_part(const double* __restrict__ A, long long K, int m,
                                 const double* __restrict__ x, int chunks,
                                 double* __restrict__ part) {
  long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  int ch = blockIdx.y;
  if (r >= K) return;
  int per = (m + chunks - 1) / chunks;
  int i0 = ch * per, i1 = min(m, i0 + per);
  double sv = 0.0, sn = 0.0, sr = 0.0;
  for (int i = i0; i < i1; ++i) {
    double a = A[(long long)i * K + r];
    double xi = x[i];
    sv += a * xi;
    sn += fabs(a);
    sr += fabs(a) * fabs(xi);
  }
  part[(long long)ch * K + r] = sv;
  part[(long long)(chunks + ch) * K + r] = sn;
  part[(long long)(2 * chunks + ch) * K + r] = sr;
}

__global__ void k_cert_rows_finish(long long K, int chunks, const double* __restrict__ part,
                                   const double* __restrict__ X, const double* __restrict__ C,
                                   double* absR, double* mixed, double* strict) {
  long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (r >= K) return;
  double sv = 0.0, sn = 0.0, sr = 0.0;
  for (int c = 0; c < chunks; ++c) {
    sv += part[(long long)c * K + r];
    sn += part[(long long)(chunks + c) * K + r];
    sr += part[(long long)(2 * chunks + c) * K + r];
  }
  double R = (sv - X[r]) - C[r];
  double nominal = fabs(C[r]) + sn;
  double realized = (fabs(X[r]) + fabs(C[r])) + sr;
  absR[r] = fabs(R);
  mixed[r] = cw_ratio(R, nominal + realized);
  strict[r] = cw_ratio(R, realized);
}

__global__ void k_cert_cols(const double* __restrict__ A, long long K, int m,
                            const double* __restrict__ Y, const double* __restrict__ c,
                            double* absv, double* mixed, double* strict,
                            const double* __restrict__ B, int n, const double* __restrict__ yv) {
  __shared__ double red[32];
  int i = blockIdx.x;
  const double* col = A + (long long)i * K;
  double sv = 0.0, sn = 0.0, sr = 0.0;
  for (long long r = threadIdx.x; r < K; r += blockDim.x) {
    double a = col[r], y = Y[r];
    sv += a * y;
    sn += fabs(a);
    sr += fabs(a) * fabs(y);
  }
  // equality rows: v_i −= Σ_j B[i,j]·y_j with their |B|, |B|·|y| scales
  // (`_accumulate_equality_dual_scales!`, src/validation.jl:629-644)
  double bv = 0.0, bn = 0.0, br = 0.0;
  for (int j = threadIdx.x; j < n; j += blockDim.x) {
    const double bij = B[i + (long long)j * m];
    bv += bij * yv[j];
    bn += fabs(bij);
    br += fabs(bij) * fabs(yv[j]);
  }
  sv = block_sum(sv, red);
  __syncthreads();
  sn = block_sum(sn, red);
  __syncthreads();
  sr = block_sum(sr, red);
  __syncthreads();
  if (n > 0) {
    bv = block_sum(bv, red);
    __syncthreads();
    bn = block_sum(bn, red);
    __syncthreads();
    br = block_sum(br, red);
  }
  if (threadIdx.x == 0) {
    double v = c[i] - sv - bv;
    double nominal = fabs(c[i]) + sn + bn;
    double realized = fabs(c[i]) + sr + br;
    absv[i] = fabs(v);
    mixed[i] = cw_ratio(v, nominal + realized);
    strict[i] = cw_ratio(v, realized);
  }
}

__global__ void k_cert_dot(long long n, const double* __restrict__ a, const double* __restrict__ b,
                           double* out) {
  __shared__ double red[32];
  double s = 0.0, bad = 0.0;
  for (long long e = threadIdx.x; e < n; e += blockDim.x) {
    double av = a[e];
    s += av * b[e];
    if (!isfinite(av)) bad += 1.0;
  }
  s = block_sum(s, red);
  __syncthreads();
  bad = block_sum(bad, red);
  if (threadIdx.x == 0) {
    out[0] += s;
    out[1] += bad;
  }
}

__global__ void k_cert_block_stats(const long long* off, const int* kk, const double* M,
                                   double* out) {
  __shared__ double red[32];
  const int b = blockIdx.x, k = kk[b];
  const double* P = M + off[b];
  double bad = 0.0, mx = 0.0, sym = 0.0;
  for (int e = threadIdx.x; e < k * k; e += blockDim.x) {
    int r = e % k, c = e / k;
    double v = P[e];
    if (!isfinite(v)) bad += 1.0;
    mx = fmax(mx, fabs(v));
    if (r < c) sym = fmax(sym, fabs(v - P[(long long)r * k + c]));
  }
  bad = block_sum(bad, red);
  __syncthreads();
  mx = block_max(mx, red);
  __syncthreads();
  sym = block_max(sym, red);
  if (threadIdx.x == 0) {
    out[3 * b] = bad;
    out[3 * b + 1] = mx;
    out[3 * b + 2] = sym;
  }
}

__global__ void k_cert_sym_shift(const long long* off, const int* kk, int nb, const double* M,
                                 const double* shift, double* S) {
  const int b = blockIdx.y;
  if (b >= nb) return;
  const int k = kk[b];
  const double* P = M + off[b];
  double* Q = S + off[b];
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < k * k; e += gridDim.x * blockDim.x) {
    int r = e % k, c = e / k;
    double v = (P[e] + P[(long long)r * k + c]) / 2.0;
    if (r == c) v += shift[b];
    Q[e] = v;
  }
}

}  // namespace

void cert_primal_rows(const double* A, long long K, int m, const double* x, const double* X,
                      const double* C, double* part, int chunks, double* absR, double* mixed,
                      double* strict, cudaStream_t st) {
  if (K == 0) return;
  dim3 g(ceil_div(K, 256), chunks);
  k_cert_rows_part<<<g, 256, 0, st>>>(A, K, m, x, chunks, part);
  k_cert_rows_finish<<<ceil_div(K, 256), 256, 0, st>>>(K, chunks, part, X, C, absR, mixed, strict);
  SDPX_LAUNCH_CHECK_N(2);
}

void cert_dual_cols(const double* A, long long K, int m, const double* Y, const double* c,
                    double* absv, double* mixed, double* strict, cudaStream_t st, const double* B,
                    int n, const double* y) {
  if (m == 0) return;
  k_cert_cols<<<m, 512, 0, st>>>(A, K, m, Y, c, absv, mixed, strict, B, n, y);
  SDPX_LAUNCH_CHECK();
}

// One CTA per equality j: lhs = Σ_i B[i,j]·x_i, residual |lhs − b_j|,
// nominal |b_j| + Σ|B[i,j]|, realized |b_j| + Σ|B[i,j]|·|x_i|
// (`_equality_backward_errors`, src/validation.jl:454-482).
__global__ void k_cert_equality(const double* __restrict__ B, int m, const double* __restrict__ x,
                                const double* __restrict__ b, double* absr, double* mixed,
                                double* strict) {
  __shared__ double red[32];
  const int j = blockIdx.x;
  const double* col = B + (long long)j * m;
  double lhs = 0.0, sn = 0.0, sr = 0.0;
  for (int i = threadIdx.x; i < m; i += blockDim.x) {
    const double a = col[i];
    lhs += a * x[i];
    sn += fabs(a);
    sr += fabs(a) * fabs(x[i]);
  }
  lhs = block_sum(lhs, red);
  __syncthreads();
  sn = block_sum(sn, red);
  __syncthreads();
  sr = block_sum(sr, red);
  if (threadIdx.x == 0) {
    const double v = lhs - b[j];
    absr[j] = fabs(v);
    mixed[j] = cw_ratio(v, fabs(b[j]) + sn + fabs(b[j]) + sr);
    strict[j] = cw_ratio(v, fabs(b[j]) + sr);
  }
}

void cert_equality_rows(const double* B, int m, int n, const double* x, const double* b,
                        double* absr, double* mixed, double* strict, cudaStream_t st) {
  if (n == 0) return;
  k_cert_equality<<<n, 256, 0, st>>>(B, m, x, b, absr, mixed, strict);
  SDPX_LAUNCH_CHECK();
}

void cert_dot(long long n, const double* a, const double* b, double* out, cudaStream_t st) {
  if (n == 0) return;
  k_cert_dot<<<1, 1024, 0, st>>>(n, a, b, out);
  SDPX_LAUNCH_CHECK();
}

void cert_block_stats(const long long* off, const int* k, int nb, const double* M, double* out,
                      cudaStream_t st) {
  if (nb == 0) return;
  k_cert_block_stats<<<nb, 256, 0, st>>>(off, k, M, out);
  SDPX_LAUNCH_CHECK();
}

void cert_sym_shift(const long long* off, const int* k, int nb, int kmax, const double* M,
                    const double* shift, double* S, cudaStream_t st) {
  if (nb == 0) return;
  dim3 g(std::min(64, ceil_div((long long)kmax * kmax, 256)), nb);
  k_cert_sym_shift<<<g, 256, 0, st>>>(off, k, nb, M, shift, S);
  SDPX_LAUNCH_CHECK();
}

}  // namespace sdpx
