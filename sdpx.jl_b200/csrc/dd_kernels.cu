// Double-double kernels over the stacked layout (see dd_kernels.h).
//
// Every reduction keeps a fixed order (rows of a chunk in increasing order,
// chunks in increasing order, a fixed shuffle tree inside a CTA), so results
// are bitwise repeatable.  These kernels serve the extended-precision
// residuals (adjoint refinement): their cost is ~20 double operations per
// multiply-add, acceptable for passes that run a few times per call.
#include "dd_kernels.h"

#include "common.cuh"
#include "dd.cuh"

namespace sdpx {

namespace {

constexpr int kTile = 16;

__global__ void k_dd_gemv_n_part(const double* __restrict__ A, long long K, int m,
                                 const double* __restrict__ vh, const double* __restrict__ vl,
                                 int chunks, double* __restrict__ ph, double* __restrict__ pl) {
  const long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (r >= K) return;
  const int ch = blockIdx.y;
  const int per = (m + chunks - 1) / chunks;
  const int i0 = ch * per, i1 = min(m, i0 + per);
  ddv acc = {0.0, 0.0};
  for (int i = i0; i < i1; ++i) acc = dd_add(acc, dd_mul_d(dd_load(vh, vl, i), A[r + (long long)i * K]));
  dd_store(ph, pl, (long long)ch * K + r, acc);
}

__global__ void k_dd_gemv_n_reduce(const double* __restrict__ ph, const double* __restrict__ pl,
                                   long long K, int chunks, double* __restrict__ oh,
                                   double* __restrict__ ol) {
  const long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (r >= K) return;
  ddv acc = {0.0, 0.0};
  for (int c = 0; c < chunks; ++c) acc = dd_add(acc, dd_load(ph, pl, (long long)c * K + r));
  dd_store(oh, ol, r, acc);
}

__global__ void k_dd_gemv_t(const double* __restrict__ A, long long K,
                            const double* __restrict__ zh, const double* __restrict__ zl,
                            double* __restrict__ oh, double* __restrict__ ol) {
  __shared__ double sh[32], sl[32];
  const int i = blockIdx.x;
  const double* col = A + (long long)i * K;
  ddv acc = {0.0, 0.0};
  for (long long r = threadIdx.x; r < K; r += blockDim.x)
    acc = dd_add(acc, dd_mul_d(dd_load(zh, zl, r), col[r]));
  for (int o = 16; o > 0; o >>= 1) acc = dd_add(acc, dd_shfl_xor(acc, o));
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0) {
    sh[w] = acc.hi;
    sl[w] = acc.lo;
  }
  __syncthreads();
  if (w == 0) {
    acc = lane < (int)(blockDim.x >> 5) ? ddv{sh[lane], sl[lane]} : ddv{0.0, 0.0};
    for (int o = 16; o > 0; o >>= 1) acc = dd_add(acc, dd_shfl_xor(acc, o));
    if (lane == 0) dd_store(oh, ol, i, acc);
  }
}

// 16×16 output tile per CTA, block b = blockIdx.z; inner dimension staged in
// shared memory 16 at a time.
__global__ void k_dd_gemm_blocks(const long long* __restrict__ doff, const int* __restrict__ dk,
                                 const double* __restrict__ Ah, const double* __restrict__ Al,
                                 const double* __restrict__ Bh, const double* __restrict__ Bl,
                                 double* __restrict__ Ch, double* __restrict__ Cl) {
  __shared__ double ash[kTile][kTile + 1], asl[kTile][kTile + 1];
  __shared__ double bsh[kTile][kTile + 1], bsl[kTile][kTile + 1];
  const int b = blockIdx.z;
  const int k = dk[b];
  const int r0 = blockIdx.x * kTile, c0 = blockIdx.y * kTile;
  if (r0 >= k || c0 >= k) return;  // uniform per CTA
  const long long o = doff[b];
  const int tx = threadIdx.x % kTile, ty = threadIdx.x / kTile;
  const int i = r0 + tx, j = c0 + ty;
  ddv acc = {0.0, 0.0};
  for (int t0 = 0; t0 < k; t0 += kTile) {
    const int ta = t0 + ty, tb = t0 + tx;
    const bool va = i < k && ta < k, vb = tb < k && j < k;
    const long long ia = o + i + (long long)ta * k, ib = o + tb + (long long)j * k;
    ash[tx][ty] = va ? Ah[ia] : 0.0;
    asl[tx][ty] = (va && Al) ? Al[ia] : 0.0;
    bsh[tx][ty] = vb ? Bh[ib] : 0.0;
    bsl[tx][ty] = (vb && Bl) ? Bl[ib] : 0.0;
    __syncthreads();
    const int tn = min(kTile, k - t0);
    for (int t = 0; t < tn; ++t)
      acc = dd_add(acc, dd_mul(ddv{ash[tx][t], asl[tx][t]}, ddv{bsh[t][ty], bsl[t][ty]}));
    __syncthreads();
  }
  if (i < k && j < k) dd_store(Ch, Cl, o + i + (long long)j * k, acc);
}

__global__ void k_dd_axpby(long long n, double sa, const double* ah, const double* al, double sb,
                           const double* bh, const double* bl, double* ch, double* cl) {
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n;
       e += (long long)gridDim.x * blockDim.x) {
    ddv v = dd_mul_d(dd_load(ah, al, e), sa);
    if (bh) v = dd_add(v, dd_mul_d(dd_load(bh, bl, e), sb));
    dd_store(ch, cl, e, v);
  }
}

__global__ void k_dd_eye_minus_blocks(const long long* __restrict__ doff,
                                      const int* __restrict__ dk, const double* ah,
                                      const double* al, double* ch, double* cl) {
  const int b = blockIdx.y;
  const int k = dk[b];
  const long long o = doff[b];
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < k * k; e += gridDim.x * blockDim.x) {
    const int r = e % k, c = e / k;
    ddv v = dd_neg(dd_load(ah, al, o + e));
    if (r == c) v = dd_add(v, ddv{1.0, 0.0});
    dd_store(ch, cl, o + e, v);
  }
}

__global__ void k_dd_sym_blocks(const long long* __restrict__ doff, const int* __restrict__ dk,
                                const double* __restrict__ ah, const double* __restrict__ al,
                                double* __restrict__ ch, double* __restrict__ cl) {
  const int b = blockIdx.y;
  const int k = dk[b];
  const long long o = doff[b];
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < k * k; e += gridDim.x * blockDim.x) {
    const int r = e % k, c = e / k;
    const ddv v = dd_add(dd_load(ah, al, o + e), dd_load(ah, al, o + c + (long long)r * k));
    dd_store(ch, cl, o + e, dd_mul_d(v, 0.5));
  }
}

__global__ void k_dd_diag_recip(int nd, long long od, const double* xh, const double* xl,
                                double* ch, double* cl) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= nd) return;
  dd_store(ch, cl, od + j, dd_div(ddv{1.0, 0.0}, dd_load(xh, xl, od + j)));
}

__global__ void k_dd_diag_mul(int nd, long long od, const double* ah, const double* al,
                              const double* bh, const double* bl, double* ch, double* cl) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= nd) return;
  dd_store(ch, cl, od + j, dd_mul(dd_load(ah, al, od + j), dd_load(bh, bl, od + j)));
}

// ⟨a, b⟩ in double-double (a, b double-double vectors; a null low half reads
// as 0), one CTA of 1024 threads; out[0], out[1] = hi, lo.
__global__ void __launch_bounds__(1024) k_dd_dot(long long n, const double* ah, const double* al,
                                                 const double* bh, const double* bl,
                                                 double* out) {
  __shared__ double red[64];
  ddv s{0.0, 0.0};
  for (long long i = threadIdx.x; i < n; i += blockDim.x)
    s = dd_add(s, dd_mul(dd_load(ah, al, i), dd_load(bh, bl, i)));
  for (int o = 16; o > 0; o >>= 1) s = dd_add(s, dd_shfl_xor(s, o));
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane == 0) {
    red[2 * w] = s.hi;
    red[2 * w + 1] = s.lo;
  }
  __syncthreads();
  if (w == 0) {
    ddv t = lane < (int)(blockDim.x >> 5) ? ddv{red[2 * lane], red[2 * lane + 1]} : ddv{0.0, 0.0};
    for (int o = 16; o > 0; o >>= 1) t = dd_add(t, dd_shfl_xor(t, o));
    if (lane == 0) {
      out[0] = t.hi;
      out[1] = t.lo;
    }
  }
}

}  // namespace

void dd_gemv_n(const double* A, long long K, int m, const double* vh, const double* vl,
               double* ph, double* pl, int chunks, double* oh, double* ol, cudaStream_t st) {
  if (K == 0) return;
  k_dd_gemv_n_part<<<dim3(ceil_div(K, 256), chunks), 256, 0, st>>>(A, K, m, vh, vl, chunks, ph,
                                                                    pl);
  k_dd_gemv_n_reduce<<<ceil_div(K, 256), 256, 0, st>>>(ph, pl, K, chunks, oh, ol);
  SDPX_LAUNCH_CHECK_N(2);
}

void dd_gemv_t(const double* A, long long K, int m, const double* zh, const double* zl,
               double* oh, double* ol, cudaStream_t st) {
  if (m == 0) return;
  k_dd_gemv_t<<<m, 512, 0, st>>>(A, K, zh, zl, oh, ol);
  SDPX_LAUNCH_CHECK();
}

void dd_gemm_blocks(const long long* doff, const int* dk, int nb, int kmax, const double* Ah,
                    const double* Al, const double* Bh, const double* Bl, double* Ch, double* Cl,
                    cudaStream_t st) {
  if (nb == 0 || kmax == 0) return;
  const int t = ceil_div(kmax, kTile);
  k_dd_gemm_blocks<<<dim3(t, t, nb), kTile * kTile, 0, st>>>(doff, dk, Ah, Al, Bh, Bl, Ch, Cl);
  SDPX_LAUNCH_CHECK();
}

void dd_axpby(long long n, double sa, const double* ah, const double* al, double sb,
              const double* bh, const double* bl, double* ch, double* cl, cudaStream_t st) {
  if (n == 0) return;
  k_dd_axpby<<<std::min(4096, ceil_div(n, 256)), 256, 0, st>>>(n, sa, ah, al, sb, bh, bl, ch, cl);
  SDPX_LAUNCH_CHECK();
}

void dd_eye_minus_blocks(const long long* doff, const int* dk, int nb, int kmax, const double* ah,
                         const double* al, double* ch, double* cl, cudaStream_t st) {
  if (nb == 0 || kmax == 0) return;
  k_dd_eye_minus_blocks<<<dim3(std::min(256, ceil_div((long long)kmax * kmax, 256)), nb), 256, 0,
                          st>>>(doff, dk, ah, al, ch, cl);
  SDPX_LAUNCH_CHECK();
}

void dd_sym_blocks(const long long* doff, const int* dk, int nb, int kmax, const double* ah,
                   const double* al, double* ch, double* cl, cudaStream_t st) {
  if (nb == 0 || kmax == 0) return;
  k_dd_sym_blocks<<<dim3(std::min(256, ceil_div((long long)kmax * kmax, 256)), nb), 256, 0, st>>>(
      doff, dk, ah, al, ch, cl);
  SDPX_LAUNCH_CHECK();
}

void dd_diag_recip(int nd, long long od, const double* xh, const double* xl, double* ch,
                   double* cl, cudaStream_t st) {
  if (nd == 0) return;
  k_dd_diag_recip<<<ceil_div(nd, 256), 256, 0, st>>>(nd, od, xh, xl, ch, cl);
  SDPX_LAUNCH_CHECK();
}

void dd_diag_mul(int nd, long long od, const double* ah, const double* al, const double* bh,
                 const double* bl, double* ch, double* cl, cudaStream_t st) {
  if (nd == 0) return;
  k_dd_diag_mul<<<ceil_div(nd, 256), 256, 0, st>>>(nd, od, ah, al, bh, bl, ch, cl);
  SDPX_LAUNCH_CHECK();
}

void dd_dot(long long n, const double* ah, const double* al, const double* bh, const double* bl,
            double* out, cudaStream_t st) {
  k_dd_dot<<<1, 1024, 0, st>>>(n, ah, al, bh, bl, out);
  SDPX_LAUNCH_CHECK();
}

}  // namespace sdpx
