// Conversion helpers of the mixed-precision KKT path.
#include "mixed.h"

namespace sdpx {

__global__ void k_copy_reg_f32(int m, const double* S, float* Sf, double reg) {
  long long tot = (long long)m * m;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < tot;
       e += (long long)gridDim.x * blockDim.x) {
    int i = (int)(e % m), j = (int)(e / m);
    double v = (i >= j) ? S[e] : 0.0;
    if (i == j && reg != 0.0) v += reg * fmax(fabs(S[e]), 1.0);
    Sf[e] = (float)v;
  }
}
void copy_reg_f32(int m, const double* S, float* Sf, double reg, cudaStream_t st) {
  k_copy_reg_f32<<<std::min(4096, ceil_div((long long)m * m, 256)), 256, 0, st>>>(m, S, Sf, reg);
  SDPX_LAUNCH_CHECK();
}
__global__ void k_f64_to_f32(long long n, const double* a, float* b) {
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n;
       e += (long long)gridDim.x * blockDim.x)
    b[e] = (float)a[e];
}
__global__ void k_f32_to_f64(long long n, const float* a, double* b) {
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n;
       e += (long long)gridDim.x * blockDim.x)
    b[e] = (double)a[e];
}
void f64_to_f32(long long n, const double* a, float* b, cudaStream_t st) {
  if (n == 0) return;
  k_f64_to_f32<<<std::min(4096, ceil_div(n, 256)), 256, 0, st>>>(n, a, b);
  SDPX_LAUNCH_CHECK();
}
void f32_to_f64(long long n, const float* a, double* b, cudaStream_t st) {
  if (n == 0) return;
  k_f32_to_f64<<<std::min(4096, ceil_div(n, 256)), 256, 0, st>>>(n, a, b);
  SDPX_LAUNCH_CHECK();
}

}  // namespace sdpx
