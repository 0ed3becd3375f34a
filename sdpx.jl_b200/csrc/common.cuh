// Shared device helpers for the SDPX B200 core (sm_100a).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <cstdio>
#include <stdexcept>
#include <string>

namespace sdpx {

struct CudaError : std::runtime_error {
  using std::runtime_error::runtime_error;
};

#define SDPX_CUDA(call)                                                                  \
  do {                                                                                   \
    cudaError_t e__ = (call);                                                            \
    if (e__ != cudaSuccess)                                                              \
      throw ::sdpx::CudaError(std::string(#call) + ": " + cudaGetErrorString(e__) +    \
                              " (" + __FILE__ + ":" + std::to_string(__LINE__) + ")"); \
  } while (0)

// Every launch site ends with SDPX_LAUNCH_CHECK(n): check the launch and add n
// to the process-wide kernel-launch counter (sdpx_b200_launch_count).
void note_launches(unsigned long long n);
#define SDPX_LAUNCH_CHECK_N(n)        \
  do {                                \
    SDPX_CUDA(cudaGetLastError());    \
    ::sdpx::note_launches(n);         \
  } while (0)
#define SDPX_LAUNCH_CHECK() SDPX_LAUNCH_CHECK_N(1)

inline int ceil_div(long long a, long long b) { return (int)((a + b - 1) / b); }

// ---------------------------------------------------------------------------
// Operand addressing.  Every matrix operand of the FP64 tile engine is read as
//   addr(mn, kk) = base + off(mn) + kk * kstride,
//   off(mn)      = (mn / inner) * outer_stride + (mn % inner) * inner_stride.
// The two-level form lets one GEMM walk a "stacked" panel whose logical columns
// are the k×k coefficient matrices of all m variables laid out one variable
// after another (column i of the stacked constraint matrix holds vec(A_i) of
// every block), without materialising a reshaped copy.
// ---------------------------------------------------------------------------
struct Opnd {
  const double* base;
  long long kstride;
  long long inner_stride;
  long long outer_stride;
  int inner;
  int mn_extent;
  int k_extent;
};

struct OutDesc {
  double* base;
  long long row_inner_stride, row_outer_stride;
  int row_inner;
  long long col_inner_stride, col_outer_stride;
  int col_inner;
  int rows, cols;
};

__host__ __device__ inline long long two_level(int idx, int inner, long long is, long long os) {
  return (long long)(idx / inner) * os + (long long)(idx % inner) * is;
}

__host__ inline Opnd plain_colmajor(const double* p, int rows, int cols, long long ld, bool k_is_row) {
  // Matrix M (rows×cols, column-major, leading dimension ld).
  // k_is_row: the contraction index runs over rows (operand is Mᵀ-like access).
  Opnd o;
  o.base = p;
  o.inner = 1 << 30;
  o.outer_stride = 0;
  if (k_is_row) {  // element (mn = col, kk = row)
    o.kstride = 1;
    o.inner_stride = ld;
    o.mn_extent = cols;
    o.k_extent = rows;
  } else {  // element (mn = row, kk = col)
    o.kstride = ld;
    o.inner_stride = 1;
    o.mn_extent = rows;
    o.k_extent = cols;
  }
  return o;
}

// ---------------------------------------------------------------------------
// FP64 tensor-core MMA: D(8×8) += A(8×4) · B(4×8), one double per thread for
// A and B, two for C/D (PTX ISA, mma.m8n8k4 with .f64).
// Fragment ownership (lane = 4*g + t):  a = A[g][t], b = B[t][g],
// c0/c1 = C[g][2t], C[g][2t+1].
// ---------------------------------------------------------------------------
__device__ __forceinline__ void dmma_8x8x4(double& c0, double& c1, double a, double b) {
  asm volatile(
      "mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
      : "+d"(c0), "+d"(c1)
      : "d"(a), "d"(b));
}

__device__ __forceinline__ void cp_async8(void* smem, const void* gmem, bool pred) {
  unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  int n = pred ? 8 : 0;  // zero-fill when out of range
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(s), "l"(gmem), "r"(n));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}

__device__ __forceinline__ double warp_sum(double v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ double warp_max(double v) {
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}
__device__ __forceinline__ double warp_min(double v) {
  for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// Block-wide reductions (blockDim.x multiple of 32, ≤ 1024). `red` holds 32 doubles.
__device__ inline double block_sum(double v, double* red) {
  v = warp_sum(v);
  int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) red[w] = v;
  __syncthreads();
  int nw = (blockDim.x + 31) >> 5;
  v = (threadIdx.x < nw) ? red[threadIdx.x] : 0.0;
  if (w == 0) v = warp_sum(v);
  if (threadIdx.x == 0) red[0] = v;
  __syncthreads();
  double r = red[0];
  __syncthreads();
  return r;
}
__device__ inline double block_max(double v, double* red) {
  v = warp_max(v);
  int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) red[w] = v;
  __syncthreads();
  int nw = (blockDim.x + 31) >> 5;
  v = (threadIdx.x < nw) ? red[threadIdx.x] : -1.0 / 0.0;
  if (w == 0) v = warp_max(v);
  if (threadIdx.x == 0) red[0] = v;
  __syncthreads();
  double r = red[0];
  __syncthreads();
  return r;
}

// Atomic max on a non-negative double (IEEE order of non-negative doubles
// matches their bit patterns as unsigned integers).  NaN is propagated as +inf
// so a poisoned input never reads as small.
__device__ inline void atomic_max_nonneg(double* addr, double v) {
  if (!(v == v)) v = 1.0 / 0.0;
  unsigned long long* a = reinterpret_cast<unsigned long long*>(addr);
  unsigned long long nv = __double_as_longlong(v);
  atomicMax(a, nv);
}

// K-range policies for triangular operands.
enum KRange : int {
  KR_FULL = 0,      // [0, K)
  KR_A_LOWER = 1,   // A lower triangular: k ≤ row → [0, min(K, m0+BM))
  KR_A_UPPER = 2,   // A upper triangular: k ≥ row → [m0, K)
  KR_B_LOWER = 3,   // B lower triangular: k ≥ col → [n0, K)
  KR_B_UPPER = 4,   // B upper triangular: k ≤ col → [0, min(K, n0+BN))
};

// Per-(kernel, device) one-time opt-in to large dynamic shared memory.
void smem_attr_ensure(const void* kern, size_t bytes);  // defined in api.cu
template <class Kern>
inline void ensure_smem(Kern kern, size_t bytes) {
  if (bytes <= 48 * 1024) return;
  smem_attr_ensure((const void*)kern, bytes);
}

}  // namespace sdpx
