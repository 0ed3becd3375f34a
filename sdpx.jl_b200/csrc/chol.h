// Batched Cholesky / triangular kernels (chol.cu).
#pragma once
#include <algorithm>

#include "common.cuh"

namespace sdpx {

template <class T>
struct MatDesc {
  T* a;     // column-major n×n, leading dimension ld
  int n;
  int ld;
};

// Lower Cholesky in place of every matrix in d_mats (device array of nmat
// descriptors, largest order nmax).  info[b] = 0 on success, else the 1-based
// index of the first non-positive pivot.  dmin/dmax receive min/max |L_ii|.
// The strict upper triangle is zeroed unless zero_upper is false (positive-
// definiteness tests that only read info/dmin/dmax).
template <class T, int NB>
void potrf_batched(const MatDesc<T>* d_mats, int nmat, int nmax, int* info, T* dmin, T* dmax,
                   cudaStream_t st, bool zero_upper = true);

// Grid-barrier state of one potrf_single call site (device memory, 16 bytes).
struct CoopBar {
  unsigned count, gen, err, fail;
};

// Lower Cholesky in place of one n×n matrix (leading dimension ld) in a single
// cooperative launch, for orders above the whole-panel shared-memory size.
// info[0] = 0 on success, the 1-based failing pivot, or −1 when a grid
// barrier timed out (the call site's `bar` must not be shared by concurrent
// calls).  dmin/dmax: min/max |L_ii|.
template <class T, int NB>
void potrf_single(T* a, int n, int ld, int* info, T* dmin, T* dmax, CoopBar* bar, bool zero_upper,
                  cudaStream_t st);

// Whether potrf_single is the faster path for one matrix of order n: FP64
// orders above the whole-panel shared-memory size (measured on the B200 with
// identical factors: 0.88 vs 0.93 ms at n = 1000, 1.78 vs 1.99 ms at 2000,
// 3.09 vs 3.26 ms at 3000; below that size, and in FP32, the batched path is
// as fast or faster).
template <class T, int NB>
inline bool potrf_single_pays(int n) {
  return sizeof(T) == 8 && sizeof(T) * (size_t)(n | 1) * NB > 224 * 1024;
}

// W_b = L_b^{-1} for lower-triangular L_b (W zero-initialised by the caller).
template <class T, int NB>
void trinv_batched(const MatDesc<T>* d_L, const MatDesc<T>* d_W, int nmat, int nmax,
                   cudaStream_t st);

// Inverses of the NB×NB diagonal tiles of a lower factor L (n×n): Dinv[s] (NB×NB, col-major).
template <class T, int NB>
void factor_diag_inverses(const T* L, long long ld, int n, T* Dinv, cudaStream_t st);

// rhs ← (L Lᵀ)^{-1} rhs by blocked forward/backward substitution (work: n).
template <class T, int NB>
void cholesky_solve(const T* L, long long ld, int n, const T* Dinv, T* rhs, T* work,
                    cudaStream_t st);

// Linv = L⁻¹ (n×n, column-major, ld n) by recursive doubling over 64×64 tiles.
// Dinv: ceil(n/64)·64·64 scratch, tmp: n·n scratch.
void trinv_recursive_f64(const double* L, int n, double* Linv, double* Dinv, double* tmp,
                         cudaStream_t st);

}  // namespace sdpx
