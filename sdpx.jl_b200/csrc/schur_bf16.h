// Split-BF16 tcgen05 GEMM engine (schur_bf16.cu).
#pragma once
#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>

#include "common.cuh"

namespace sdpx {

// Row r of an operand/output starts at base + (r / inner)·os + (r % inner)·is elements.
struct RowMap {
  long long base;
  int inner;
  long long is, os;
  int extent;
};

// Three BF16 planes of a K-major operand stored as a row-major 2D tensor:
// element (row, k) of plane p is plane[p][row·pitch + k] for row < rows
// (pitch a multiple of 8 elements, bases 16-byte aligned).  Rows and K beyond
// the tensor read as zeros.
struct Plane2D {
  const __nv_bfloat16* plane[3];
  long long rows;
  long long pitch;
};

// Output planes: element (row, col) at plane[p][row_off(row) + (col / col_inner)·col_os + col % col_inner].
// col_inner, row offsets and col_extent are multiples of 8 (16-byte stores of 8 columns).
struct OutMap {
  __nv_bfloat16* plane[3];
  RowMap rows;
  int col_inner;
  long long col_os;
  int col_extent;
};

struct SplitSyrkPlan {
  int ntri = 0, nchunk = 0, kchunk = 0;
  size_t partial_floats = 0;
};

// out = A·Bᵀ (A rows × B rows, contraction over k < Ktot), split into planes.
// kmode: 0 full K, 1 A lower-triangular (k ≤ row), 2 B lower-triangular (k ≥ col).
void split_gemm_planes(const Plane2D& A, const Plane2D& B, int Ktot, const OutMap& out, int kmode,
                       int* err, cudaStream_t st);
SplitSyrkPlan plan_split_syrk(int m, long long Kp, int sm_count);
// Lower tiles of S (m×m FP64, column-major) = P̂ᵀP̂ over K = Kp, FP32 chunk tiles summed in FP64.
// ev_begin/ev_end (optional) are recorded around the SYRK kernel alone.
void split_syrk(const Plane2D& P, int m, int Kp, const SplitSyrkPlan& plan, float* partial,
                double* S, int* err, cudaStream_t st, cudaEvent_t ev_begin = nullptr,
                cudaEvent_t ev_end = nullptr);

// Rows of a column-major FP64 matrix (rows columns of K entries, leading
// dimension ld) → three BF16 planes of pitch Kp (zero padded past K).
void split_rows_f64(const double* src, long long ld, int rows, long long K, long long Kp,
                    __nv_bfloat16* const* planes, cudaStream_t st);
void split_A_dense(const double* A, long long K, int m, long long off, int k, int kp,
                   __nv_bfloat16* const* planes, long long Kp, long long o, cudaStream_t st);
void split_diag_rows(const double* A, long long K, int m, long long od, int nd, const double* LX,
                     const double* MY, __nv_bfloat16* const* planes, long long Kp, long long o,
                     cudaStream_t st);
void split_small(const double* M, int k, int kp, bool row_major, __nv_bfloat16* const* planes,
                 cudaStream_t st);

}  // namespace sdpx
