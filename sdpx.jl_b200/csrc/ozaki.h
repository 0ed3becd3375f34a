// FP64 Gram matrix on the int8 tensor cores by exact integer digit products
// (ozaki.cu).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "common.cuh"

namespace sdpx {

constexpr int OZ_DIGITS = 8;  // int8 digits per value: 6 + 7·7 = 55 significant bits

struct OzakiPlan {
  int m = 0;
  long long K = 0, Kp = 0;    // contraction length, padded to a multiple of 64
  int ntile_r = 0, ntile_c = 0, ntri = 0, nchunk = 0, kchunk = 0;
  size_t digit_bytes = 0;     // OZ_DIGITS · m · Kp
  size_t partial_doubles = 0; // nchunk · ntri · 128 · 64
  size_t partial_alloc_doubles = 0;  // partial tiles + the tile-pair table
};

OzakiPlan plan_ozaki_syrk(int m, long long K, int sm_count);

// S (m×m, column-major, lower triangle and diagonal written) = PᵀP for P
// (K×m, column-major, ld = K).  digits: plan.digit_bytes of scratch, exps: m
// ints, partial: plan.partial_alloc_doubles.  err: device flag set when a bounded
// wait gave up.  ev_begin/ev_end (optional) bracket the tensor-core kernel.
// dense_hi (optional, m entries): the rows [0, tail_off) of P were written by
// ozaki_gemm with OzGemm::colmax = dense_hi, so their per-column maxima are
// known and only the rows [tail_off, K) are scanned for the column exponents.
void ozaki_syrk(const double* P, const OzakiPlan& plan, int8_t* digits, int* exps, double* partial,
                double* S, int* err, cudaStream_t st, cudaEvent_t ev_begin = nullptr,
                cudaEvent_t ev_end = nullptr, const unsigned* dense_hi = nullptr,
                long long tail_off = 0);

// ---- general products C[a, b] = Σ_j X[a, j]·Y[b, j] on digit planes --------

// `rows` FP64 row vectors of length `len`: row n starts at
// base + (n / inner)·os + (n % inner)·is, its element j sits at +j·es.
// tri = 1 keeps only the elements j ≤ n of row n, tri = 2 only j ≥ n (the
// others read as zero: triangular factors whose other half is not stored).
struct OzRows {
  const double* base = nullptr;
  long long rows = 0;
  int inner = 1 << 30;
  long long is = 0, os = 0, es = 1;
  int len = 0;
  int tri = 0;
};

// Padded digit-row width for a contraction length (multiple of 32, ≥ 32).
long long oz_kpad(int len);

// Digit planes of the rows, stored in pairs (t, t + 4): digit t of row n,
// position j, at digits[(t mod 4)·2·plane + n·2·Kp + 64·(j div 32) +
// 32·(t div 4) + (j mod 32)] (zero for j ≥ len), the row's power-of-two
// exponent at exps[n].  plane ≥ rows·Kp (8·plane bytes in all).
void ozaki_digits_rows(const OzRows& r, long long Kp, long long plane, int8_t* digits, int* exps,
                       cudaStream_t st);

// out[(a / a_inner)·a_os + (a % a_inner)·a_is + b·b_stride] = Σ_j X[a, j]·Y[b, j]
// for the digit planes of X (rows_a rows) and Y (rows_b rows), both Kp wide, in
// the pair layout of ozaki_digits_rows (x_plane, y_plane: its `plane`).
// kmode 1: row b of Y is zero beyond j = b, kmode 2: before j = b (the
// contraction of a tile of Y rows is cut to where they can be nonzero).
struct OzGemm {
  const int8_t* xd = nullptr;
  long long x_plane = 0;
  int rows_a = 0;
  const int* ea = nullptr;
  const int8_t* yd = nullptr;
  long long y_plane = 0;
  int rows_b = 0;
  const int* eb = nullptr;
  long long Kp = 0;
  int kmode = 0;
  double* out = nullptr;
  int a_inner = 1 << 30;
  long long a_is = 0, a_os = 0, b_stride = 0;
  // Optional: colmax[a / a_inner] = max(colmax[...], high word of |out|) — the
  // exponent field of each group's largest written magnitude (caller zeroes it).
  unsigned* colmax = nullptr;
};
void ozaki_gemm(const OzGemm& g, int sm_count, int* err, cudaStream_t st);

}  // namespace sdpx
