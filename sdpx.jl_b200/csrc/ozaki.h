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
void ozaki_syrk(const double* P, const OzakiPlan& plan, int8_t* digits, int* exps, double* partial,
                double* S, int* err, cudaStream_t st, cudaEvent_t ev_begin = nullptr,
                cudaEvent_t ev_end = nullptr);

}  // namespace sdpx
