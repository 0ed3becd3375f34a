// Mixed-precision workspace of the B200 core: FP32 factor of the Schur
// complement and buffers of the split-BF16 Schur assembly.
#pragma once
#include "common.cuh"

namespace sdpx {

struct MixedWorkspace {
  float* Sf = nullptr;      // m×m FP32 factor
  float* Dinv = nullptr;    // FP32 inverses of the 64×64 diagonal tiles
  float* v32 = nullptr;     // m
  float* w32 = nullptr;     // m
  int* info = nullptr;
  float* dmin = nullptr;
  float* dmax = nullptr;
  float* diag_store = nullptr;
  void* desc = nullptr;
  double cond_estimate = 1.0;
  ~MixedWorkspace() {
    for (void* p : {(void*)Sf, (void*)Dinv, (void*)v32, (void*)w32, (void*)info, (void*)dmin,
                    (void*)dmax, (void*)diag_store, desc})
      if (p) cudaFree(p);
  }
};

// FP64 ↔ FP32 conversions and the regularised FP32 copy of the lower S.
void copy_reg_f32(int m, const double* S, float* Sf, double reg, cudaStream_t st);
void f64_to_f32(long long n, const double* a, float* b, cudaStream_t st);
void f32_to_f64(long long n, const float* a, double* b, cudaStream_t st);

}  // namespace sdpx
