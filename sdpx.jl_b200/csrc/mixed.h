// Mixed-precision workspace of the B200 core: FP32 factor of the Schur
// complement and buffers of the split-BF16 Schur assembly.
#pragma once
#include <vector>

#include "common.cuh"

namespace sdpx {

struct MixedWorkspace {
  // split-BF16 Schur assembly buffers (allocated on first use)
  bool planes_ready = false;   // buffers allocated
  bool a_planes_valid = false; // planes of the current (scaled) constraint data
  long long Kp = 0;            // padded stacked K of the plane layout
  std::vector<int> kp;         // padded order per dense block
  std::vector<long long> po;   // plane offset per dense block
  std::vector<long long> ao;   // constraint-plane region of each dense block
  long long pog = 0;           // plane offset of the 1×1 group
  long long Ts = 0;            // per-variable stride of the T planes
  void* Apl[3] = {nullptr, nullptr, nullptr};
  void* Ppl[3] = {nullptr, nullptr, nullptr};
  void* Tpl[3] = {nullptr, nullptr, nullptr};
  void* Wpl[3] = {nullptr, nullptr, nullptr};
  void* Lpl[3] = {nullptr, nullptr, nullptr};
  float* partial = nullptr;
  int* err = nullptr;
  double* L64 = nullptr;    // FP32 factor promoted to FP64
  double* Linv = nullptr;   // explicit inverse of the factor (preconditioner apply)
  double* Dinv64 = nullptr;
  double* tmp64 = nullptr;
  float* Sf = nullptr;      // m×m FP32 factor
  float* Dinv = nullptr;    // FP32 inverses of the 64×64 diagonal tiles
  float* v32 = nullptr;     // m
  float* w32 = nullptr;     // m
  int* info = nullptr;
  float* dmin = nullptr;
  float* dmax = nullptr;
  void* desc = nullptr;
  double cond_estimate = 1.0;
  ~MixedWorkspace() {
    for (void* p : {(void*)Sf, (void*)Dinv, (void*)v32, (void*)w32, (void*)info, (void*)dmin,
                    (void*)dmax, desc, (void*)partial, (void*)err, (void*)L64,
                    (void*)Linv, (void*)Dinv64, (void*)tmp64})
      if (p) cudaFree(p);
    for (int i = 0; i < 3; ++i)
      for (void* p : {Apl[i], Ppl[i], Tpl[i], Wpl[i], Lpl[i]})
        if (p) cudaFree(p);
  }
};

// FP64 ↔ FP32 conversions and the regularised FP32 copy of the lower S.
void copy_reg_f32(int m, const double* S, float* Sf, double reg, cudaStream_t st);
void f64_to_f32(long long n, const double* a, float* b, cudaStream_t st);
void f32_to_f64(long long n, const float* a, double* b, cudaStream_t st);

}  // namespace sdpx
