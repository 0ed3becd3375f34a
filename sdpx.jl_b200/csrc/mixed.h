// Mixed-precision workspace of the B200 core: FP32 factor of the Schur
// complement and buffers of the split-BF16 Schur assembly.
#pragma once
#include <vector>

#include "common.cuh"
#include "dbuf.h"

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
  // The device blocks behind the pointers above come from the process-wide
  // cache of idle device blocks, so a handle created and destroyed per solve
  // neither allocates them from the driver again nor synchronises the device
  // to free them.
  static constexpr int kBlocks = 32;
  DBuf<unsigned char> blocks[kBlocks];
  int n_blocks = 0;
  template <class P>
  void take(P*& ptr, size_t bytes) {
    if (n_blocks == kBlocks) throw CudaError("mixed workspace: more device blocks than reserved");
    blocks[n_blocks].alloc(bytes);
    ptr = static_cast<P*>(static_cast<void*>(blocks[n_blocks++].p));
  }
};

// FP64 ↔ FP32 conversions and the regularised FP32 copy of the lower S.
void copy_reg_f32(int m, const double* S, float* Sf, double reg, cudaStream_t st);
void f64_to_f32(long long n, const double* a, float* b, cudaStream_t st);
void f32_to_f64(long long n, const float* a, double* b, cudaStream_t st);

}  // namespace sdpx
