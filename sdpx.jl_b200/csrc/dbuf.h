// Owning device buffer used by the handles (api.cu, normal.cu).
#pragma once
#include <cuda_runtime.h>

#include <cstddef>

#include "common.cuh"

namespace sdpx {

template <class T>
struct DBuf {
  T* p = nullptr;
  size_t n = 0;
  void alloc(size_t count) {
    release();
    if (count == 0) count = 1;
    SDPX_CUDA(cudaMalloc(&p, count * sizeof(T)));
    n = count;
  }
  void zero(cudaStream_t st) { SDPX_CUDA(cudaMemsetAsync(p, 0, n * sizeof(T), st)); }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
  }
  ~DBuf() { release(); }
};

}  // namespace sdpx
