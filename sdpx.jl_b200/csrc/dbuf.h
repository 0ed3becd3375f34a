// Owning device buffer used by the handles (api.cu, normal.cu).
//
// Released buffers go to a process-wide cache of idle device blocks instead of
// back to the driver: cudaMalloc costs ≈ 1.8 ms and cudaFree ≈ 2.9 ms per GB on
// the B200, and one dense-SDP handle of the m = 2000 workload holds ≈ 25 GB, so
// creating and destroying a handle per solve would spend > 100 ms in the driver.
// A request takes an idle block of the same device whose size is within
// [bytes, 1.25·bytes + 1 MB]; otherwise it calls cudaMalloc, and when that
// fails the device's idle blocks are freed and the call is retried.  A block
// enters the cache only once no queued work still uses it (the guarantee
// cudaFree gives): after a device synchronisation, or — while an owner that
// issues all its work on one stream releases its buffers after synchronising
// that stream (ReleaseScope) — without one, so that tearing down one solve
// does not wait for the work of concurrent solves on other streams.  Idle
// blocks of a device are capped at kIdleCap bytes;
// sdpx_b200_trim_device_cache() returns them all.
#pragma once
#include <cuda_runtime.h>

#include <cstddef>
#include <map>
#include <mutex>
#include <utility>

#include "common.cuh"

namespace sdpx {

namespace dcache {

constexpr size_t kIdleCap = 64ull << 30;  // idle bytes kept per device
constexpr int kMaxDev = 64;

struct Cache {
  std::mutex mu;
  std::multimap<size_t, std::pair<int, void*>> idle;  // block bytes → (device, pointer)
  size_t idle_bytes[kMaxDev] = {};
};
inline Cache& cache() {
  static Cache c;
  return c;
}

// True on this thread while an owner whose only stream is synchronised
// releases its buffers.
inline bool& owner_synced() {
  static thread_local bool flag = false;
  return flag;
}

// Frees every idle block of `dev` (all devices when dev < 0).
inline void trim(int dev) {
  Cache& c = cache();
  std::lock_guard<std::mutex> g(c.mu);
  for (auto it = c.idle.begin(); it != c.idle.end();) {
    if (dev < 0 || it->second.first == dev) {
      int cur = 0;
      cudaGetDevice(&cur);
      cudaSetDevice(it->second.first);
      cudaFree(it->second.second);
      cudaSetDevice(cur);
      if (it->second.first >= 0 && it->second.first < kMaxDev)
        c.idle_bytes[it->second.first] -= it->first;
      it = c.idle.erase(it);
    } else {
      ++it;
    }
  }
}

inline size_t idle_bytes(int dev) {
  Cache& c = cache();
  std::lock_guard<std::mutex> g(c.mu);
  return (dev >= 0 && dev < kMaxDev) ? c.idle_bytes[dev] : 0;
}

// A block of at least `bytes` on the current device; its true size in *got.
inline void* get(size_t bytes, int* dev_out, size_t* got) {
  int dev = 0;
  SDPX_CUDA(cudaGetDevice(&dev));
  *dev_out = dev;
  Cache& c = cache();
  {
    std::lock_guard<std::mutex> g(c.mu);
    const size_t hi = bytes + bytes / 4 + (1u << 20);
    for (auto it = c.idle.lower_bound(bytes); it != c.idle.end() && it->first <= hi; ++it) {
      if (it->second.first != dev) continue;
      void* p = it->second.second;
      *got = it->first;
      if (dev < kMaxDev) c.idle_bytes[dev] -= it->first;
      c.idle.erase(it);
      return p;
    }
  }
  void* p = nullptr;
  if (cudaMalloc(&p, bytes) != cudaSuccess) {
    cudaGetLastError();  // clear the allocation failure, free the idle blocks, retry
    trim(dev);
    SDPX_CUDA(cudaMalloc(&p, bytes));
  }
  *got = bytes;
  return p;
}

// Returns a block: after a device synchronisation it is idle, or freed when
// the device's idle blocks would exceed kIdleCap.
inline void put(void* p, size_t bytes, int dev) {
  if (!p) return;
  int cur = 0;
  cudaGetDevice(&cur);
  if (cur != dev) cudaSetDevice(dev);
  if (!owner_synced()) cudaDeviceSynchronize();
  Cache& c = cache();
  bool keep = false;
  {
    std::lock_guard<std::mutex> g(c.mu);
    if (dev >= 0 && dev < kMaxDev && c.idle_bytes[dev] + bytes <= kIdleCap) {
      c.idle.insert({bytes, {dev, p}});
      c.idle_bytes[dev] += bytes;
      keep = true;
    }
  }
  if (!keep) cudaFree(p);
  if (cur != dev) cudaSetDevice(cur);
}

// Declared as an owner's first member (so destroyed last): the owner's
// destructor synchronises its stream and calls begin(); the buffers released
// by the members destroyed after that skip the device synchronisation, and
// this member's destructor ends the scope.
struct ReleaseScope {
  void begin() { owner_synced() = true; }
  ~ReleaseScope() { owner_synced() = false; }
};

}  // namespace dcache

template <class T>
struct DBuf {
  T* p = nullptr;
  size_t n = 0;
  size_t bytes = 0;  // size of the block held (≥ n·sizeof(T))
  int dev = 0;
  void alloc(size_t count) {
    release();
    if (count == 0) count = 1;
    p = static_cast<T*>(dcache::get(count * sizeof(T), &dev, &bytes));
    n = count;
  }
  void zero(cudaStream_t st) { SDPX_CUDA(cudaMemsetAsync(p, 0, n * sizeof(T), st)); }
  void release() {
    if (p) dcache::put(p, bytes, dev);
    p = nullptr;
    n = 0;
    bytes = 0;
  }
  DBuf() = default;
  DBuf(const DBuf&) = delete;
  DBuf& operator=(const DBuf&) = delete;
  ~DBuf() { release(); }
};

}  // namespace sdpx
