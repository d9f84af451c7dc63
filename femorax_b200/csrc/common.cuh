// Shared device helpers: CUDA error checks, device buffers, launch helpers.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "host.hpp"

namespace fx {

inline void cuda_check(cudaError_t e, const char* what) {
  if (e != cudaSuccess) throw Error(FX_E_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}
#define FX_CUDA(call) ::fx::cuda_check((call), #call)
#define FX_LAUNCH_CHECK(name) ::fx::cuda_check(cudaGetLastError(), name)

// An owning device array.
template <class T>
struct DeviceArray {
  T* ptr = nullptr;
  size_t n = 0;
  DeviceArray() = default;
  DeviceArray(const DeviceArray&) = delete;
  DeviceArray& operator=(const DeviceArray&) = delete;
  ~DeviceArray() { release(); }
  void release() {
    if (ptr) cudaFree(ptr);
    ptr = nullptr;
    n = 0;
  }
  void alloc(size_t count) {
    release();
    n = count;
    if (count == 0) return;
    if (cudaMalloc(&ptr, count * sizeof(T)) != cudaSuccess) {
      cudaGetLastError();
      ptr = nullptr;
      throw Error(FX_E_NOMEM, "cudaMalloc of " + std::to_string(count * sizeof(T)) + " bytes failed");
    }
  }
  void upload(const T* h, size_t count) {
    alloc(count);
    if (count) FX_CUDA(cudaMemcpy(ptr, h, count * sizeof(T), cudaMemcpyHostToDevice));
  }
  void upload(const std::vector<T>& h) { upload(h.data(), h.size()); }
  void zero(cudaStream_t s = nullptr) {
    if (n) FX_CUDA(cudaMemsetAsync(ptr, 0, n * sizeof(T), s));
  }
  size_t bytes() const { return n * sizeof(T); }
};

inline int num_sms() {
  static int sms = [] {
    int dev = 0, v = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev);
    return v > 0 ? v : 148;
  }();
  return sms;
}

inline unsigned grid_for(int64_t n, int block) { return static_cast<unsigned>((n + block - 1) / block); }

}  // namespace fx
