// Small CUDA helpers: error propagation without exceptions across the C ABI,
// RAII device buffers, and the %globaltimer clock used for in-kernel budgets.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <string>

namespace simba {

void set_last_error(const std::string& e);

#define SB_CUDA(call)                                                              \
  do {                                                                             \
    cudaError_t err__ = (call);                                                    \
    if (err__ != cudaSuccess) {                                                    \
      ::simba::set_last_error(std::string(#call) + ": " + cudaGetErrorString(err__)); \
      return err__ == cudaErrorMemoryAllocation ? SIMBA_E_NOMEM : SIMBA_E_CUDA;    \
    }                                                                              \
  } while (0)

// Device allocation owned by the host object; freed on destruction.
struct DevBuf {
  void* p = nullptr;
  size_t bytes = 0;
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  ~DevBuf() { release(); }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    bytes = 0;
  }
  // Grows (never shrinks) to at least n bytes; contents are not preserved.
  cudaError_t reserve(size_t n) {
    if (n <= bytes) return cudaSuccess;
    release();
    cudaError_t e = cudaMalloc(&p, n);
    if (e == cudaSuccess) bytes = n;
    else p = nullptr;
    return e;
  }
  template <class T>
  T* as() const { return static_cast<T*>(p); }
};

#if defined(__CUDACC__)
__device__ __forceinline__ unsigned long long globaltimer_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
#endif

}  // namespace simba
