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

// Process-wide cache of device allocations (capi.cpp): a buffer released by
// one call is handed to the next call that needs one of about its size, so
// that repeated searches do not pay cudaMalloc / cudaFree for gigabytes of
// value tables every time.  Blocks are cached only after the work that used
// them has been synchronised (every engine synchronises before it releases
// its buffers); the cache is capped (SIMBA_DEVICE_CACHE_BYTES, default
// 32 GiB, 0 = off) and emptied by simba_release_device_cache and, for a
// device, whenever a cudaMalloc there runs out of memory.
cudaError_t pool_alloc(void** p, size_t n, size_t* got);
void pool_free(void* p, size_t bytes);
size_t pool_cached_bytes(int device);  // bytes the cache holds on a device

// Device allocation owned by the host object; released on destruction.
struct DevBuf {
  void* p = nullptr;
  size_t bytes = 0;
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  ~DevBuf() { release(); }
  void release() {
    if (p) pool_free(p, bytes);
    p = nullptr;
    bytes = 0;
  }
  // Grows (never shrinks) to at least n bytes; contents are not preserved.
  cudaError_t reserve(size_t n) {
    if (n <= bytes) return cudaSuccess;
    release();
    size_t got = 0;
    cudaError_t e = pool_alloc(&p, n, &got);
    if (e == cudaSuccess) bytes = got;
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
