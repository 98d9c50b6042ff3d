// Integer-ALU peak of the device, measured: the denominator of the search
// kernels' roofline.  Every thread runs 16 independent dependency chains of
// 32-bit LOP3 (ALU pipe) interleaved with IMAD (FMA pipe) over enough CTAs
// to fill every SM; the rate is lane-operations per second.
#include <cuda_runtime.h>

#include <algorithm>

#include "cuda_util.h"
#include "engine.h"

namespace simba {

constexpr int kPeakChains = 16;

__global__ void __launch_bounds__(256) int_peak_kernel(unsigned* out, int iters, unsigned seed) {
  unsigned x[kPeakChains];
#pragma unroll
  for (int i = 0; i < kPeakChains; ++i) x[i] = seed * (threadIdx.x + 1) + i * 0x9E3779B9u;
  const unsigned a = seed ^ 0x5bd1e995u, b = seed + 0x1b873593u;
  for (int it = 0; it < iters; ++it) {
#pragma unroll
    for (int i = 0; i < kPeakChains; i += 2) {
      asm volatile("lop3.b32 %0, %0, %1, %2, 0x96;" : "+r"(x[i]) : "r"(a), "r"(b));
      asm volatile("mad.lo.u32 %0, %0, %1, %2;" : "+r"(x[i + 1]) : "r"(a), "r"(b));
    }
  }
  unsigned acc = 0;
#pragma unroll
  for (int i = 0; i < kPeakChains; ++i) acc ^= x[i];
  if (acc == 0x12345678u) out[blockIdx.x] = acc;  // keeps the chains live
}

// Same shape with LOP3 only: the ALU pipe alone (the search kernels'
// masked compares are all ALU-pipe instructions).
__global__ void __launch_bounds__(256) alu_peak_kernel(unsigned* out, int iters, unsigned seed) {
  unsigned x[kPeakChains];
#pragma unroll
  for (int i = 0; i < kPeakChains; ++i) x[i] = seed * (threadIdx.x + 1) + i * 0x9E3779B9u;
  const unsigned a = seed ^ 0x5bd1e995u, b = seed + 0x1b873593u;
  for (int it = 0; it < iters; ++it) {
#pragma unroll
    for (int i = 0; i < kPeakChains; ++i)
      asm volatile("lop3.b32 %0, %0, %1, %2, 0x96;" : "+r"(x[i]) : "r"(a), "r"(b));
  }
  unsigned acc = 0;
#pragma unroll
  for (int i = 0; i < kPeakChains; ++i) acc ^= x[i];
  if (acc == 0x12345678u) out[blockIdx.x] = acc;
}

static int time_peak(int device, bool alu_only, double* lane_ops_per_s);

int measure_int_peak(int device, double* lane_ops_per_s) { return time_peak(device, false, lane_ops_per_s); }
int measure_alu_peak(int device, double* lane_ops_per_s) { return time_peak(device, true, lane_ops_per_s); }

static int time_peak(int device, bool alu_only, double* lane_ops_per_s) {
  *lane_ops_per_s = 0;
  SB_CUDA(cudaSetDevice(device));
  int sms = 0;
  SB_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
  int occ = 1;
  SB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, alu_only ? alu_peak_kernel : int_peak_kernel,
                                                        256, 0));
  const int grid = sms * std::max(occ, 1);
  DevBuf out;
  SB_CUDA(out.reserve(sizeof(unsigned) * grid));
  cudaEvent_t e0, e1;
  SB_CUDA(cudaEventCreate(&e0));
  SB_CUDA(cudaEventCreate(&e1));
  const int iters = 4096;
  auto kern = alu_only ? alu_peak_kernel : int_peak_kernel;
  kern<<<grid, 256>>>(out.as<unsigned>(), iters, 1u);  // warm-up
  SB_CUDA(cudaGetLastError());
  float best = 1e30f;
  for (int rep = 0; rep < 5; ++rep) {
    SB_CUDA(cudaEventRecord(e0));
    kern<<<grid, 256>>>(out.as<unsigned>(), iters, 2u + rep);
    SB_CUDA(cudaEventRecord(e1));
    SB_CUDA(cudaEventSynchronize(e1));
    float ms = 0;
    SB_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    best = std::min(best, ms);
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  const double ops = (double)grid * 256 * iters * kPeakChains;
  *lane_ops_per_s = ops / (best * 1e-3);
  return 0;
}

}  // namespace simba
