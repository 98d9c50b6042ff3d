// Learned proposal for the guided search: a 3-layer MLP over bit-level
// features of an instance's samples, predicting the shape class of the
// minimal expression (root operator x root split / unary-chain length,
// 8 x 8 = 64 classes).  No counterpart in the reference.
//
//   features  X[b] = 8192 values in {-1, 0, +1}: for the first 64 samples
//             (repeated cyclically when an instance has fewer) 128 features
//             each: the 64 bits of the output word, then the low 16 bits of
//             (output XOR variable j) for j = 0..3 (0 when the variable does
//             not exist).
//   network   Z1 = X W1 + b1, H1 = relu(Z1), Z2 = H1 W2 + b2, H2 = relu(Z2),
//             Z3 = H2 W3 + b3, p = softmax(Z3), loss = mean cross-entropy.
//   GEMMs     BF16 operands, FP32 accumulation, tcgen05.mma on the
//             5th-generation tensor cores with the accumulator in TMEM
//             (128x128 CTA tiles, two-stage cp.async pipeline, gemm_tc_kernel).
//   training  hand-written backward pass and Adam (FP32 master weights,
//             BF16 copies feed the GEMMs).
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <random>
#include <vector>

#include "cuda_util.h"
#include "engine.h"

namespace simba {

typedef __nv_bfloat16 bf16;

constexpr int kFeat = 8192, kHid = 512, kCls = 64, kFeatSamples = 64, kFeatPerSample = 128;

// ---------------------------------------------------------------- features

struct FeatInst {
  unsigned long long in_off, out_off;  // word offsets into the packed arrays
  int S, K;
};

__global__ void features_kernel(const unsigned long long* in, const unsigned long long* out,
                                const FeatInst* fi, int n, bf16* X) {
  const long long total = (long long)n * kFeat;
  for (long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x; g < total;
       g += (long long)gridDim.x * blockDim.x) {
    const int b = (int)(g / kFeat), f = (int)(g % kFeat);
    const FeatInst d = fi[b];
    const int smp = (f / kFeatPerSample) % d.S;
    const int j = f % kFeatPerSample;
    const unsigned long long y = out[d.out_off + smp];
    float v;
    if (j < 64) {
      v = ((y >> j) & 1ULL) ? 1.f : -1.f;
    } else {
      const int var = (j - 64) / 16, bit = (j - 64) % 16;
      if (var < d.K) {
        const unsigned long long x = in[d.in_off + (unsigned long long)smp * d.K + var];
        v = (((y ^ x) >> bit) & 1ULL) ? 1.f : -1.f;
      } else {
        v = 0.f;
      }
    }
    X[g] = __float2bfloat16(v);
  }
}

// ---------------------------------------------------------------- GEMM

// C[M x N] = A[M x K] * Bt[N x K]^T (+ bias[n]) on the 5th-generation tensor
// cores: tcgen05.mma (kind::f16, BF16 operands, FP32 accumulation in TMEM),
// one elected thread issuing, the accumulator read back with tcgen05.ld.
//   * One CTA (4 warps) per 128 x 128 tile of C; K in steps of 64.
//   * Operands are staged in shared memory in the canonical K-major layout
//     without swizzle: 8 x 8 core matrices of 128 contiguous bytes (8 rows of
//     16 bytes), core matrix (row group i, k group j) at (8 i + j) * 128, so
//     the leading (K) byte offset is 128 and the stride (M/N) byte offset is
//     1024; each MMA covers K = 16, i.e. two k groups (+256 bytes).
//   * Two stages: the asynchronous copies (cp.async, zero-filled past the
//     matrix edges) of step k+1 run while the MMAs of step k do; a stage is
//     refilled only after tcgen05.commit has signalled (mbarrier) that the
//     MMAs reading it are done.  Every wait is bounded and reports through
//     *err.
// Both operands are K-major (row stride lda / ldb elements, multiples of 8,
// 16-byte aligned rows); the caller transposes where needed.
constexpr int kTcM = 128, kTcN = 128, kTcK = 64, kTcStages = 2;
constexpr int kTcTileA = kTcM * kTcK * 2, kTcTileB = kTcN * kTcK * 2;
constexpr size_t kTcSmem = kTcStages * (kTcTileA + kTcTileB) + 1024;  // 3 CTAs (384 TMEM columns) per SM

__device__ __forceinline__ uint64_t tc_desc(uint32_t saddr) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFF);   // start address
  d |= (uint64_t)(128 >> 4) << 16;          // leading (K) byte offset
  d |= (uint64_t)(1024 >> 4) << 32;         // stride (M/N) byte offset
  d |= 1ull << 46;                          // descriptor version of sm_100
  return d;                                 // base offset 0, no swizzle
}

__device__ __forceinline__ bool tc_wait(uint32_t mbar, uint32_t phase) {
  for (int i = 0; i < (1 << 22); ++i) {
    uint32_t done;
    asm volatile("{\n.reg .pred p;\nmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
                 "selp.u32 %0, 1, 0, p;\n}\n" : "=r"(done) : "r"(mbar), "r"(phase) : "memory");
    if (done) return true;
  }
  return false;
}

// rows [r0, r0 + rows) x k [k0, k0 + 64) of a K-major matrix into the
// canonical tile at shared address `tile`, by 16-byte asynchronous copies;
// bytes past row nrows_total or column K are zero-filled
__device__ __forceinline__ void tc_stage(uint32_t tile, const bf16* G, int ld, int r0, int nrows_total,
                                         int rows, int k0, int K) {
  for (int c = threadIdx.x; c < rows * 8; c += blockDim.x) {
    const int row = c >> 3, kc = c & 7;
    const int gr = r0 + row, gk = k0 + kc * 8;
    const bf16* src = G;
    int bytes = 0;
    if (gr < nrows_total && gk < K) {
      src = G + (size_t)gr * ld + gk;
      bytes = (K - gk < 8 ? K - gk : 8) * 2;
    }
    const uint32_t dst = tile + (uint32_t)(((row >> 3) * 8 + kc) * 128 + (row & 7) * 16);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" :: "r"(dst), "l"(src), "r"(bytes)
                 : "memory");
  }
}

__global__ void __launch_bounds__(128) gemm_tc_kernel(int M, int N, int K, const bf16* A, int lda,
                                                      const bf16* Bt, int ldb, float* C, int ldc,
                                                      const float* bias, int* err) {
  extern __shared__ __align__(1024) uint8_t tc_smem[];
  __shared__ __align__(8) uint64_t mbar[kTcStages];
  __shared__ uint32_t tmem_base;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t base = ((uint32_t)__cvta_generic_to_shared(tc_smem) + 1023u) & ~1023u;
  uint32_t sA[kTcStages], sB[kTcStages], mb[kTcStages];
#pragma unroll
  for (int s = 0; s < kTcStages; ++s) {
    sA[s] = base + (uint32_t)(s * (kTcTileA + kTcTileB));
    sB[s] = sA[s] + (uint32_t)kTcTileA;
    mb[s] = (uint32_t)__cvta_generic_to_shared(&mbar[s]);
  }
  if (warp == 0) {
    const uint32_t dst = (uint32_t)__cvta_generic_to_shared(&tmem_base);
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 128;" :: "r"(dst));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (threadIdx.x == 0) {
#pragma unroll
    for (int s = 0; s < kTcStages; ++s) asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" :: "r"(mb[s]));
    asm volatile("fence.mbarrier_init.release.cluster;");
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;");
  const uint32_t tmem = tmem_base;
  const int m0 = blockIdx.y * kTcM, n0 = blockIdx.x * kTcN;
  // kind::f16 instruction descriptor: FP32 D, BF16 A and B, both K-major, N, M
  const uint32_t idesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(kTcN >> 3) << 17) |
                         ((uint32_t)(kTcM >> 4) << 24);
  const int nk = (K + kTcK - 1) / kTcK;
  uint32_t ph[kTcStages] = {0u, 0u};
  bool ok = true;
  tc_stage(sA[0], A, lda, m0, M, kTcM, 0, K);
  tc_stage(sB[0], Bt, ldb, n0, N, kTcN, 0, K);
  asm volatile("cp.async.commit_group;" ::: "memory");
  for (int k = 0; k < nk && ok; ++k) {
    const int s = k & 1;
    if (k + 1 < nk) {
      if (k >= 1) {  // stage s^1 was read by the MMAs of step k-1
        // one verdict for the whole CTA, so that every thread leaves together
        if (__syncthreads_or(tc_wait(mb[s ^ 1], ph[s ^ 1]) ? 0 : 1)) {
          ok = false;
          if (threadIdx.x == 0) atomicOr(err, 1);
          break;
        }
        ph[s ^ 1] ^= 1u;
      }
      tc_stage(sA[s ^ 1], A, lda, m0, M, kTcM, (k + 1) * kTcK, K);
      tc_stage(sB[s ^ 1], Bt, ldb, n0, N, kTcN, (k + 1) * kTcK, K);
      asm volatile("cp.async.commit_group;" ::: "memory");
      asm volatile("cp.async.wait_group 1;" ::: "memory");
    } else {
      asm volatile("cp.async.wait_group 0;" ::: "memory");
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // copies -> tensor core
    __syncthreads();
    if (threadIdx.x == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;");
#pragma unroll
      for (int kk = 0; kk < kTcK / 16; ++kk) {
        const uint64_t ad = tc_desc(sA[s] + kk * 256), bd = tc_desc(sB[s] + kk * 256);
        const uint32_t accumulate = (k > 0 || kk > 0) ? 1u : 0u;
        asm volatile("{\n.reg .pred p;\nsetp.ne.b32 p, %4, 0;\n"
                     "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n"
                     :: "r"(tmem), "l"(ad), "l"(bd), "r"(idesc), "r"(accumulate));
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                   :: "r"(mb[s]) : "memory");
    }
    __syncwarp();
  }
  asm volatile("cp.async.wait_group 0;" ::: "memory");
  // the last commit covers every MMA issued before it
  if (ok && __syncthreads_or(tc_wait(mb[(nk - 1) & 1], ph[(nk - 1) & 1]) ? 0 : 1)) {
    ok = false;
    if (threadIdx.x == 0) atomicOr(err, 1);
  }
  asm volatile("tcgen05.fence::after_thread_sync;");
  if (ok) {  // warp w owns TMEM lanes (rows) 32 w .. 32 w + 31
    const int row = m0 + warp * 32 + lane;
#pragma unroll
    for (int j0 = 0; j0 < kTcN; j0 += 16) {
      uint32_t r[16];
      const uint32_t ta = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)j0;
      asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
                   : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
                     "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
                     "=r"(r[14]), "=r"(r[15])
                   : "r"(ta));
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
      if (row < M) {
#pragma unroll
        for (int j = 0; j < 16; ++j) {
          const int col = n0 + j0 + j;
          if (col < N) C[(size_t)row * ldc + col] = __uint_as_float(r[j]) + (bias ? bias[col] : 0.f);
        }
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 128;" :: "r"(tmem));
}

// out[c][r] = in[r][c] for a rows x cols BF16 matrix; out rows are ldo
// elements (>= rows, the tail zero-filled).
__global__ void transpose_bf16_kernel(const bf16* in, int rows, int cols, int ldi, bf16* out, int ldo) {
  __shared__ bf16 t[32][33];
  const int r0 = blockIdx.y * 32, c0 = blockIdx.x * 32;
  for (int y = threadIdx.y; y < 32; y += blockDim.y) {
    const int r = r0 + y, c = c0 + threadIdx.x;
    t[y][threadIdx.x] = (r < rows && c < cols) ? in[(size_t)r * ldi + c] : __float2bfloat16(0.f);
  }
  __syncthreads();
  for (int y = threadIdx.y; y < 32; y += blockDim.y) {
    const int c = c0 + y, r = r0 + threadIdx.x;
    if (c < cols && r < ldo) out[(size_t)c * ldo + r] = t[threadIdx.x][y];
  }
}

// ---------------------------------------------------------------- elementwise

__global__ void relu_bf16_kernel(const float* Z, bf16* H, long long n) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    H[i] = __float2bfloat16(fmaxf(Z[i], 0.f));
}

// dZ = dH * (Z > 0), as BF16 for the next GEMMs
__global__ void relu_back_kernel(const float* dH, const float* Z, bf16* dZ, long long n) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    dZ[i] = __float2bfloat16(Z[i] > 0.f ? dH[i] : 0.f);
}

// One warp per row: softmax of the 64 logits, probabilities out, and (with
// labels) the cross-entropy summed into *loss and dZ = (p - onehot) / B.
__global__ void softmax_ce_kernel(const float* Z, const int* labels, int B, float* P, bf16* dZ,
                                  float* loss) {
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (warp >= B) return;
  const float* z = Z + (long long)warp * kCls;
  float a = z[lane], b = z[lane + 32];
  float mx = fmaxf(a, b);
  for (int o = 16; o; o >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
  float ea = expf(a - mx), eb = expf(b - mx);
  float s = ea + eb;
  for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  const float pa = ea / s, pb = eb / s;
  if (P) {
    P[(long long)warp * kCls + lane] = pa;
    P[(long long)warp * kCls + lane + 32] = pb;
  }
  if (labels) {
    const int y = labels[warp];
    if (lane == (y & 31)) {
      const float py = y < 32 ? pa : pb;
      atomicAdd(loss, -logf(fmaxf(py, 1e-30f)));
    }
    const float inv = 1.f / (float)B;
    dZ[(long long)warp * kCls + lane] = __float2bfloat16((pa - (lane == y ? 1.f : 0.f)) * inv);
    dZ[(long long)warp * kCls + lane + 32] = __float2bfloat16((pb - (lane + 32 == y ? 1.f : 0.f)) * inv);
  }
}

// column sums of a B x N BF16 matrix into FP32 (bias gradients)
__global__ void colsum_kernel(const bf16* D, int B, int N, float* out) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= N) return;
  float s = 0.f;
  for (int r = 0; r < B; ++r) s += __bfloat162float(D[(long long)r * N + c]);
  out[c] = s;
}

// Adam (Kingma & Ba 2015) on FP32 master weights; refreshes the BF16 copy.
__global__ void adam_kernel(float* w, const float* g, float* m, float* v, bf16* wb, long long n,
                            float lr, float b1, float b2, float eps, float c1, float c2) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    const float wi = w[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    w[i] = wi;
    if (wb) wb[i] = __float2bfloat16(wi);
  }
}

__global__ void to_bf16_kernel(const float* a, bf16* b, long long n) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    b[i] = __float2bfloat16(a[i]);
}

// ---------------------------------------------------------------- model

static const long long kSizes[6] = {(long long)kFeat * kHid, kHid, (long long)kHid * kHid, kHid,
                                    (long long)kHid * kCls, kCls};

long long mlp_param_count() {
  long long s = 0;
  for (long long x : kSizes) s += x;
  return s;
}

class Mlp {
 public:
  explicit Mlp(int device) : dev_(device) {}

  // C = op(A) op(B) (+ bias) through gemm_tc_kernel: op(A)(m,k) = TA ?
  // A[k*lda + m] : A[m*lda + k], op(B)(k,n) = TB ? B[n*ldb + k] : B[k*ldb + n].
  // The tensor-core kernel takes K-major operands, so an operand stored the
  // other way is transposed into scratch first (rows padded to 8 elements,
  // zero-filled).  Errors are kept in gemm_rc_ until the caller checks.
  template <bool TA, bool TB>
  void gemm(int M, int N, int K, const bf16* A, int lda, const bf16* B, int ldb, float* C, int ldc,
            const float* bias) {
    if (gemm_rc_) return;
    const int Kp = (K + 7) / 8 * 8;
    const dim3 tb(32, 8);
    if (TA) {  // A is stored K x M: make it M x Kp
      if ((gemm_rc_ = ta_.reserve((size_t)M * Kp * 2) == cudaSuccess ? 0 : SIMBA_E_NOMEM)) return;
      transpose_bf16_kernel<<<dim3((M + 31) / 32, (Kp + 31) / 32), tb, 0, st_>>>(A, K, M, lda, ta_.as<bf16>(), Kp);
      A = ta_.as<bf16>();
      lda = Kp;
    }
    if (!TB) {  // B is stored K x N: make it N x Kp
      if ((gemm_rc_ = tb_.reserve((size_t)N * Kp * 2) == cudaSuccess ? 0 : SIMBA_E_NOMEM)) return;
      transpose_bf16_kernel<<<dim3((N + 31) / 32, (Kp + 31) / 32), tb, 0, st_>>>(B, K, N, ldb, tb_.as<bf16>(), Kp);
      B = tb_.as<bf16>();
      ldb = Kp;
    }
    gemm_tc_kernel<<<dim3((N + kTcN - 1) / kTcN, (M + kTcM - 1) / kTcM), 128, kTcSmem, st_>>>(
        M, N, K, A, lda, B, ldb, C, ldc, bias, err_.as<int>());
    if (cudaGetLastError() != cudaSuccess) gemm_rc_ = SIMBA_E_CUDA;
  }
  ~Mlp() {
    if (st_) cudaStreamDestroy(st_);
  }

  int init(unsigned long long seed) {
    SB_CUDA(cudaSetDevice(dev_));
    SB_CUDA(cudaStreamCreateWithFlags(&st_, cudaStreamNonBlocking));
    const long long P = mlp_param_count();
    SB_CUDA(w_.reserve(P * 4));
    SB_CUDA(g_.reserve(P * 4));
    SB_CUDA(m_.reserve(P * 4));
    SB_CUDA(v_.reserve(P * 4));
    SB_CUDA(wb_.reserve(P * 2));
    SB_CUDA(loss_.reserve(16));
    SB_CUDA(err_.reserve(16));
    SB_CUDA(cudaMemsetAsync(err_.p, 0, 16, st_));
    SB_CUDA(cudaFuncSetAttribute(gemm_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTcSmem));
    // He-uniform initialisation of the weights, zero biases
    std::vector<float> h(P, 0.f);
    std::mt19937_64 rng(seed);
    long long off = 0;
    const int fan_in[3] = {kFeat, kHid, kHid};
    for (int l = 0; l < 3; ++l) {
      const float lim = std::sqrt(6.f / (float)fan_in[l]);
      std::uniform_real_distribution<float> U(-lim, lim);
      for (long long i = 0; i < kSizes[2 * l]; ++i) h[off + i] = U(rng);
      off += kSizes[2 * l] + kSizes[2 * l + 1];
    }
    return set_params(h.data());
  }

  int set_params(const float* h) {
    const long long P = mlp_param_count();
    SB_CUDA(cudaMemcpy(w_.p, h, P * 4, cudaMemcpyHostToDevice));
    SB_CUDA(cudaMemset(m_.p, 0, P * 4));
    SB_CUDA(cudaMemset(v_.p, 0, P * 4));
    to_bf16_kernel<<<1024, 256, 0, st_>>>(w_.as<float>(), wb_.as<bf16>(), P);
    SB_CUDA(cudaGetLastError());
    SB_CUDA(cudaStreamSynchronize(st_));
    step_ = 0;
    return 0;
  }

  int get_params(float* h) {
    SB_CUDA(cudaMemcpy(h, w_.p, mlp_param_count() * 4, cudaMemcpyDeviceToHost));
    return 0;
  }

  // Features of n instances into Xd (device, n x 8192 BF16).
  int features(const std::vector<HostInstance>& hs, DevBuf* Xd) {
    const int n = (int)hs.size();
    std::vector<unsigned long long> in, out;
    std::vector<FeatInst> fi(n);
    for (int i = 0; i < n; ++i) {
      fi[i].in_off = in.size();
      fi[i].out_off = out.size();
      fi[i].S = hs[i].S;
      fi[i].K = hs[i].k;
      in.insert(in.end(), hs[i].in.begin(), hs[i].in.end());
      out.insert(out.end(), hs[i].out.begin(), hs[i].out.end());
    }
    SB_CUDA(fin_.reserve(std::max<size_t>(1, in.size()) * 8));
    SB_CUDA(fout_.reserve(std::max<size_t>(1, out.size()) * 8));
    SB_CUDA(finst_.reserve(std::max(1, n) * sizeof(FeatInst)));
    SB_CUDA(Xd->reserve((size_t)std::max(1, n) * kFeat * 2));
    SB_CUDA(cudaMemcpyAsync(fin_.p, in.data(), in.size() * 8, cudaMemcpyHostToDevice, st_));
    SB_CUDA(cudaMemcpyAsync(fout_.p, out.data(), out.size() * 8, cudaMemcpyHostToDevice, st_));
    SB_CUDA(cudaMemcpyAsync(finst_.p, fi.data(), n * sizeof(FeatInst), cudaMemcpyHostToDevice, st_));
    features_kernel<<<1024, 256, 0, st_>>>(fin_.as<unsigned long long>(), fout_.as<unsigned long long>(),
                                           finst_.as<FeatInst>(), n, Xd->as<bf16>());
    SB_CUDA(cudaGetLastError());
    SB_CUDA(cudaStreamSynchronize(st_));
    return 0;
  }

  // Forward (and with labels backward) for a batch already featurised in X_.
  int forward_backward(int B, const int* labels_host, bool backward, float* loss_out, float* probs) {
    SB_CUDA(z1_.reserve((size_t)B * kHid * 4));
    SB_CUDA(z2_.reserve((size_t)B * kHid * 4));
    SB_CUDA(z3_.reserve((size_t)B * kCls * 4));
    SB_CUDA(h1_.reserve((size_t)B * kHid * 2));
    SB_CUDA(h2_.reserve((size_t)B * kHid * 2));
    SB_CUDA(p_.reserve((size_t)B * kCls * 4));
    SB_CUDA(lab_.reserve((size_t)std::max(1, B) * 4));
    const bf16* W1 = wb_.as<bf16>();
    const bf16* W2 = W1 + kSizes[0] + kSizes[1];
    const bf16* W3 = W2 + kSizes[2] + kSizes[3];
    const float* b1 = w_.as<float>() + kSizes[0];
    const float* b2 = b1 + kSizes[1] + kSizes[2];
    const float* b3 = b2 + kSizes[3] + kSizes[4];
    const bf16* X = X_.as<bf16>();
    gemm<false, false>(B, kHid, kFeat, X, kFeat, W1, kHid, z1_.as<float>(), kHid, b1);
    relu_bf16_kernel<<<512, 256, 0, st_>>>(z1_.as<float>(), h1_.as<bf16>(), (long long)B * kHid);
    gemm<false, false>(B, kHid, kHid, h1_.as<bf16>(), kHid, W2, kHid, z2_.as<float>(), kHid, b2);
    relu_bf16_kernel<<<512, 256, 0, st_>>>(z2_.as<float>(), h2_.as<bf16>(), (long long)B * kHid);
    gemm<false, false>(B, kCls, kHid, h2_.as<bf16>(), kHid, W3, kCls, z3_.as<float>(), kCls, b3);
    SB_CUDA(cudaMemsetAsync(loss_.p, 0, 4, st_));
    int* lab = nullptr;
    if (labels_host) {
      SB_CUDA(cudaMemcpyAsync(lab_.p, labels_host, B * 4, cudaMemcpyHostToDevice, st_));
      lab = lab_.as<int>();
      SB_CUDA(dz3_.reserve((size_t)B * kCls * 2));
    }
    softmax_ce_kernel<<<(B * 32 + 255) / 256, 256, 0, st_>>>(z3_.as<float>(), lab, B, p_.as<float>(),
                                                            lab ? dz3_.as<bf16>() : nullptr,
                                                            loss_.as<float>());
    SB_CUDA(cudaGetLastError());
    if (backward && lab) {
      SB_CUDA(dh_.reserve((size_t)B * kHid * 4));
      SB_CUDA(dz2_.reserve((size_t)B * kHid * 2));
      SB_CUDA(dz1_.reserve((size_t)B * kHid * 2));
      float* G = g_.as<float>();
      float* gW1 = G;
      float* gb1 = gW1 + kSizes[0];
      float* gW2 = gb1 + kSizes[1];
      float* gb2 = gW2 + kSizes[2];
      float* gW3 = gb2 + kSizes[3];
      float* gb3 = gW3 + kSizes[4];
      // layer 3
      gemm<true, false>(kHid, kCls, B, h2_.as<bf16>(), kHid, dz3_.as<bf16>(), kCls, gW3, kCls, nullptr);
      colsum_kernel<<<1, kCls, 0, st_>>>(dz3_.as<bf16>(), B, kCls, gb3);
      gemm<false, true>(B, kHid, kCls, dz3_.as<bf16>(), kCls, W3, kCls, dh_.as<float>(), kHid, nullptr);
      relu_back_kernel<<<512, 256, 0, st_>>>(dh_.as<float>(), z2_.as<float>(), dz2_.as<bf16>(),
                                             (long long)B * kHid);
      // layer 2
      gemm<true, false>(kHid, kHid, B, h1_.as<bf16>(), kHid, dz2_.as<bf16>(), kHid, gW2, kHid, nullptr);
      colsum_kernel<<<(kHid + 255) / 256, 256, 0, st_>>>(dz2_.as<bf16>(), B, kHid, gb2);
      gemm<false, true>(B, kHid, kHid, dz2_.as<bf16>(), kHid, W2, kHid, dh_.as<float>(), kHid, nullptr);
      relu_back_kernel<<<512, 256, 0, st_>>>(dh_.as<float>(), z1_.as<float>(), dz1_.as<bf16>(),
                                             (long long)B * kHid);
      // layer 1
      gemm<true, false>(kFeat, kHid, B, X, kFeat, dz1_.as<bf16>(), kHid, gW1, kHid, nullptr);
      colsum_kernel<<<(kHid + 255) / 256, 256, 0, st_>>>(dz1_.as<bf16>(), B, kHid, gb1);
      SB_CUDA(cudaGetLastError());
    }
    SB_CUDA(cudaStreamSynchronize(st_));
    {
      int e = 0;
      SB_CUDA(cudaMemcpy(&e, err_.p, 4, cudaMemcpyDeviceToHost));
      const int rc = gemm_rc_;
      gemm_rc_ = 0;
      if (rc) {
        set_last_error("tensor-core GEMM launch failed");
        return rc;
      }
      if (e) {
        set_last_error("tensor-core GEMM: an MMA completion wait timed out");
        return SIMBA_E_INTERNAL;
      }
    }
    if (loss_out) {
      float l = 0;
      SB_CUDA(cudaMemcpy(&l, loss_.p, 4, cudaMemcpyDeviceToHost));
      *loss_out = l / (float)std::max(1, B);
    }
    if (probs) SB_CUDA(cudaMemcpy(probs, p_.p, (size_t)B * kCls * 4, cudaMemcpyDeviceToHost));
    return 0;
  }

  int train_step(const std::vector<HostInstance>& hs, const int* labels, float lr, float* loss) {
    int rc = features(hs, &X_);
    if (rc) return rc;
    rc = forward_backward((int)hs.size(), labels, true, loss, nullptr);
    if (rc) return rc;
    ++step_;
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.f - std::pow(b1, (float)step_), c2 = 1.f - std::pow(b2, (float)step_);
    // biases have no BF16 copy in use; refreshing the whole copy keeps one kernel
    adam_kernel<<<2048, 256, 0, st_>>>(w_.as<float>(), g_.as<float>(), m_.as<float>(), v_.as<float>(),
                                       wb_.as<bf16>(), mlp_param_count(), lr, b1, b2, 1e-8f, c1, c2);
    SB_CUDA(cudaGetLastError());
    SB_CUDA(cudaStreamSynchronize(st_));
    return 0;
  }

  // One Adam step with gradients computed elsewhere (data-parallel training:
  // the ranks' gradients, averaged by an all-reduce).
  int apply(const float* grads, float lr) {
    SB_CUDA(cudaMemcpyAsync(g_.p, grads, mlp_param_count() * 4, cudaMemcpyHostToDevice, st_));
    ++step_;
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.f - std::pow(b1, (float)step_), c2 = 1.f - std::pow(b2, (float)step_);
    adam_kernel<<<2048, 256, 0, st_>>>(w_.as<float>(), g_.as<float>(), m_.as<float>(), v_.as<float>(),
                                       wb_.as<bf16>(), mlp_param_count(), lr, b1, b2, 1e-8f, c1, c2);
    SB_CUDA(cudaGetLastError());
    SB_CUDA(cudaStreamSynchronize(st_));
    return 0;
  }

  int gradients(const std::vector<HostInstance>& hs, const int* labels, float* grads, float* loss) {
    int rc = features(hs, &X_);
    if (rc) return rc;
    rc = forward_backward((int)hs.size(), labels, true, loss, nullptr);
    if (rc) return rc;
    SB_CUDA(cudaMemcpy(grads, g_.p, mlp_param_count() * 4, cudaMemcpyDeviceToHost));
    return 0;
  }

  int predict(const std::vector<HostInstance>& hs, float* probs) {
    int rc = features(hs, &X_);
    if (rc) return rc;
    return forward_backward((int)hs.size(), nullptr, false, nullptr, probs);
  }

  int features_host(const std::vector<HostInstance>& hs, float* out) {
    int rc = features(hs, &X_);
    if (rc) return rc;
    std::vector<bf16> tmp((size_t)hs.size() * kFeat);
    SB_CUDA(cudaMemcpy(tmp.data(), X_.p, tmp.size() * 2, cudaMemcpyDeviceToHost));
    for (size_t i = 0; i < tmp.size(); ++i) out[i] = __bfloat162float(tmp[i]);
    return 0;
  }

 private:
  int dev_;
  cudaStream_t st_ = nullptr;
  long long step_ = 0;
  int gemm_rc_ = 0;
  DevBuf ta_, tb_, err_;
  DevBuf w_, g_, m_, v_, wb_, loss_, fin_, fout_, finst_, X_, z1_, z2_, z3_, h1_, h2_, p_, lab_, dz3_, dh_,
      dz2_, dz1_;
};

int mlp_create(int device, unsigned long long seed, Mlp** out) {
  *out = nullptr;
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n <= device || device < 0) {
    cudaGetLastError();
    set_last_error("no usable CUDA device");
    return SIMBA_E_NODEV;
  }
  Mlp* m = new Mlp(device);
  const int rc = m->init(seed);
  if (rc) {
    delete m;
    return rc;
  }
  *out = m;
  return 0;
}
void mlp_destroy(Mlp* m) { delete m; }
int mlp_train_step(Mlp* m, const std::vector<HostInstance>& hs, const int* labels, float lr, float* loss) {
  return m->train_step(hs, labels, lr, loss);
}
int mlp_gradients(Mlp* m, const std::vector<HostInstance>& hs, const int* labels, float* grads,
                  float* loss) {
  return m->gradients(hs, labels, grads, loss);
}
int mlp_apply(Mlp* m, const float* grads, float lr) { return m->apply(grads, lr); }
int mlp_predict(Mlp* m, const std::vector<HostInstance>& hs, float* probs) { return m->predict(hs, probs); }
int mlp_features(Mlp* m, const std::vector<HostInstance>& hs, float* out) { return m->features_host(hs, out); }
int mlp_get_params(Mlp* m, float* h) { return m->get_params(h); }
int mlp_set_params(Mlp* m, const float* h) { return m->set_params(h); }

}  // namespace simba
