// Plain search in the extended grammar (ext_grammar.h): ~ & | ^ << >> neg
// + - * / %.  The reference declares these operators but runs none of the
// four new ones (vfb/src/full-cache.cu:460-472 comments them out of the
// enumeration; evaluateRPN, simba/src/mba.cuh:71-131, has no caller), so
// this path is an option of simba_solve (simba_options.grammar = 1).
//
// Engine: one thread per rank, the reference's per-candidate algorithm
// (simba/src/nocache.cu:85-107) -- unrank, then evaluate sample by sample
// with an exit at the first mismatch -- with the twelve-operator count table
// and the samples staged in shared memory, a grid-stride loop over the
// ranks of a whole size (no gridDim overflow), and the minimum matching rank
// by atomicMin.  Ranks of a size are ordered by operator block, so that
// minimum lies in the first block with a match, which is the reference's
// stop rule.  The spine engine's inversion and value tables are not built
// for the new operators (a shift amount, divisor or modulus on the spine
// has no inverse under a mask); this path is for completeness of the
// grammar, not for speed.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstring>
#include <vector>

#include "cuda_util.h"
#include "engine.h"
#include "ext_grammar.h"

namespace simba {

namespace {

constexpr int kExtThreads = 256;

template <class W>
struct ExtParams {
  const unsigned long long* counts;  // (kMaxSize + 1) x kExtCols
  const W* in;                       // S x K sample-major
  const W* out;                      // S
  unsigned long long* scal;          // [0] best rank, [1] evaluated, [2] budget flag, [3] start ns
  unsigned long long lo, hi;         // ranks of the size
  unsigned long long budget_ns;
  int size, S, K;
};

template <class W>
__device__ __forceinline__ W ext_eval_sample(const char* post, int len, const W* row) {
  W st[kMaxSize + 1];
  int sp = -1;
  for (int j = 0; j < len; ++j) {
    const char ch = post[j];
    const int code = ext_char_code(ch);
    if (code < 0) {
      st[++sp] = row[ch - '0'];
    } else if (code == OP_NOT || code == OP_NEG) {
      st[sp] = ext_apply<W>(code, W(0), st[sp]);
    } else {
      const W r = st[sp--];
      st[sp] = ext_apply<W>(code, st[sp], r);
    }
  }
  return st[0];
}

__global__ void ext_stamp_kernel(unsigned long long* t) {
  unsigned long long v;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(v));
  *t = v;
}

template <class W>
__global__ void __launch_bounds__(kExtThreads) ext_naive_kernel(ExtParams<W> p) {
  extern __shared__ __align__(16) unsigned char ext_smem[];
  unsigned long long(*counts)[kExtCols] = reinterpret_cast<unsigned long long(*)[kExtCols]>(ext_smem);
  W* s_in = reinterpret_cast<W*>(ext_smem + sizeof(unsigned long long) * (kMaxSize + 1) * kExtCols);
  W* s_out = s_in + p.S * p.K;
  for (int i = threadIdx.x; i < (kMaxSize + 1) * kExtCols; i += blockDim.x)
    (&counts[0][0])[i] = p.counts[i];
  for (int i = threadIdx.x; i < p.S * p.K; i += blockDim.x) s_in[i] = p.in[i];
  for (int i = threadIdx.x; i < p.S; i += blockDim.x) s_out[i] = p.out[i];
  __syncthreads();
  const unsigned long long stride = (unsigned long long)gridDim.x * blockDim.x;
  unsigned long long evaluated = 0;
  char post[kMaxSize + 1];
  unsigned it = 0;
  for (unsigned long long r = p.lo + (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; r < p.hi;
       r += stride, ++it) {
    // ranks only grow along a thread's loop: past the best match, stop
    if (r > *(volatile unsigned long long*)&p.scal[0]) break;
    if ((it & 1023) == 1023 && p.budget_ns && globaltimer_ns() - p.scal[3] > p.budget_ns) {
      atomicOr(&p.scal[2], 1ULL);
      break;
    }
    ext_unrank(r, p.size, (const uint64_t(*)[kExtCols])counts, post);
    ++evaluated;
    bool ok = true;
    for (int i = 0; i < p.S && ok; ++i) ok = ext_eval_sample<W>(post, p.size, s_in + i * p.K) == s_out[i];
    if (ok) atomicMin(&p.scal[0], r);
  }
  if (evaluated) atomicAdd(&p.scal[1], evaluated);
}

template <class W>
bool ext_host_check(const std::string& post, const HostInstance& h) {
  std::vector<W> st(post.size() + 1);
  for (int i = 0; i < h.S; ++i) {
    int sp = -1;
    for (char ch : post) {
      const int code = ext_char_code(ch);
      if (code < 0) {
        const int t = ch - '0';
        if (t < 0 || t >= h.k) return false;
        st[++sp] = (W)h.in[(size_t)i * h.k + t];
      } else if (code == OP_NOT || code == OP_NEG) {
        if (sp < 0) return false;
        st[sp] = ext_apply<W>(code, W(0), st[sp]);
      } else {
        if (sp < 1) return false;
        const W r = st[sp--];
        st[sp] = ext_apply<W>(code, st[sp], r);
      }
    }
    if (sp != 0 || st[0] != (W)h.out[i]) return false;
  }
  return true;
}

template <class W>
int ext_typed(const HostInstance& h, int max_size, const EngineOptions& o, SolveOutcome* out) {
  *out = SolveOutcome();
  SB_CUDA(cudaSetDevice(o.device));
  cudaStream_t st = nullptr;
  bool own = false;
  if (o.stream) {
    st = reinterpret_cast<cudaStream_t>(o.stream);
  } else {
    SB_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    own = true;
  }
  struct Guard {
    cudaStream_t s;
    bool own;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    ~Guard() {
      if (e0) cudaEventDestroy(e0);
      if (e1) cudaEventDestroy(e1);
      if (own && s) cudaStreamDestroy(s);
    }
  } g{st, own};
  ExtCountTable ct;
  int ms = std::min(max_size, kMaxSize);
  while (ms > 1 && !build_ext_count_table(ms, h.k, &ct)) --ms;
  const int first = o.size_range ? 1 : 2;
  const int last = o.size_range ? max_size : max_size - 1;
  if (last > ms) {
    set_last_error("candidate counts exceed 64 bits at this size");
    return SIMBA_E_OVERFLOW;
  }
  if (first == 1) {  // size 1: the terminals, checked on the host
    for (int v = 0; v < h.k; ++v) {
      out->candidates++;
      out->per_size[1]++;
      bool eq = true;
      for (int i = 0; i < h.S && eq; ++i) eq = (W)h.in[(size_t)i * h.k + v] == (W)h.out[i];
      if (eq) {
        out->status = SIMBA_OK;
        out->size = 1;
        out->op = 8;
        out->rank = (uint64_t)v;
        out->postfix = std::string(1, (char)('0' + v));
        out->max_size_searched = 1;
        return SIMBA_OK;
      }
    }
  }
  std::vector<W> win((size_t)h.S * h.k), wout(h.S);
  for (size_t i = 0; i < win.size(); ++i) win[i] = (W)h.in[i];
  for (int i = 0; i < h.S; ++i) wout[i] = (W)h.out[i];
  DevBuf d_counts, d_in, d_out, d_scal;
  SB_CUDA(d_counts.reserve(sizeof(ct.n)));
  SB_CUDA(d_in.reserve(win.size() * sizeof(W)));
  SB_CUDA(d_out.reserve(wout.size() * sizeof(W)));
  SB_CUDA(d_scal.reserve(4 * sizeof(unsigned long long)));
  SB_CUDA(cudaMemcpyAsync(d_counts.p, ct.n, sizeof(ct.n), cudaMemcpyHostToDevice, st));
  SB_CUDA(cudaMemcpyAsync(d_in.p, win.data(), win.size() * sizeof(W), cudaMemcpyHostToDevice, st));
  SB_CUDA(cudaMemcpyAsync(d_out.p, wout.data(), wout.size() * sizeof(W), cudaMemcpyHostToDevice, st));
  const size_t smem = sizeof(ct.n) + (size_t)(h.S * h.k + h.S) * sizeof(W);
  SB_CUDA(cudaFuncSetAttribute(ext_naive_kernel<W>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  int sms = 0, occ = 1;
  SB_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, o.device));
  SB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, ext_naive_kernel<W>, kExtThreads, smem));
  const int grid = sms * std::max(occ, 1);
  SB_CUDA(cudaEventCreate(&g.e0));
  SB_CUDA(cudaEventCreate(&g.e1));
  SB_CUDA(cudaEventRecord(g.e0, st));
  ExtParams<W> p;
  p.counts = d_counts.as<unsigned long long>();
  p.in = d_in.as<W>();
  p.out = d_out.as<W>();
  p.scal = d_scal.as<unsigned long long>();
  p.S = h.S;
  p.K = h.k;
  p.budget_ns = o.budget_s > 0 ? (unsigned long long)(o.budget_s * 1e9) : 0;
  ext_stamp_kernel<<<1, 1, 0, st>>>(p.scal + 3);
  out->launches++;
  const auto t0 = std::chrono::steady_clock::now();
  for (int s = std::max(first, 2); s <= last; ++s) {
    if (o.budget_s > 0 &&
        std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count() > o.budget_s) {
      out->status = SIMBA_BUDGET;
      break;
    }
    const unsigned long long init[3] = {~0ULL, 0, 0};
    SB_CUDA(cudaMemcpyAsync(p.scal, init, sizeof(init), cudaMemcpyHostToDevice, st));
    p.size = s;
    p.lo = 0;
    p.hi = ct.n[s][kExtOps];
    ext_naive_kernel<W><<<grid, kExtThreads, smem, st>>>(p);
    out->launches++;
    SB_CUDA(cudaGetLastError());
    unsigned long long hs[3];
    SB_CUDA(cudaMemcpyAsync(hs, p.scal, sizeof(hs), cudaMemcpyDeviceToHost, st));
    SB_CUDA(cudaStreamSynchronize(st));
    out->evaluated += hs[1];
    out->max_size_searched = s;
    if (hs[2]) {
      out->status = SIMBA_BUDGET;
      break;
    }
    if (hs[0] != ~0ULL) {
      uint64_t off = 0;
      int e = 0;
      while (e < kExtOps - 1 && hs[0] >= off + ct.n[s][e]) off += ct.n[s][e++];
      out->per_size[s] = off + ct.n[s][e];
      out->candidates += out->per_size[s];
      char buf[kMaxSize + 1];
      ext_unrank(hs[0], s, ct.n, buf);
      buf[s] = 0;
      out->postfix = buf;
      out->size = s;
      out->op = ext_code(e);
      out->rank = hs[0];
      if (!ext_host_check<W>(out->postfix, h)) {
        set_last_error("device match failed the host re-check");
        return SIMBA_E_INTERNAL;
      }
      out->status = SIMBA_OK;
      break;
    }
    out->per_size[s] = ct.n[s][kExtOps];
    out->candidates += ct.n[s][kExtOps];
  }
  SB_CUDA(cudaEventRecord(g.e1, st));
  SB_CUDA(cudaEventSynchronize(g.e1));
  float ms_dev = 0;
  SB_CUDA(cudaEventElapsedTime(&ms_dev, g.e0, g.e1));
  out->device_ms = ms_dev;
  out->kernel_ms = ms_dev;
  out->nested_ms = ms_dev;
  out->nested_candidates = out->evaluated;
  return out->status;
}

}  // namespace

int ext_solve(const HostInstance& h, int max_size, const EngineOptions& o, SolveOutcome* out) {
  if (h.k > kExtMaxTerms) {
    set_last_error("the extended grammar takes at most 10 terminals");
    return SIMBA_E_ARG;
  }
  if (h.bits == 64) return ext_typed<uint64_t>(h, max_size, o, out);
  return ext_typed<uint32_t>(h, max_size, o, out);
}

bool ext_check_host(const std::string& postfix, const HostInstance& h) {
  if (h.bits == 64) return ext_host_check<uint64_t>(postfix, h);
  return ext_host_check<uint32_t>(postfix, h);
}

namespace {

// Whole-vector evaluation: every node is computed on all samples, so that
// / and % can take the dividend vector when the divisor vector has a zero.
template <class W>
bool ext_vector_check_t(const std::string& post, const HostInstance& h) {
  std::vector<std::vector<W>> st;
  for (char ch : post) {
    const int code = ext_char_code(ch);
    if (code < 0) {
      const int t = ch - '0';
      if (t < 0 || t >= h.k) return false;
      std::vector<W> v(h.S);
      for (int i = 0; i < h.S; ++i) v[i] = (W)h.in[(size_t)i * h.k + t];
      st.push_back(std::move(v));
    } else if (code == OP_NOT || code == OP_NEG) {
      if (st.empty()) return false;
      for (auto& x : st.back()) x = ext_apply<W>(code, W(0), x);
    } else {
      if (st.size() < 2) return false;
      std::vector<W> r = std::move(st.back());
      st.pop_back();
      std::vector<W>& l = st.back();
      bool zero = false;
      if (code == OP_DIV || code == OP_MOD)
        for (W x : r) zero = zero || x == W(0);
      if (!zero)
        for (int i = 0; i < h.S; ++i) l[i] = ext_apply<W>(code, l[i], r[i]);
    }
  }
  if (st.size() != 1) return false;
  for (int i = 0; i < h.S; ++i)
    if (st[0][i] != (W)h.out[i]) return false;
  return true;
}

}  // namespace

bool ext_vector_check(const std::string& postfix, const HostInstance& h) {
  if (h.bits == 64) return ext_vector_check_t<uint64_t>(postfix, h);
  return ext_vector_check_t<uint32_t>(postfix, h);
}

}  // namespace simba
