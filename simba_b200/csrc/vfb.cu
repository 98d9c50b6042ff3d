// VFB on sm_100a: bottom-up enumeration of characteristic vectors with
// observational-equivalence dedup (vfb/src/full-cache.cu:568-774).
//
// Same search as the reference: sizes 2..max_len, operators in the order
// ~ & | ^ neg + - *, unary operators over the rows of size L-1, binary ones
// over rows(i) x rows(L-1-i) for 2i <= L-1 (Minus also tries the swapped
// pair), and stop after the operator block that produces the target.
//
// Built differently:
//  * One kernel per (size, operator, split) block; a candidate's vector is
//    computed element by element from the two operand rows and folded into a
//    64-bit fingerprint A plus a 32-bit check B on the fly -- never stored.
//  * Open-addressing hash table (linear probing from a multiplicative mix of
//    A, power-of-two capacity, 64-bit keys, CAS insert).  Dedup is exact: the
//    thread that claims a slot appends its vector with an atomic row counter
//    (no separate compaction pass) and then publishes the row index in the
//    slot; a thread whose fingerprint hits the slot waits for that
//    publication (bounded) and compares its vector with the stored row
//    element by element, so two different vectors are never merged, whatever
//    their fingerprints.  New vectors are compared with the target.
//  * Kernels of a size run back to back on one stream; each one exits at
//    once if an earlier kernel already found the target, so the host
//    synchronises once per size instead of after every chunk.
// reference_dedup = 1 keeps the reference's uniqueness test as written: a
// vector is stored when the hash set already held it and dropped on a fresh
// insert (warpcore HashSet::insert returns i+1 > 0 for a present key,
// vfb/include/warpcore/hash_set.cuh:210-214,230-233, and the caller keeps
// `insert(...) > 0`, full-cache.cu:285-286).  The first occurrence of a
// vector is then never stored, so this mode keeps the reference's
// fingerprint-only test (here 64-bit A plus a 32-bit check B) instead of
// the exact comparison.
// SIMBA_VFB_FP_BITS=b (1..63, tests only) keeps b bits of A, which forces
// fingerprint collisions; the exact mode must still store every distinct
// vector once.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <climits>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "cuda_util.h"
#include "engine.h"
#include "grammar.h"
#include "ext_grammar.h"

namespace simba {

constexpr unsigned long long kEmptyKey = ~0ULL;

template <class W>
struct VfbArgs {
  W* rows;                    // [cap][S] row-major characteristic vectors
  int8_t* rop;                // provenance: operator (-1 = variable)
  uint32_t* rl;               //             left operand row
  uint32_t* rr;               //             right operand row
  unsigned long long* keys;   // hash keys (fingerprint A), kEmptyKey = free
  unsigned* vals;             // exact mode: stored row + 1 (0 = not yet published,
                              // kNoRow = the cache was full); reference mode: check B
  unsigned long long mask;    // hash capacity - 1
  int shift;                  // 64 - log2(hash capacity): start slot of a key
  unsigned long long fp_mask; // bits of A kept (all but in collision tests)
  unsigned long long* nrows;  // row counter
  unsigned long long cap;     // row capacity
  const W* target;            // S words
  unsigned long long* found;  // (left << 32) | right of the matching candidate
  int* found_launch;          // launch id that found the target (INT_MAX = none)
  int* flags;                 // [0] cache full, [1] hash full
  unsigned long long l0, nl, r0, nr;
  int S;
  int swap;                   // Minus: also op(right, left)
  int inverted;               // reference dedup semantics
  int launch;                 // id of this launch within the search
};

// One element of a composed vector.  z (division and modulo only): the
// divisor vector holds a zero somewhere, and the result is the dividend
// vector (full-cache.cu:230-256); otherwise every divisor element is nonzero.
template <class W, int OP>
__device__ __forceinline__ W vop(W l, W r, bool z = false) {
  if (OP == OP_NOT) return (W)~l;
  if (OP == OP_NEG) return (W)(W(0) - l);
  if (OP == OP_AND) return l & r;
  if (OP == OP_OR) return l | r;
  if (OP == OP_XOR) return l ^ r;
  if (OP == OP_ADD) return (W)(l + r);
  if (OP == OP_SUB) return (W)(l - r);
  if (OP == OP_MUL) return (W)(l * r);
  if (OP == OP_SHL) return r >= (W)(8 * sizeof(W)) ? W(0) : (W)(l << r);
  if (OP == OP_SHR) return r >= (W)(8 * sizeof(W)) ? W(0) : (W)(l >> r);
  if (OP == OP_DIV) return z ? l : (W)(l / r);
  return z ? l : (W)(l % r);  // OP_MOD
}

// Fingerprint: A is a multiply-xorshift fold finished with the MurmurHash3
// 64-bit finaliser (Appleby); B is an independent position-weighted sum.
__device__ __forceinline__ void fp_step(unsigned long long& a, unsigned long long& b,
                                        unsigned long long x, int i) {
  a ^= x;
  a *= 0x9E3779B97F4A7C15ULL;
  a ^= a >> 29;
  b += x * (0xD6E8FEB86659FD93ULL + 2ULL * (unsigned long long)i);
}

__device__ __forceinline__ unsigned long long fp_final(unsigned long long a, int S) {
  a ^= (unsigned long long)S;
  a ^= a >> 33;
  a *= 0xff51afd7ed558ccdULL;
  a ^= a >> 33;
  a *= 0xc4ceb9fe1a85ec53ULL;
  a ^= a >> 33;
  return a == kEmptyKey ? kEmptyKey - 1 : a;
}

__device__ __forceinline__ unsigned fp_check(unsigned long long b) {
  unsigned c = (unsigned)(b ^ (b >> 32));
  return c ? c : 1u;
}

enum { INS_NEW = 0, INS_DUP = 1, INS_FULL = 2 };
constexpr unsigned kNoRow = 0xFFFFFFFFu;   // published by an insert that found the cache full
constexpr int kPublishSpin = 1 << 20;      // polls of an unpublished slot before giving up

__device__ __forceinline__ unsigned long long start_slot(unsigned long long A, int shift) {
  return (A * 0x9E3779B97F4A7C15ULL) >> shift;
}

// Reference mode: fingerprint-only set semantics (a key hit whose published
// check B differs is a collision and probing continues).
__device__ int hash_insert(unsigned long long* keys, unsigned* vals, unsigned long long mask, int shift,
                           unsigned long long A, unsigned B) {
  const unsigned long long s0 = start_slot(A, shift);
  for (unsigned long long p = 0; p <= mask; ++p) {
    const unsigned long long s = (s0 + p) & mask;
    unsigned long long k = keys[s];
    if (k == kEmptyKey) {
      const unsigned long long old = atomicCAS(&keys[s], kEmptyKey, A);
      if (old == kEmptyKey) {
        atomicExch(&vals[s], B);
        return INS_NEW;
      }
      k = old;
    }
    if (k == A) {
      const unsigned v = *(volatile unsigned*)&vals[s];
      if (v == 0 || v == B) return INS_DUP;  // unpublished: same key, treat as equal
    }
  }
  return INS_FULL;
}

template <class W>
__device__ __forceinline__ W load_cg(const W* p) {
  if (sizeof(W) == 8) return (W)__ldcg(reinterpret_cast<const unsigned long long*>(p));
  return (W)__ldcg(reinterpret_cast<const unsigned*>(p));
}

// Exact mode: claim a slot for key A (INS_NEW, *slot set: the caller stores
// the vector and publishes its row), or find the vector already stored
// (INS_DUP): every slot holding A is compared element by element with the
// vector `elem` once its row is published.  INS_FULL: no free slot.  A
// publication that does not come within kPublishSpin polls sets flags[2] and
// reports a duplicate; the host turns that flag into an error.
template <class W, class Elem>
__device__ int hash_claim_exact(const VfbArgs<W>& a, unsigned long long A, Elem elem,
                                unsigned long long* slot) {
  const unsigned long long s0 = start_slot(A, a.shift);
  for (unsigned long long p = 0; p <= a.mask; ++p) {
    const unsigned long long s = (s0 + p) & a.mask;
    unsigned long long k = a.keys[s];
    if (k == kEmptyKey) {
      const unsigned long long old = atomicCAS(&a.keys[s], kEmptyKey, A);
      if (old == kEmptyKey) {
        *slot = s;
        return INS_NEW;
      }
      k = old;
    }
    if (k != A) continue;
    unsigned v = *(volatile unsigned*)&a.vals[s];
    for (int t = 0; v == 0; ++t) {
      if (t == kPublishSpin) {
        atomicOr(&a.flags[2], 1);
        return INS_DUP;
      }
      __nanosleep(64);
      v = *(volatile unsigned*)&a.vals[s];
    }
    if (v == kNoRow) return INS_DUP;  // not stored: the cache is full and the search ends here
    __threadfence();                  // the row's words were written before the publication
    const W* row = a.rows + (unsigned long long)(v - 1) * a.S;
    bool same = true;
    if ((a.S * sizeof(W)) % 16 == 0) {  // rows 16-byte aligned: 16-byte loads
      constexpr int VW = 16 / sizeof(W);
      const uint4* r4 = reinterpret_cast<const uint4*>(row);
      for (int i = 0; i < a.S && same; i += VW) {
        const uint4 q = __ldcg(r4 + i / VW);
        W w[VW];
        memcpy(w, &q, 16);
#pragma unroll
        for (int j = 0; j < VW; ++j) same &= w[j] == elem(i + j);
      }
    } else {
      for (int i = 0; i < a.S && same; ++i) same = load_cg<W>(row + i) == elem(i);
    }
    if (same) return INS_DUP;
    // the same fingerprint for another vector: keep probing
  }
  return INS_FULL;
}

// Keep / store one composed candidate (x, y) whose fingerprint is (A, B):
// insert into the hash set, append the vector when it is kept, compare it
// with the target.  `elem(i)` recomputes element i of the vector.
template <class W, int OP, class Elem>
__device__ __forceinline__ void vfb_offer(const VfbArgs<W>& a, unsigned long long x, unsigned long long y,
                                          unsigned long long A, unsigned B, Elem elem) {
  if (*(volatile int*)&a.flags[0]) return;  // the cache is full: nothing more is stored
  A &= a.fp_mask;
  unsigned long long slot = ~0ULL;
  if (a.inverted) {
    // INS_FULL is kept too, as in the reference
    if (hash_insert(a.keys, a.vals, a.mask, a.shift, A, B) == INS_NEW) return;
  } else {
    const int ins = hash_claim_exact<W>(a, A, elem, &slot);
    if (ins == INS_FULL) atomicOr(&a.flags[1], 1);
    if (ins != INS_NEW) return;
  }
  const unsigned long long row = atomicAdd(a.nrows, 1ULL);
  bool match = true;
  W* out = row < a.cap ? a.rows + row * a.S : nullptr;
  for (int i = 0; i < a.S; ++i) {
    const W v = elem(i);
    match &= v == a.target[i];
    if (out) out[i] = v;
  }
  if (out) {
    a.rop[row] = (int8_t)OP;
    a.rl[row] = (uint32_t)x;
    a.rr[row] = (uint32_t)y;
  } else {
    atomicOr(&a.flags[0], 1);
  }
  if (slot != ~0ULL) {  // publish the stored row to threads waiting on the slot
    __threadfence();
    atomicExch(&a.vals[slot], out ? (unsigned)(row + 1) : kNoRow);
  }
  if (match) {
    atomicCAS(a.found, ~0ULL, (x << 32) | y);
    atomicMin(a.found_launch, a.launch);
  }
}

template <class W, int OP>
__global__ void __launch_bounds__(256) vfb_compose_kernel(VfbArgs<W> a) {
  if (*(volatile int*)a.found_launch < a.launch) return;  // an earlier block found it
  constexpr bool unary = OP == OP_NOT || OP == OP_NEG;
  const unsigned long long per = unary ? a.nl : a.nl * a.nr;
  const unsigned long long total = per << (a.swap ? 1 : 0);
  const int S = a.S;
  for (unsigned long long idx = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
       idx += (unsigned long long)gridDim.x * blockDim.x) {
    // the cache or the hash table is full: the search ends with this size
    if (*(volatile int*)&a.flags[0] | *(volatile int*)&a.flags[1]) break;
    const unsigned long long pair = a.swap ? idx >> 1 : idx;
    unsigned long long x, y;
    if (unary) {
      x = a.l0 + pair;
      y = 0;
    } else {
      const unsigned long long li = pair / a.nr;
      x = a.l0 + li;
      y = a.r0 + (pair - li * a.nr);
      if (a.swap && (idx & 1)) {
        const unsigned long long t = x;
        x = y;
        y = t;
      }
    }
    const W* L = a.rows + x * S;
    const W* R = a.rows + y * S;
    bool z = false;
    if (OP == OP_DIV || OP == OP_MOD)
      for (int i = 0; i < S && !z; ++i) z = R[i] == W(0);
    unsigned long long fa = 0x243F6A8885A308D3ULL, fb = 0;
    for (int i = 0; i < S; ++i) {
      const W v = vop<W, OP>(L[i], unary ? W(0) : R[i], z);
      fp_step(fa, fb, (unsigned long long)v, i);
    }
    vfb_offer<W, OP>(a, x, y, fp_final(fa, S), fp_check(fb),
                     [&](int i) { return vop<W, OP>(L[i], unary ? W(0) : R[i], z); });
  }
}

// Binary compositions, tiled: a CTA stages kTL left rows and kTR right rows
// in shared memory (row pitch S+1 words, so the 32 right rows a warp reads
// fall in different banks) and composes all kTL x kTR pairs from there, so
// each operand row crosses L2/HBM once per tile instead of once per pair.
// Thread t takes right row t % kTR and left rows t / kTR + 8 j, j < 2.
constexpr int kTL = 16, kTR = 32;

template <class W, int OP>
__global__ void __launch_bounds__(256) vfb_tile_kernel(VfbArgs<W> a) {
  if (*(volatile int*)a.found_launch < a.launch) return;  // an earlier block found it
  extern __shared__ __align__(16) unsigned char vfb_smem[];
  W* sl = reinterpret_cast<W*>(vfb_smem);
  const int S = a.S, P = S + 1;
  W* sr = sl + kTL * P;
  const unsigned long long tl = (a.nl + kTL - 1) / kTL, tr = (a.nr + kTR - 1) / kTR;
  const int ri = threadIdx.x % kTR, li0 = threadIdx.x / kTR;
  __shared__ int s_stop;
  for (unsigned long long tile = blockIdx.x; tile < tl * tr; tile += gridDim.x) {
    const unsigned long long lb = (tile / tr) * kTL, rb = (tile % tr) * kTR;
    const int nl = (int)(a.nl - lb < (unsigned long long)kTL ? a.nl - lb : kTL);
    const int nr = (int)(a.nr - rb < (unsigned long long)kTR ? a.nr - rb : kTR);
    // one read per CTA, so that every thread leaves the loop together: a full
    // cache or hash table ends the search with this size
    if (threadIdx.x == 0) s_stop = *(volatile int*)&a.flags[0] | *(volatile int*)&a.flags[1];
    __syncthreads();  // the previous tile's reads are done
    if (s_stop) break;
    const W* gl = a.rows + (a.l0 + lb) * S;
    const W* gr = a.rows + (a.r0 + rb) * S;
    for (int q = threadIdx.x; q < nl * S; q += blockDim.x) sl[(q / S) * P + q % S] = gl[q];
    for (int q = threadIdx.x; q < nr * S; q += blockDim.x) sr[(q / S) * P + q % S] = gr[q];
    __syncthreads();
    if (ri >= nr) continue;
    const W* R = sr + ri * P;
    const unsigned long long y = a.r0 + rb + ri;
#pragma unroll
    for (int j = 0; j < kTL / 8; ++j) {
      const int li = li0 + 8 * j;
      if (li >= nl) break;
      const W* L = sl + li * P;
      const unsigned long long x = a.l0 + lb + li;
      unsigned long long fa = 0x243F6A8885A308D3ULL, fb = 0, ga = fa, gb = 0;
      for (int i = 0; i < S; ++i) {
        const W l = L[i], r = R[i];
        fp_step(fa, fb, (unsigned long long)vop<W, OP>(l, r), i);
        if (a.swap) fp_step(ga, gb, (unsigned long long)vop<W, OP>(r, l), i);
      }
      vfb_offer<W, OP>(a, x, y, fp_final(fa, S), fp_check(fb),
                       [&](int i) { return vop<W, OP>(L[i], R[i]); });
      if (a.swap)
        vfb_offer<W, OP>(a, y, x, fp_final(ga, S), fp_check(gb),
                         [&](int i) { return vop<W, OP>(R[i], L[i]); });
    }
  }
}

template <class W>
__global__ void vfb_init_kernel(VfbArgs<W> a, int k) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= k) return;
  const W* v = a.rows + (unsigned long long)j * a.S;
  unsigned long long fa = 0x243F6A8885A308D3ULL, fb = 0;
  for (int i = 0; i < a.S; ++i) fp_step(fa, fb, (unsigned long long)v[i], i);
  const unsigned long long A = fp_final(fa, a.S) & a.fp_mask;
  if (a.inverted) {
    hash_insert(a.keys, a.vals, a.mask, a.shift, A, fp_check(fb));
  } else {  // the variables' rows are in place already
    unsigned long long slot;
    if (hash_claim_exact<W>(a, A, [&](int i) { return v[i]; }, &slot) == INS_NEW) {
      __threadfence();
      atomicExch(&a.vals[slot], (unsigned)(j + 1));
    }
  }
  a.rop[j] = -1;
  a.rl[j] = (uint32_t)j;
  a.rr[j] = 0;
}

template <class W>
static void launch_tiled(int op, int grid, size_t smem, cudaStream_t st, const VfbArgs<W>& a) {
  switch (op) {
    case OP_AND: vfb_tile_kernel<W, OP_AND><<<grid, 256, smem, st>>>(a); break;
    case OP_OR: vfb_tile_kernel<W, OP_OR><<<grid, 256, smem, st>>>(a); break;
    case OP_XOR: vfb_tile_kernel<W, OP_XOR><<<grid, 256, smem, st>>>(a); break;
    case OP_ADD: vfb_tile_kernel<W, OP_ADD><<<grid, 256, smem, st>>>(a); break;
    case OP_SUB: vfb_tile_kernel<W, OP_SUB><<<grid, 256, smem, st>>>(a); break;
    default: vfb_tile_kernel<W, OP_MUL><<<grid, 256, smem, st>>>(a); break;
  }
}

template <class W>
static int tile_smem_setup(int S, size_t* smem) {
  *smem = (size_t)(kTL + kTR) * (S + 1) * sizeof(W);
  const int ops[6] = {OP_AND, OP_OR, OP_XOR, OP_ADD, OP_SUB, OP_MUL};
  for (int op : ops) {
    const void* f = nullptr;
    switch (op) {
      case OP_AND: f = (const void*)vfb_tile_kernel<W, OP_AND>; break;
      case OP_OR: f = (const void*)vfb_tile_kernel<W, OP_OR>; break;
      case OP_XOR: f = (const void*)vfb_tile_kernel<W, OP_XOR>; break;
      case OP_ADD: f = (const void*)vfb_tile_kernel<W, OP_ADD>; break;
      case OP_SUB: f = (const void*)vfb_tile_kernel<W, OP_SUB>; break;
      default: f = (const void*)vfb_tile_kernel<W, OP_MUL>; break;
    }
    SB_CUDA(cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)*smem));
  }
  return 0;
}

template <class W>
static void launch_compose(int op, int grid, cudaStream_t st, const VfbArgs<W>& a) {
  switch (op) {
    case OP_NOT: vfb_compose_kernel<W, OP_NOT><<<grid, 256, 0, st>>>(a); break;
    case OP_AND: vfb_compose_kernel<W, OP_AND><<<grid, 256, 0, st>>>(a); break;
    case OP_OR: vfb_compose_kernel<W, OP_OR><<<grid, 256, 0, st>>>(a); break;
    case OP_XOR: vfb_compose_kernel<W, OP_XOR><<<grid, 256, 0, st>>>(a); break;
    case OP_NEG: vfb_compose_kernel<W, OP_NEG><<<grid, 256, 0, st>>>(a); break;
    case OP_ADD: vfb_compose_kernel<W, OP_ADD><<<grid, 256, 0, st>>>(a); break;
    case OP_SUB: vfb_compose_kernel<W, OP_SUB><<<grid, 256, 0, st>>>(a); break;
    case OP_MUL: vfb_compose_kernel<W, OP_MUL><<<grid, 256, 0, st>>>(a); break;
    case OP_SHL: vfb_compose_kernel<W, OP_SHL><<<grid, 256, 0, st>>>(a); break;
    case OP_SHR: vfb_compose_kernel<W, OP_SHR><<<grid, 256, 0, st>>>(a); break;
    case OP_DIV: vfb_compose_kernel<W, OP_DIV><<<grid, 256, 0, st>>>(a); break;
    default: vfb_compose_kernel<W, OP_MOD><<<grid, 256, 0, st>>>(a); break;
  }
}

template <class W>
static int vfb_typed(const HostInstance& h, int max_len, const EngineOptions& o, int inverted,
                     int64_t cache_rows, VfbOutcome* out) {
  *out = VfbOutcome();
  const int S = h.S, k = h.k;
  SB_CUDA(cudaSetDevice(o.device));
  cudaStream_t st = nullptr;
  bool own = false;
  if (o.stream) st = reinterpret_cast<cudaStream_t>(o.stream);
  else {
    SB_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    own = true;
  }
  struct StreamGuard {
    cudaStream_t s;
    bool own;
    ~StreamGuard() {
      if (own && s) cudaStreamDestroy(s);
    }
  } guard{st, own};
  int sms = 0;
  SB_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, o.device));
  // Row capacity: the reference's rule (max pitch / (S * 4 bytes),
  // full-cache.cu:713-718) unless the caller sets one.
  unsigned long long cap = (unsigned long long)cache_rows;
  if (cap == 0) {
    int pitch = 0;
    SB_CUDA(cudaDeviceGetAttribute(&pitch, cudaDevAttrMaxPitch, o.device));
    cap = (unsigned long long)pitch / ((unsigned long long)S * 4ULL);
  }
  cap = std::max<unsigned long long>(cap, (unsigned long long)k + 1);
  cap = std::min<unsigned long long>(cap, 0xFFFFFFF0ULL);
  unsigned long long slots = 1;
  while (slots < cap * (inverted ? 4 : 2)) slots <<= 1;
  DevBuf rows, rop, rl, rr, keys, vals, scal, tgt;
  SB_CUDA(rows.reserve(cap * S * sizeof(W)));
  SB_CUDA(rop.reserve(cap));
  SB_CUDA(rl.reserve(cap * 4));
  SB_CUDA(rr.reserve(cap * 4));
  SB_CUDA(keys.reserve(slots * 8));
  SB_CUDA(vals.reserve(slots * 4));
  SB_CUDA(scal.reserve(64));
  SB_CUDA(tgt.reserve(S * sizeof(W)));
  out->cache_bytes = cap * S * sizeof(W) + cap * 9;
  out->table_bytes = slots * 12;
  SB_CUDA(cudaMemsetAsync(keys.p, 0xFF, slots * 8, st));
  SB_CUDA(cudaMemsetAsync(vals.p, 0, slots * 4, st));
  // scalars: [0] nrows, [1] found pair, [2] found_launch|flags
  unsigned long long init[4] = {(unsigned long long)k, ~0ULL, 0, 0};
  SB_CUDA(cudaMemcpyAsync(scal.p, init, sizeof(init), cudaMemcpyHostToDevice, st));
  int* iflags = reinterpret_cast<int*>(scal.as<unsigned long long>() + 2);
  const int fl_init[4] = {INT_MAX, 0, 0, 0};
  SB_CUDA(cudaMemcpyAsync(iflags, fl_init, sizeof(fl_init), cudaMemcpyHostToDevice, st));
  std::vector<W> hv((size_t)k * S), ht(S);
  for (int j = 0; j < k; ++j)
    for (int i = 0; i < S; ++i) hv[(size_t)j * S + i] = (W)h.in[(size_t)i * k + j];
  for (int i = 0; i < S; ++i) ht[i] = (W)h.out[i];
  SB_CUDA(cudaMemcpyAsync(rows.p, hv.data(), hv.size() * sizeof(W), cudaMemcpyHostToDevice, st));
  SB_CUDA(cudaMemcpyAsync(tgt.p, ht.data(), ht.size() * sizeof(W), cudaMemcpyHostToDevice, st));

  VfbArgs<W> a;
  memset(&a, 0, sizeof(a));
  a.rows = rows.as<W>();
  a.rop = rop.as<int8_t>();
  a.rl = rl.as<uint32_t>();
  a.rr = rr.as<uint32_t>();
  a.keys = keys.as<unsigned long long>();
  a.vals = vals.as<unsigned>();
  a.mask = slots - 1;
  a.shift = 64;
  for (unsigned long long q = slots; q > 1; q >>= 1) --a.shift;
  a.fp_mask = ~0ULL;
  if (const char* fb = getenv("SIMBA_VFB_FP_BITS")) {
    const int b = atoi(fb);
    if (b >= 1 && b < 64) a.fp_mask = (1ULL << b) - 1;
  }
  a.nrows = scal.as<unsigned long long>();
  a.cap = cap;
  a.target = tgt.as<W>();
  a.found = scal.as<unsigned long long>() + 1;
  a.found_launch = iflags;
  a.flags = iflags + 1;
  a.S = S;
  a.inverted = inverted;

  const auto t0 = std::chrono::steady_clock::now();
  // size 1: the variables (full-cache.cu:694-707), checked on the host
  for (int j = 0; j < k; ++j) {
    out->candidates++;
    bool eq = true;
    for (int i = 0; i < S && eq; ++i) eq = (W)h.in[(size_t)i * k + j] == (W)h.out[i];
    if (eq) {
      out->status = SIMBA_OK;
      out->size = 1;
      out->op = 8;
      out->postfix = std::string(1, (char)('0' + j));
      out->rows_per_size[1] = k;
      out->rows_total = k;
      return SIMBA_OK;
    }
  }
  cudaEvent_t e0, e1;
  SB_CUDA(cudaEventCreate(&e0));
  SB_CUDA(cudaEventCreate(&e1));
  SB_CUDA(cudaEventRecord(e0, st));
  vfb_init_kernel<W><<<(k + 63) / 64, 64, 0, st>>>(a, k);
  out->launches++;
  SB_CUDA(cudaGetLastError());
  std::vector<unsigned long long> start(max_len + 3, 0);
  start[1] = 0;
  start[2] = (unsigned long long)k;
  out->rows_per_size[1] = k;
  const int grid = sms * 8;
  // tiled binary compositions unless SIMBA_VFB_TILED=0 (the per-pair kernel)
  const char* te = getenv("SIMBA_VFB_TILED");
  const bool tiled = !(te && te[0] == '0');
  size_t tile_smem = 0;
  int tile_grid = grid;
  if (tiled) {
    if (tile_smem_setup<W>(S, &tile_smem)) return SIMBA_E_CUDA;
    int occ = 1;
    SB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, vfb_tile_kernel<W, OP_MUL>, 256,
                                                          tile_smem));
    tile_grid = sms * std::max(occ, 1);
  }
  const bool ext = o.grammar == 1;  // the extended operators (ext_grammar.h)
  const int nops = ext ? kExtOps : 8;
  int launch = 0;
  struct LaunchInfo {
    int op;
    unsigned long long cand;
  };
  std::vector<LaunchInfo> info;
  unsigned long long hs[4];
  int status = SIMBA_NOT_FOUND;
  for (int L = 2; L <= max_len; ++L) {
    if (o.budget_s > 0 &&
        std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count() > o.budget_s) {
      status = SIMBA_BUDGET;
      break;
    }
    info.clear();
    const int first_launch = launch;
    for (int oi = 0; oi < nops; ++oi) {
      const int op = ext ? ext_code(oi) : oi;
      if (is_unary(op)) {
        a.l0 = start[L - 1];
        a.nl = start[L] - start[L - 1];
        a.r0 = 0;
        a.nr = 1;
        a.swap = 0;
        if (a.nl == 0) continue;
        a.launch = launch++;
        info.push_back({op, a.nl});
        launch_compose<W>(op, (int)std::min<unsigned long long>((a.nl + 255) / 256, grid), st, a);
      } else {
        for (int i = 1; 2 * i <= L - 1; ++i) {
          const int j = L - 1 - i;
          a.l0 = start[i];
          a.nl = start[i + 1] - start[i];
          a.r0 = start[j];
          a.nr = start[j + 1] - start[j];
          // non-commutative operators also compose the swapped pair
          a.swap = (op == OP_SUB || op >= OP_SHL) ? 1 : 0;
          const unsigned long long n = (a.nl * a.nr) << a.swap;
          if (n == 0) continue;
          a.launch = launch++;
          info.push_back({op, n});
          const unsigned long long tiles = ((a.nl + kTL - 1) / kTL) * ((a.nr + kTR - 1) / kTR);
          if (tiled && op < OP_SHL)  // the extended operators: one pair per thread
            launch_tiled<W>(op, (int)std::min<unsigned long long>(tiles, tile_grid), tile_smem, st, a);
          else
            launch_compose<W>(op, (int)std::min<unsigned long long>((n + 255) / 256, grid), st, a);
        }
      }
    }
    SB_CUDA(cudaGetLastError());
    out->launches = launch + 1;
    SB_CUDA(cudaMemcpyAsync(hs, scal.p, sizeof(hs), cudaMemcpyDeviceToHost, st));
    SB_CUDA(cudaStreamSynchronize(st));
    const int fl = (int)(hs[2] & 0xFFFFFFFFULL);
    const int full = (int)(hs[2] >> 32);
    const int hfull = (int)(hs[3] & 0xFFFFFFFFULL);
    if (hs[3] >> 32) {
      set_last_error("VFB hash slot not published within its wait limit");
      return SIMBA_E_INTERNAL;
    }
    const unsigned long long nrows = std::min<unsigned long long>(hs[0], cap);
    // reference-rule candidate count: every launch up to the one that found
    for (size_t q = 0; q < info.size(); ++q)
      if (fl == INT_MAX || first_launch + (int)q <= fl) out->candidates += info[q].cand;
    start[L + 1] = nrows;
    out->rows_per_size[L] = (int64_t)(nrows - start[L]);
    out->rows_total = (int64_t)nrows;
    out->max_size_searched = L;
    if (o.verbose)
      fprintf(stderr, "vfb size %2d | rows %llu | candidates %llu\n", L, nrows,
              (unsigned long long)out->candidates);
    if (fl != INT_MAX) {
      out->status = SIMBA_OK;
      out->size = L;
      out->op = info[fl - first_launch].op;
      // reconstruct the expression from the provenance arrays
      const unsigned long long pair = hs[1];
      std::string post;
      struct Node {
        static int build(const DevBuf& rop, const DevBuf& rl, const DevBuf& rr, unsigned long long row,
                         int k, std::string* p, int depth) {
          if (depth > 200) return -1;
          if (row < (unsigned long long)k) {
            p->push_back((char)('0' + (int)row));
            return 0;
          }
          int8_t op;
          uint32_t l, r;
          if (cudaMemcpy(&op, rop.as<int8_t>() + row, 1, cudaMemcpyDeviceToHost) != cudaSuccess) return -1;
          if (cudaMemcpy(&l, rl.as<uint32_t>() + row, 4, cudaMemcpyDeviceToHost) != cudaSuccess) return -1;
          if (cudaMemcpy(&r, rr.as<uint32_t>() + row, 4, cudaMemcpyDeviceToHost) != cudaSuccess) return -1;
          if (build(rop, rl, rr, l, k, p, depth + 1)) return -1;
          if (!is_unary(op) && build(rop, rl, rr, r, k, p, depth + 1)) return -1;
          p->push_back(code_char(op));
          return 0;
        }
      };
      const unsigned long long x = pair >> 32, y = pair & 0xFFFFFFFFULL;
      int rc = Node::build(rop, rl, rr, x, k, &post, 0);
      if (!rc && !is_unary(out->op)) rc = Node::build(rop, rl, rr, y, k, &post, 0);
      if (rc) {
        set_last_error("VFB expression reconstruction failed");
        return SIMBA_E_INTERNAL;
      }
      post.push_back(code_char(out->op));
      out->postfix = post;
      status = SIMBA_OK;
      break;
    }
    if (full || hfull) {
      status = SIMBA_CACHE_FULL;
      break;
    }
  }
  SB_CUDA(cudaEventRecord(e1, st));
  SB_CUDA(cudaEventSynchronize(e1));
  float ms = 0;
  SB_CUDA(cudaEventElapsedTime(&ms, e0, e1));
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  out->device_ms = ms;
  out->status = status;
  // algorithmic bytes: two operand rows per candidate (one for unary), one
  // 12-byte hash probe, one written row per stored vector
  out->bytes_moved = (double)out->candidates * (2.0 * S * sizeof(W) + 12.0) +
                     (double)out->rows_total * S * sizeof(W);
  if (status == SIMBA_OK && !(ext ? ext_vector_check(out->postfix, h) : host_check(out->postfix, h))) {
    set_last_error("VFB answer failed the host re-check");
    return SIMBA_E_INTERNAL;
  }
  return status;
}

int vfb_run(const HostInstance& h, int max_len, const EngineOptions& o, int inverted, int64_t cache_rows,
            VfbOutcome* out) {
  int rc = validate(h, 1);
  if (rc) return rc;
  if (max_len < 1 || max_len > 100) {
    set_last_error("maxLen must be between 1 and 100");
    return SIMBA_E_ARG;
  }
  if (o.grammar == 1 && (inverted || h.k > kExtMaxTerms)) {
    set_last_error("the extended grammar takes at most 10 terminals and exact dedup");
    return SIMBA_E_ARG;
  }
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= o.device || o.device < 0) {
    cudaGetLastError();
    set_last_error("no usable CUDA device");
    return SIMBA_E_NODEV;
  }
  if (h.bits == 64) return vfb_typed<uint64_t>(h, max_len, o, inverted, cache_rows, out);
  return vfb_typed<uint32_t>(h, max_len, o, inverted, cache_rows, out);
}

}  // namespace simba
