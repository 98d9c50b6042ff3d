// Plain SIMBA search on sm_100a: tabled spine engine + one-thread-per-rank
// engine.
//
// What is computed is exactly the reference's search (simba/src/nocache.cu:
// 197-289): sizes in increasing order, the rank space of each size in the
// reference order, stop after the first (size, root-operator) block holding
// an expression that matches every sample, and report the minimum matching
// rank of that block.
//
// How it is computed differs.  The reference unranks every rank from
// scratch and interprets the postfix string (nocache.cu:23-107,
// mba.cuh:6-69).  Here:
//
//  * Value tables.  V_t[r] = value on sample 0 of the size-t expression of
//    rank r, for every t <= T, built bottom-up (one operator per entry) in
//    HBM.  Building V_t is itself the search of size t.
//  * Spines.  A candidate of size s > T is a path from the root along its
//    larger operand ("big side") down to a subtree of size <= T (the
//    "bottom", read from V_tb); every level on the path combines the big
//    side with a "small side" of size <= T (read from V_ts), or applies a
//    chain of unary operators.  A spine shape with fixed small-side indices
//    is a "context"; its candidates are all bottom values v in V_tb, and
//    their ranks are base + sum(idx_l * coef_l) + v * coefv, so the whole
//    rank space of a size is a disjoint union of (context x bottom range)
//    rectangles.  Unary chains that compose to the same affine map
//    (x -> +-x + c) are tested once with the smallest of their ranks, which
//    yields the same minimum matching rank.
//  * Inversion.  The sample-0 test "root value == target" is pushed down
//    the spine into a constraint "(v & M) == K" on the bottom value, so a
//    candidate costs one load (amortised over R contexts) and one masked
//    compare.  Operators that cannot be inverted under the mask left by
//    & / | above them are evaluated explicitly instead.
//  * Verification.  A sample-0 match is queued in shared memory and then
//    verified by a whole warp: each lane evaluates different samples (staged
//    in shared memory) and a ballot rejects the candidate at the first
//    mismatching group of samples.
#pragma once
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <chrono>
#include <map>
#include <cstdio>
#include <cstddef>
#include <cstdlib>
#include <cstring>
#include <limits>
#include <memory>
#include <vector>

#include "cuda_util.h"
#include "engine.h"
#include "grammar.h"

namespace simba {

constexpr int kMaxDepth = 12;  // spine levels
constexpr int kThreads = 256;  // CTA size of the search kernels
constexpr int kQueue = 128;    // shared-memory queue of matches to verify
constexpr int kPre = 256;      // shared-memory queue of sample-0 matches to filter
constexpr int kPreG = 131072;  // the same queue per CTA in global memory, when given
                               // (8-byte entries: context << 32 | bottom index)
constexpr int kLive = 512;     // live contexts of a nested-compare unit listed in shared memory
// Tuning knobs (compile-time): contexts per thread, minimum resident CTAs
// per SM.
#ifndef SIMBA_NESTED_PACK16
#define SIMBA_NESTED_PACK16 1  // masked nested compares: two candidates per 32-bit prefilter word
#endif
#ifndef SIMBA_KR
#define SIMBA_KR 8
#endif
#ifndef SIMBA_NESTED_PIPELINE
#define SIMBA_NESTED_PIPELINE 0  // nested compares: next loads issued before the current tests
#endif                           // (measured: no gain at 3 CTAs/SM, the extra registers spill)
#ifndef SIMBA_PACK_ALWAYS
#define SIMBA_PACK_ALWAYS 0  // packed prefilter in every warp (for comparisons)
#endif
#ifndef SIMBA_PACK_IMAD
#define SIMBA_PACK_IMAD 1  // packed prefilter: the subtraction as a multiply-add (FMA pipe)
#endif
#ifndef SIMBA_XOP_SPECIALIZE
#define SIMBA_XOP_SPECIALIZE 1  // one explicit level: its operator as a template argument
#endif                          // (a spine_kernel variant of its own; compile time grows)
#ifndef SIMBA_JOIN_VALS_LOG2
#define SIMBA_JOIN_VALS_LOG2 15  // hash join: bottom values per work unit
#endif
// Resident CTAs per SM the spine kernel is compiled for: 3 caps it at 85
// registers (80 used, a few hundred bytes of spills), the occupancy its work
// units were tuned at; left to itself the compiler picked 48 registers and
// spilled the nested compare loop's constraints.
#ifndef SIMBA_MINB
#define SIMBA_MINB 3
#endif
#if SIMBA_MINB > 0
#define SIMBA_SPINE_BOUNDS __launch_bounds__(256, SIMBA_MINB)
#else
#define SIMBA_SPINE_BOUNDS __launch_bounds__(256)
#endif
constexpr int kR = SIMBA_KR;   // contexts per thread
constexpr int kMaxExplicit = 2;
constexpr int kExtra = 3;       // samples besides sample 0 with value tables (match filters)
// Hash join of fully inverted spines: contexts per block, table slots, bits
// of the membership filter, bottom values per block, and the fewest contexts
// for which the join beats the nested compare loop.  Kept small: shared
// memory taken here is L1 cache lost to every other work unit.
constexpr int kJoinCtx = 512;
constexpr int kJoinSlots = 1024;
constexpr int kJoinBits = 16384;
constexpr unsigned long long kJoinVals = 1ULL << SIMBA_JOIN_VALS_LOG2;
constexpr unsigned long long kJoinMin = 1;

// One level of a spine, top-down (level 0 is the root).
struct Level {
  uint64_t coef;     // rank coefficient of this level's small index
  uint64_t nsmall;   // N(ts) (binary), 1 (chain)
  uint64_t c;        // chain: additive constant (two's complement)
  int8_t kind;       // 0 binary, 1 unary chain x -> eps * x + c
  int8_t op;         // binary operator
  int8_t small_left; // small operand is the left one
  int8_t ts;         // small side size
  int8_t eps;        // chain sign
  int8_t chain_len;  // chain: number of unary operators it stands for
  int8_t pad[2];
};

struct alignas(16) Item {
  uint64_t base;        // rank of the all-zero indices
  uint64_t coefv;       // rank coefficient of the bottom index
  uint64_t nctx;        // number of contexts
  uint64_t nv;          // bottom values N(tb)
  uint64_t unit_begin;  // first work unit of this item
  uint64_t vb;          // bottom values per unit (multiple of 64)
  uint64_t cblocks;     // context blocks
  uint64_t vblocks;     // value blocks
  uint16_t cb;          // contexts per unit = G * kR (join: per block)
  int8_t joinable;      // every context's constraint is v & M == K with M a low-bit mask
  int8_t group;         // fused member: index of its group (live-context lists)
  uint16_t G, L;        // G context groups x L value lanes = kThreads
  int8_t depth, inv, bottom, full, nexp;
  int8_t fused;         // 1: contexts are read from the materialised list; 2: the list
                        // holds only the live contexts (see materialize_kernel)
  uint16_t cpu;         // context blocks per work unit (> 1 for small bottoms)
  uint64_t ctx_off;     // fused: first context in Params::ctxs
  uint32_t inst;        // instance (index into Params::insts)
  float prio;           // guided search: prior of the spine's shape class
  Level lv[kMaxDepth];
};

// A materialised context of a fused group: the bottom-value constraint
// (v & M) == K, the rank base of candidate v (base + v * the member spine's
// coefv), and where the context comes from (for the sample-1 filter).
template <class W>
struct Ctx {
  W M, K;
  unsigned long long base;
  unsigned member;  // index of the member spine in Params::sitems
  unsigned c;       // context index inside that spine
};
static_assert(sizeof(Item) % 16 == 0, "Item must be 16-byte sized");

// First bottom index of an item: a whole tabled size split into shape-class
// ranges for the guided search keeps its range start in lv[0].coef (a
// depth-0 item has no levels); every other item starts at 0.  The candidate
// of bottom index v of a depth-0 item has rank base + v.
SB_HD uint64_t item_voff(const Item& it) { return it.depth == 0 ? it.lv[0].coef : 0; }

// Match-filter samples with value tables (options.filter_samples, 0 = all).
inline int filter_samples(const EngineOptions& o) {
  return o.filter_samples > 0 ? std::min(o.filter_samples, kExtra) : kExtra;
}

// Work units of a spine: groups of `cpu` context blocks x value blocks.
SB_HD uint64_t item_units(const Item& it) {
  const uint64_t cpu = it.cpu ? it.cpu : 1;
  return (it.cblocks + cpu - 1) / cpu * it.vblocks;
}

// Everything the kernels need about one instance (several per launch in
// batch mode): value tables, samples, count table, the sample-0 target, the
// size being searched and where its minimum matching rank accumulates.
template <class W>
struct alignas(16) InstDesc {
  const W* tab[kMaxSize + 1];
  const W* in;                      // S*K words, 16-byte padded
  const W* out;                     // S words, 16-byte padded
  const unsigned long long* counts; // (kMaxSize+1) x kCols count table
  unsigned long long* best;         // minimum verified matching rank
  unsigned long long* ns;           // batch, or null: [0] first verified match,
                                    // [1] last unit that ran (globaltimer ns)
  const W* tabx[kExtra][kMaxSize + 1];  // value tables on samples 1..kExtra (null: absent)
  W target;                         // output on sample 0
  W targetx[kExtra];                // outputs on samples 1..kExtra
  int size;
  int S, K;
  int rtid;                         // 1: best holds RTid keys (positions), not ranks
  int pad[2];
  unsigned long long rt_inv[8];     // RTid: inverse multiplier of each operator block
};

// Batch mode: one instance's search of one size, pointing at a shared spine
// list (TmplDesc) that lives once on the device for all instances with the
// same (terminals, tabled size, size, unit size).
struct Task {
  unsigned long long unit_begin;  // first global unit of this task
  unsigned long long ctx_base;    // first materialised context of the instance
  unsigned int inst;
  unsigned int tmpl;
  int bucket;                     // guided: the one shape-class bucket covered; -1: whole list
  int pad;
};

struct TmplDesc {
  unsigned long long item_off;    // into Params::items
  unsigned long long small_off;   // into Params::sitems
  unsigned int nitems;
  unsigned int nsmall;
  unsigned long long bucket_off;  // guided lists: into Params::buckets
};

// Guided batch: a spine list grouped by shape class (64 buckets, each in
// rank order) -- where each bucket's spines and units start in the list.
struct TmplBuckets {
  unsigned int item[65];
  unsigned int pad;
  unsigned long long unit[65];
};

template <class W>
struct Params {
  const InstDesc<W>* insts;
  const Task* tasks;        // batch mode when non-null
  const TmplDesc* tmpls;
  const TmplBuckets* buckets;  // guided batch
  int ntasks;
  const Item* items;
  const Ctx<W>* ctxs;     // materialised contexts of fused groups
  const Item* sitems;     // spines whose contexts are materialised
  int nsitems;
  unsigned long long nctxs;
  unsigned long long* counter;
  unsigned long long* evaluated;
  unsigned long long* start_ns;
  int* flags;  // [0] budget expired, [1] inversion failure, [2] queue overflows
  unsigned long long* hits;  // sample-0 matches sent to verification (may be null)
  unsigned long long* live;  // candidates of live nested-compare contexts (may be null)
  unsigned long long* ctx_live;  // per fused group: [2g] live contexts appended, [2g+1] the
                                 // group's first list slot (null: every context in place)
  unsigned long long* preq;  // per-CTA queues of sample-0 matches, [grid][kPreG] (may be null)
  unsigned join_off;         // byte offset of JoinSmem in dynamic shared memory; 0: no join units
  unsigned long long total_units;
  unsigned long long unit_offset;  // this shard's first unit (multi-GPU)
  unsigned long long unit_stride;  // number of shards (0 is read as 1)
  unsigned long long budget_ns;
  int nitems;
  int stop_on_match;
  int maxS, maxK;  // largest instance staged in shared memory
};

struct alignas(16) Smem {
  unsigned long long counts[(kMaxSize + 1) * kCols];
  Item item;  // 16-byte aligned: filled with uint4 copies
  alignas(16) unsigned char desc[sizeof(InstDesc<unsigned long long>)];
  int inst_idx;
  unsigned one;  // 1, read back so that the compiler cannot fold it (see process_unit)
  int pad_[2];
  unsigned long long queue[kQueue];
  unsigned long long pre_c[kPre], pre_v[kPre];  // sample-0 matches: context, bottom index
  int pn;
  int nlive;                   // live contexts of the current nested-compare unit
  unsigned short live[kLive];  // their offsets from the unit's first context
  unsigned long long unit;
  unsigned long long unit_local;  // unit index within its spine
  int qn;
  int item_idx;
  int next_item;
  int skip;
  int task_idx;
  int next_task;
  // thread 0's last lookups: the unit ranges of the last task and spine
  unsigned long long lk_task_lo, lk_task_hi, lk_item_lo, lk_item_hi;
  int lk_task, lk_item;
  char post[kThreads / 32][kMaxSize + 8];
};

// Hash join tables of a CTA: membership filter, the block's constraint
// values, their context indices and mask widths.  They sit after the
// staged samples in the dynamic shared memory of the launches that run
// join units only (Params::join_off), so that the other launches keep
// their shared memory, and L1 cache, as they were.
struct alignas(16) JoinSmem {
  unsigned long long key[kJoinSlots];
  unsigned ctx[kJoinSlots];
  unsigned bits[kJoinBits / 32];
  unsigned char b[kJoinSlots];  // low-bit mask width of the slot's constraint
  unsigned long long mc;        // AND of the block's masks: the bits joined on
  unsigned long long tag;       // item and context block the tables hold (~0: none)
};

static_assert(offsetof(Smem, item) % 16 == 0, "Smem::item must be 16-byte aligned");
static_assert(alignof(Item) == 16, "Item must be 16-byte aligned");

// ------------------------------------------------------------------ device ops

__host__ __device__ __forceinline__ unsigned long long umin64(unsigned long long a,
                                                             unsigned long long b) {
  return a < b ? a : b;
}

template <class W>
__device__ __forceinline__ W bin_apply(int op, W l, W r) {
  switch (op) {
    case OP_AND: return l & r;
    case OP_OR: return l | r;
    case OP_XOR: return l ^ r;
    case OP_ADD: return l + r;
    case OP_SUB: return l - r;
    default: return l * r;  // OP_MUL
  }
}

template <class W>
__device__ __forceinline__ W un_apply(int op, W x) {
  return op == OP_NOT ? (W)~x : (W)(W(0) - x);
}

// Multiplicative inverse of an odd word modulo 2^bits by Newton iteration
// x <- x (2 - a x), which doubles the number of correct low bits each step.
template <class W>
__host__ __device__ __forceinline__ W odd_inverse(W a) {
  W x = a;  // correct to 3 bits for odd a
#pragma unroll
  for (int i = 0; i < 5; ++i) x *= (W)2 - a * x;
  return x;
}

template <class W>
__device__ __forceinline__ int word_ctz(W w) {
  if (sizeof(W) == 8) return w ? __ffsll((long long)w) - 1 : 64;
  return w ? __ffs((int)w) - 1 : 32;
}

template <class W>
__device__ __forceinline__ int word_popc(W w) {
  return sizeof(W) == 8 ? __popcll((unsigned long long)w) : __popc((unsigned)w);
}

// Push the constraint (y & M) == K through one level y = f(w, x) to a
// constraint on x.  Infeasible constraints become M = 0, K = 1.  Returns
// false if the level is arithmetic and M is not of the form 2^n - 1.
template <class W>
__device__ bool invert_level(const Level& L, W w, W& M, W& K) {
  if (M == 0 && K != 0) return true;
  const bool low = (M & (M + 1)) == 0;
  if (L.kind == 1) {
    const W c = (W)L.c;
    if (L.eps < 0 && c == (W)~W(0)) {  // ~x
      K = (W)~K & M;
      return true;
    }
    if (!low) return false;
    K = (L.eps > 0 ? (W)(K - c) : (W)(c - K)) & M;
    return true;
  }
  switch (L.op) {
    case OP_XOR:
      K = (K ^ w) & M;
      return true;
    case OP_AND:
      if (K & (W)~w) { M = 0; K = 1; }
      else M &= w;
      return true;
    case OP_OR:
      if (w & M & (W)~K) { M = 0; K = 1; }
      else { M &= (W)~w; K &= (W)~w; }
      return true;
    case OP_ADD:
      if (!low) return false;
      K = (W)(K - w) & M;
      return true;
    case OP_SUB:
      if (!low) return false;
      K = (L.small_left ? (W)(w - K) : (W)(K + w)) & M;
      return true;
    case OP_MUL: {
      if (!low) return false;
      const int n = word_popc<W>(M);
      const int e = word_ctz<W>(w);
      if (e >= n) {
        if (K != 0) { M = 0; K = 1; }
        else { M = 0; K = 0; }
        return true;
      }
      if (e > 0 && (K & (((W)1 << e) - 1))) { M = 0; K = 1; return true; }
      const W inv = odd_inverse<W>((W)(w >> e));
      M = (W)(M >> e);
      K = (W)((W)(K >> e) * inv) & M;
      return true;
    }
  }
  return false;
}

template <class W>
__device__ __forceinline__ W level_apply(int kind, int op, int small_left, int eps, W c, W w,
                                         W y) {
  if (kind == 1) return eps > 0 ? (W)(y + c) : (W)(c - y);
  return small_left ? bin_apply<W>(op, w, y) : bin_apply<W>(op, y, w);
}

// Evaluate a postfix expression on one sample row (k words in shared memory).
template <class W>
__device__ W eval_postfix(const char* p, int len, const W* row) {
  W st[kMaxSize + 1];
  int sp = -1;
  for (int j = 0; j < len; ++j) {
    const char ch = p[j];
    const int op = char_op(ch);
    if (op < 0) {
      st[++sp] = row[ch - '0'];
    } else if (is_unary(op)) {
      st[sp] = un_apply<W>(op, st[sp]);
    } else {
      const W r = st[sp--];
      st[sp] = bin_apply<W>(op, st[sp], r);
    }
  }
  return st[0];
}

// Single-thread verification on every sample (used when the queue is full).
template <class W>
__device__ bool thread_verify(const InstDesc<W>& d, const Smem& sm, const W* s_in, const W* s_out,
                              unsigned long long rank) {
  char post[kMaxSize + 1];
  unrank(rank, d.size, (const uint64_t(*)[kCols])sm.counts, post);
  for (int i = 0; i < d.S; ++i)
    if (eval_postfix<W>(post, d.size, s_in + i * d.K) != s_out[i]) return false;
  return true;
}

// The quantity whose minimum is the answer: the rank, or in RTid order the
// rank's position off + t in its operator block (t = (rank - off) / C mod N).
template <class W>
__device__ __forceinline__ unsigned long long match_key(const InstDesc<W>& d, unsigned long long rank) {
  if (!d.rtid) return rank;
  const unsigned long long* c = d.counts + (size_t)d.size * kCols;
  unsigned long long off = 0;
  int op = 0;
  while (op < 7 && rank - off >= c[op]) off += c[op++];
  return off + mulmod64(rank - off, d.rt_inv[op], c[op]);
}

// RTid: end of the operator block that holds `key`; spines starting there
// or later can only give larger keys.
template <class W>
__device__ __forceinline__ unsigned long long rtid_block_end(const InstDesc<W>& d, unsigned long long key) {
  const unsigned long long* c = d.counts + (size_t)d.size * kCols;
  unsigned long long end = 0;
  for (int op = 0; op < 8; ++op) {
    end += c[op];
    if (key < end) break;
  }
  return end;
}

// Record a verified match: the minimum rank (key), and in batch mode the
// time of the instance's first match.
template <class W>
__device__ __forceinline__ void note_match(const InstDesc<W>& d, unsigned long long rank) {
  const unsigned long long prev = atomicMin(d.best, match_key<W>(d, rank));
  if (prev == ~0ULL && d.ns) atomicCAS(d.ns, 0ULL, globaltimer_ns());
}

// Warp-cooperative verification of the queued sample-0 matches: lane i
// checks samples i, i+32, ...; a ballot after each group of 32 samples
// rejects the candidate at the first mismatch.
template <class W>
__device__ void verify_queue(const InstDesc<W>& d, Smem& sm, const W* s_in, const W* s_out) {
  const int nq = min(sm.qn, kQueue);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int h = warp; h < nq; h += kThreads / 32) {
    const unsigned long long rank = sm.queue[h];
    unsigned long long cur = 0;
    if (lane == 0) cur = *(volatile unsigned long long*)d.best;
    cur = __shfl_sync(0xffffffffu, cur, 0);
    if (match_key<W>(d, rank) >= cur) continue;
    char* post = sm.post[warp];
    if (lane == 0) unrank(rank, d.size, (const uint64_t(*)[kCols])sm.counts, post);
    __syncwarp();
    bool all_ok = true;
    for (int base = 0; base < d.S; base += 32) {
      const int i = base + lane;
      bool ok = true;
      if (i < d.S) ok = eval_postfix<W>(post, d.size, s_in + i * d.K) == s_out[i];
      if (__ballot_sync(0xffffffffu, !ok)) { all_ok = false; break; }
    }
    if (all_ok && lane == 0) note_match<W>(d, rank);
    __syncwarp();
  }
}

// Decode context index c into small-side indices (deepest level fastest)
// and return its rank base; optionally fetch the small values.
template <class W>
__device__ __forceinline__ unsigned long long decode_context(const InstDesc<W>& d, const Item& it,
                                                             unsigned long long c, W* wl,
                                                             const W* const* tabs = nullptr) {
  if (!tabs) tabs = d.tab;
  unsigned long long rank = it.base;
  for (int l = it.depth - 1; l >= 0; --l) {
    const Level& L = it.lv[l];
    if (L.kind != 0) continue;
    unsigned long long idx;
    if ((c >> 32) == 0 && (L.nsmall >> 32) == 0) {  // 32-bit division when it fits
      const unsigned c32 = (unsigned)c, n32 = (unsigned)L.nsmall;
      const unsigned q = c32 / n32;
      idx = c32 - q * n32;
      c = q;
    } else {
      idx = c % L.nsmall;
      c /= L.nsmall;
    }
    rank += idx * L.coef;
    if (wl) wl[l] = tabs[L.ts][idx];
  }
  return rank;
}

template <class W>
__device__ __forceinline__ void push_hit(const Params<W>& p, const InstDesc<W>& d, Smem& sm,
                                         const W* s_in, const W* s_out, unsigned long long rank) {
  const int i = atomicAdd(&sm.qn, 1);
  if (i < kQueue) {
    sm.queue[i] = rank;
  } else {
    atomicAdd(&p.flags[2], 1);
    if (thread_verify<W>(d, sm, s_in, s_out, rank)) note_match<W>(d, rank);
  }
}

template <class W>
struct Explicit {
  int kind[kMaxExplicit], op[kMaxExplicit], sl[kMaxExplicit], eps[kMaxExplicit];
  W c[kMaxExplicit];
};

// Bottom-up evaluation of the levels the inversion could not absorb.
template <class W, int E>
__device__ __forceinline__ W eval_explicit(const Explicit<W>& X, const W* w, W x) {
  W y = x;
#pragma unroll
  for (int j = E - 1; j >= 0; --j) y = level_apply<W>(X.kind[j], X.op[j], X.sl[j], X.eps[j], X.c[j], w[j], y);
  return y;
}

// One work unit: kR contexts per thread x a strided share of the bottom
// values.  Loads are 16-byte vectors of the bottom table, four in flight per
// thread.  FUSED units take their contexts from the materialised list.
// Further filters for a sample-0 match (context c, bottom index v): the same
// spine inverted against samples 1..kExtra, from their value tables.  Exact
// like the first (a rejected candidate does not match that sample); they
// spare the unrank-and-evaluate verification the candidates whose sample-0
// mask is sparse (spines under nested & and |).  Passes what it cannot decide.
template <class W>
__device__ __forceinline__ bool extra_check(const InstDesc<W>& d, const Item& it, unsigned long long c,
                                            unsigned long long v) {
  for (int j = 0; j < kExtra; ++j) {
    const W* const* tb = d.tabx[j];
    if (!tb[it.bottom]) break;
    for (int l = 0; l < it.depth; ++l)  // filter tables may stop below the tabled size
      if (it.lv[l].kind == 0 && !tb[it.lv[l].ts]) return true;
    W wl[kMaxDepth];
    decode_context<W>(d, it, c, wl, tb);
    W m = (W)~W(0), k = d.targetx[j];
    bool ok = true;
    for (int l = 0; l < it.inv && ok; ++l) ok = invert_level<W>(it.lv[l], wl[l], m, k);
    if (!ok) return true;
    W y = tb[it.bottom][v];
    for (int l = it.depth - 1; l >= it.inv; --l) {  // explicit levels, bottom-up
      const Level& Lv = it.lv[l];
      y = level_apply<W>(Lv.kind, Lv.op, Lv.small_left, Lv.eps, (W)Lv.c, wl[l], y);
    }
    if ((W)(y & m) != k) return false;
  }
  return true;
}

// Rank of candidate (context c, bottom index v) of the item; for a fused
// item c indexes the materialised contexts.
template <class W>
__device__ __forceinline__ unsigned long long candidate_rank(const Params<W>& p, const InstDesc<W>& d,
                                                             const Item& it, unsigned long long c,
                                                             unsigned long long v) {
  if (it.fused) {
    const Ctx<W> cx = p.ctxs[it.ctx_off + c];
    return cx.base + v * p.sitems[cx.member].coefv;
  }
  return decode_context<W>(d, it, c, nullptr) + v * it.coefv;
}

// A sample-0 match is queued (context, bottom index) for the filter samples,
// which run after the work unit (filter_queue), so that the search loop keeps
// only this small inlined step; on overflow it goes straight to verification.
template <class W>
__device__ __forceinline__ void pre_push(const Params<W>& p, const InstDesc<W>& d, Smem& sm, const Item& it,
                                         unsigned long long c, unsigned long long v, const W* s_in,
                                         const W* s_out) {
  if (p.preq) {
    // a context or bottom index beyond 32 bits (deep spines, huge tables)
    // skips the queue and goes straight to verification
    if ((c >> 32) == 0 && (v >> 32) == 0) {
      const int i = atomicAdd(&sm.pn, 1);
      if (i < kPreG) {
        p.preq[(size_t)blockIdx.x * kPreG + i] = c << 32 | v;
        return;
      }
    }
  } else if (const int i = atomicAdd(&sm.pn, 1); i < kPre) {
    sm.pre_c[i] = c;
    sm.pre_v[i] = v;
    return;
  }
  push_hit<W>(p, d, sm, s_in, s_out, candidate_rank<W>(p, d, it, c, v));
}

// All threads: run the filter samples on the queued sample-0 matches of the
// unit's item and queue the survivors for verification.
template <class W>
__device__ void filter_queue(const Params<W>& p, const InstDesc<W>& d, Smem& sm, const W* s_in,
                             const W* s_out) {
  const int n = min(sm.pn, p.preq ? kPreG : kPre);
  const Item& it = sm.item;
  const unsigned long long* gq = p.preq ? p.preq + (size_t)blockIdx.x * kPreG : nullptr;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    const unsigned long long c = gq ? gq[i] >> 32 : sm.pre_c[i];
    const unsigned long long v = gq ? gq[i] & 0xFFFFFFFFULL : sm.pre_v[i];
    bool pass;
    if (it.fused) {
      const Ctx<W> cx = p.ctxs[it.ctx_off + c];
      pass = extra_check<W>(d, p.sitems[cx.member], cx.c, v);
    } else {
      pass = extra_check<W>(d, it, c, v);
    }
    if (pass) push_hit<W>(p, d, sm, s_in, s_out, candidate_rank<W>(p, d, it, c, v));
  }
}

// Sample-0 constraint (v & M) == K on the bottom value of context c, from the
// levels the inversion absorbs; the small values of the explicit levels go
// to wx.  M = 0 with K != 0: no bottom value can match.
template <class W, int E, bool FUSED>
__device__ __forceinline__ void context_constraint(const Params<W>& p, const InstDesc<W>& d,
                                                   const Item& it, unsigned long long c, W& m, W& k,
                                                   W* wx) {
  if (FUSED) {
    const Ctx<W> cx = p.ctxs[it.ctx_off + c];
    m = cx.M;
    k = cx.K;
    return;
  }
  W wl[kMaxDepth];
  decode_context<W>(d, it, c, wl);
  m = (W)~W(0);
  k = d.target;
  for (int l = 0; l < it.inv; ++l)
    if (!invert_level<W>(it.lv[l], wl[l], m, k)) atomicOr(&p.flags[1], 1);
  if (E > 0 && wx) {
#pragma unroll
    for (int j = 0; j < (E > 0 ? E : 1); ++j) wx[j] = wl[it.inv + j];
  }
}

// One explicit level with its operator fixed at compile time (XOP >= 0):
// 0 &, 1 |, 2 ^, 3 +, 4 y - w, 5 w - y, 6 *, 7 y + c, 8 c - y.
template <class W, int XOP>
__device__ __forceinline__ W xop_apply(W c, W w, W y) {
  if (XOP == 0) return y & w;
  if (XOP == 1) return y | w;
  if (XOP == 2) return y ^ w;
  if (XOP == 3) return y + w;
  if (XOP == 4) return y - w;
  if (XOP == 5) return w - y;
  if (XOP == 6) return y * w;
  if (XOP == 7) return y + c;
  return c - y;
}

template <class W, int E, bool FULL, bool FUSED, int XOP = -1>
__device__ void process_unit(const Params<W>& p, const InstDesc<W>& d, Smem& sm, const Item& it,
                             unsigned long long local, const W* s_in, const W* s_out) {
  constexpr int VW = 16 / sizeof(W);
  constexpr int EE = E > 0 ? E : 1;
  const unsigned long long cblk = local / it.vblocks;
  const unsigned long long vblk = local - cblk * it.vblocks;
  const unsigned long long cbase = cblk * it.cb;  // the unit's first context
  const unsigned ncu = (unsigned)umin64(it.cb, it.nctx - cbase);

  // Contexts that no bottom value can complete to a sample-0 match (the
  // inversion ended with M = 0, K != 0: an & whose small value lacks a bit
  // the constraint needs, an | that sets a bit it must not) are decided here
  // without reading the bottom table; on random targets most contexts under
  // an & or | are such.  The live ones are listed in shared memory and, when
  // the list holds them all, the CTA's threads are laid out over them alone:
  // ceil(live / kR) groups, the rest of the threads as value lanes.
  // A compacted context list (fused == 2) holds live contexts only.
  const bool all_live = FUSED && it.fused == 2;
  if (!all_live) {
    if (threadIdx.x == 0) sm.nlive = 0;
    __syncthreads();
    for (unsigned j = threadIdx.x; j < ncu; j += blockDim.x) {
      W m, k;
      context_constraint<W, E, FUSED>(p, d, it, cbase + j, m, k, nullptr);
      if (!(m == 0 && k != 0)) {
        const int i = atomicAdd(&sm.nlive, 1);
        if (i < kLive) sm.live[i] = (unsigned short)j;
      }
    }
    __syncthreads();
  }
  const int nlive = all_live ? (int)ncu : sm.nlive;
  if (nlive == 0) return;
  const bool listed = !all_live && nlive <= kLive;
  const int L = listed ? kThreads / ((nlive + kR - 1) / kR) : (int)it.L;
  const int g = threadIdx.x / L, lane = threadIdx.x - g * L;
  // context of slot r of this thread: the listed live contexts in list
  // order, or the unit's contexts in index order (dead ones stay dead)
  auto ctx_at = [&](int r) -> unsigned long long {
    const int s = g * kR + r;
    if (listed) return cbase + sm.live[s < nlive ? s : 0];
    return cbase + (unsigned long long)(s < (int)ncu ? s : 0);
  };
  const int nslots = listed ? nlive : (int)ncu;

  W M[kR], K[kR], WX[kR][EE];
  unsigned valid = 0;
  Explicit<W> X;
  if (E > 0) {
#pragma unroll
    for (int j = 0; j < EE; ++j) {
      const Level& Lv = it.lv[it.inv + j];
      X.kind[j] = Lv.kind;
      X.op[j] = Lv.op;
      X.sl[j] = Lv.small_left;
      X.eps[j] = Lv.eps;
      X.c[j] = (W)Lv.c;
    }
  }
#pragma unroll
  for (int r = 0; r < kR; ++r) {
    W wx[EE];
    context_constraint<W, E, FUSED>(p, d, it, ctx_at(r), M[r], K[r], wx);
    if (g * kR + r < nslots && !(M[r] == 0 && K[r] != 0)) {
      valid |= 1u << r;
    } else {  // padding and dead contexts: a constraint nothing satisfies
      M[r] = 0;
      K[r] = 1;
    }
    if (E > 0) {
#pragma unroll
      for (int j = 0; j < EE; ++j) WX[r][j] = wx[j];
    }
  }

  const W* V = d.tab[it.bottom];
  const unsigned long long v0 = item_voff(it) + vblk * it.vb;
  const unsigned long long v1 = umin64(v0 + it.vb, item_voff(it) + it.nv);
  const unsigned long long q0 = v0 / VW, q1 = (v1 + VW - 1) / VW;
  const uint4* V4 = reinterpret_cast<const uint4*>(V);
  if (threadIdx.x == 0 && p.live) atomicAdd(p.live, (unsigned long long)nlive * (v1 - v0));

  // First pass on the low 32 bits only (64-bit words): the low half of every
  // level's result (bitwise operators, +, -, *, x -> +-x + c) depends only on
  // the low halves of its operands, so a candidate whose low halves fail the
  // masked compare cannot match.  The rare survivors are compared in full.
  using H = unsigned;
  Explicit<H> XH;
  if (E > 0) {
#pragma unroll
    for (int j = 0; j < EE; ++j) {
      XH.kind[j] = X.kind[j];
      XH.op[j] = X.op[j];
      XH.sl[j] = X.sl[j];
      XH.eps[j] = X.eps[j];
      XH.c[j] = (H)X.c[j];
    }
  }
  // Masked compares without explicit levels: the low 16 bits of two bottom
  // values share one 32-bit word (yp), each context's low 16 mask and key bits
  // are doubled the same way, z = (yp & Mp) ^ Kp has a zero half exactly where
  // a candidate's low 16 bits pass, and (z - 0x00010001) & ~z keeps bit 15 or
  // 31 set iff a half is zero (the borrow of a zero half sets its top bit; a
  // nonzero half never does, and borrows cannot cross from a nonzero low
  // half).  One subtraction and two bitwise operations test two candidates.
  // A 16-bit window passes a random value with probability 2^-(mask bits in
  // it): a thread's 16-bit tests of one 16-byte load (2 values x kR
  // contexts) let something through with probability about
  // 2 * sum_r 2^-bits_r, and a pass costs the 32-bit tests of those
  // candidates.  The packed test pays while that probability stays under
  // ~0.25 (16 bitwise operations instead of 32 per load, plus the passes);
  // warps with a thread above it (sparse masks, e.g. an & with a small value
  // of few bits) take the 32-bit test throughout.  The choice is uniform
  // across the warp.
  constexpr bool PACK = SIMBA_NESTED_PACK16 && E == 0 && !FULL;
  unsigned Mp[PACK ? kR : 1], Kp[PACK ? kR : 1];
  bool use_pack = false;
  if (PACK) {
    float pass = 0.f;
#pragma unroll
    for (int r = 0; r < kR; ++r) {
      const unsigned m16 = (unsigned)M[r] & 0xFFFFu, k16 = (unsigned)K[r] & 0xFFFFu;
      Mp[r] = m16 | (m16 << 16);
      Kp[r] = k16 | (k16 << 16);
      if (valid >> r & 1) pass += __int_as_float((127 - __popc(m16)) << 23);  // 2^-bits
    }
    use_pack = SIMBA_PACK_ALWAYS || __all_sync(0xFFFFFFFFu, 2.f * pass < 0.25f);
  }
  // z - 0x00010001 as z * one + 0xFFFEFFFF with `one` unknown to the
  // compiler: a multiply-add, which runs on the FMA pipe, so that the ALU
  // pipe keeps only the two bitwise operations of each context test
  const unsigned one = SIMBA_PACK_IMAD ? *(volatile unsigned*)&sm.one : 1u;
  auto test = [&](const uint4& raw, unsigned long long q) {
    W xs[VW];
    memcpy(xs, &raw, 16);
    bool hit = false;
    // independent accumulators: the or-chains of the contexts run in parallel
    if (PACK && use_pack) {
      unsigned acc[4] = {0u, 0u, 0u, 0u};
#pragma unroll
      for (int e = 0; e < VW; e += 2) {
        const unsigned yp = __byte_perm((unsigned)xs[e], (unsigned)xs[e + 1], 0x5410);
#pragma unroll
        for (int r = 0; r < kR; ++r) {
          const unsigned z = (yp & Mp[r]) ^ Kp[r];
          acc[r & 3] |= (z * one + 0xFFFEFFFFu) & ~z;
        }
      }
      hit = ((acc[0] | acc[1] | acc[2] | acc[3]) & 0x80008000u) != 0;
    } else {
      bool h4[4] = {false, false, false, false};
#pragma unroll
      for (int e = 0; e < VW; ++e) {
#pragma unroll
        for (int r = 0; r < kR; ++r) {
          H y = (H)xs[e];
          if (E > 0) {
            H wh[EE];
#pragma unroll
            for (int j = 0; j < EE; ++j) wh[j] = (H)WX[r][j];
            y = XOP >= 0 ? xop_apply<H, (XOP < 0 ? 0 : XOP)>(XH.c[0], wh[0], y) : eval_explicit<H, E>(XH, wh, y);
          }
          h4[r & 3] |= FULL ? (y == (H)K[r]) : ((H)(y & (H)M[r]) == (H)K[r]);
        }
      }
      hit = h4[0] | h4[1] | h4[2] | h4[3];
    }
    if (!hit) return;
    for (int e = 0; e < VW; ++e) {
      const unsigned long long v = q * VW + e;
      if (v < v0 || v >= v1) continue;
      for (int r = 0; r < kR; ++r) {
        if (!(valid >> r & 1)) continue;
        W y = xs[e];
        if (E > 0)
          y = XOP >= 0 ? xop_apply<W, (XOP < 0 ? 0 : XOP)>(X.c[0], WX[r][0], y) : eval_explicit<W, E>(X, WX[r], y);
        const bool h = FULL ? (y == K[r]) : ((W)(y & M[r]) == K[r]);
        if (h) pre_push<W>(p, d, sm, it, ctx_at(r), v, s_in, s_out);
      }
    }
  };

  // The bottom values are streamed with four 16-byte loads in flight.
  if (!valid) return;  // after the warp-wide vote: no live context in this thread
  unsigned long long q = q0 + lane;
  const unsigned long long step = (unsigned long long)L;
  {
#if SIMBA_NESTED_PIPELINE
    if (E == 0) {
    // software pipeline: the next four loads are issued before the current
    // four are tested, so the tests overlap their latency
    if (q + 3 * step < q1) {
      uint4 a0 = __ldg(V4 + q), a1 = __ldg(V4 + q + step);
      uint4 a2 = __ldg(V4 + q + 2 * step), a3 = __ldg(V4 + q + 3 * step);
      for (; q + 7 * step < q1; q += 4 * step) {
        const uint4 b0 = __ldg(V4 + q + 4 * step), b1 = __ldg(V4 + q + 5 * step);
        const uint4 b2 = __ldg(V4 + q + 6 * step), b3 = __ldg(V4 + q + 7 * step);
        test(a0, q);
        test(a1, q + step);
        test(a2, q + 2 * step);
        test(a3, q + 3 * step);
        a0 = b0;
        a1 = b1;
        a2 = b2;
        a3 = b3;
      }
      test(a0, q);
      test(a1, q + step);
      test(a2, q + 2 * step);
      test(a3, q + 3 * step);
      q += 4 * step;
    }
    }
#else
    for (; q + 3 * step < q1; q += 4 * step) {
      const uint4 a0 = __ldg(V4 + q);
      const uint4 a1 = __ldg(V4 + q + step);
      const uint4 a2 = __ldg(V4 + q + 2 * step);
      const uint4 a3 = __ldg(V4 + q + 3 * step);
      test(a0, q);
      test(a1, q + step);
      test(a2, q + 2 * step);
      test(a3, q + 3 * step);
    }
#endif
  }
  for (; q < q1; q += step) test(__ldg(V4 + q), q);
}

// Materialise the contexts of the spines listed in p.sitems: one thread per
// context writes its fully inverted constraint and rank coefficients.
template <class W>
__global__ void __launch_bounds__(256) materialize_kernel(Params<W> p, Ctx<W>* out) {
  for (unsigned long long gi = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; gi < p.nctxs;
       gi += (unsigned long long)gridDim.x * blockDim.x) {
    int lo = 0, hi = p.nsitems - 1;
    unsigned long long key = gi;
    int inst = -1;
    if (p.tasks) {  // batch: the task owning context gi, then its shared list
      int tl = 0, th = p.ntasks - 1;
      while (tl < th) {
        const int mid = (tl + th + 1) >> 1;
        if (p.tasks[mid].ctx_base <= gi) tl = mid;
        else th = mid - 1;
      }
      const Task tk = p.tasks[tl];
      const TmplDesc td = p.tmpls[tk.tmpl];
      key = gi - tk.ctx_base;
      lo = (int)td.small_off;
      hi = (int)(td.small_off + td.nsmall) - 1;
      inst = (int)tk.inst;
    }
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (p.sitems[mid].ctx_off <= key) lo = mid;
      else hi = mid - 1;
    }
    const Item& it = p.sitems[lo];
    const InstDesc<W>& d = p.insts[inst >= 0 ? inst : (int)it.inst];
    const unsigned long long c = key - it.ctx_off;
    W wl[kMaxDepth];
    Ctx<W> cx;
    cx.base = decode_context<W>(d, it, c, wl);
    cx.member = (unsigned)lo;
    cx.c = (unsigned)c;
    W m = (W)~W(0), k = d.target;
    for (int l = 0; l < it.depth; ++l)
      if (!invert_level<W>(it.lv[l], wl[l], m, k)) atomicOr(&p.flags[1], 1);
    cx.M = m;
    cx.K = k;
    if (p.ctx_live) {  // compacted lists: only contexts some bottom value can complete
      if (m == 0 && k != 0) continue;
      unsigned long long* gl = p.ctx_live + 2 * it.group;
      out[gl[1] + atomicAdd(gl, 1ULL)] = cx;
    } else {
      out[gi] = cx;
    }
  }
}

// Generic unit for spines with more than kMaxExplicit explicit levels:
// straightforward bottom-up evaluation of every level, one context at a time.
template <class W>
__device__ void process_unit_generic(const Params<W>& p, const InstDesc<W>& d, Smem& sm,
                                     const Item& it, unsigned long long local, const W* s_in,
                                     const W* s_out) {
  const unsigned long long cblk = local / it.vblocks;
  const unsigned long long vblk = local - cblk * it.vblocks;
  const int L = it.L;
  const int g = threadIdx.x / L, lane = threadIdx.x % L;
  const unsigned long long v0 = item_voff(it) + vblk * it.vb;
  const unsigned long long v1 = umin64(v0 + it.vb, item_voff(it) + it.nv);
  const W* V = d.tab[it.bottom];
  for (int r = 0; r < kR; ++r) {
    const unsigned long long c = cblk * it.cb + (unsigned long long)g * kR + r;
    if (c >= it.nctx) break;
    W wl[kMaxDepth];
    const unsigned long long rb = decode_context<W>(d, it, c, wl);
    for (unsigned long long v = v0 + lane; v < v1; v += L) {
      W y = V[v];
      for (int l = it.depth - 1; l >= 0; --l) {
        const Level& Lv = it.lv[l];
        y = level_apply<W>(Lv.kind, Lv.op, Lv.small_left, Lv.eps, (W)Lv.c, wl[l], y);
      }
      if (y != d.target) continue;
      (void)rb;
      pre_push<W>(p, d, sm, it, c, v, s_in, s_out);
    }
  }
}

// 32-bit mix of a value; its top 14 bits index the filter, the top 10 the table
__device__ __forceinline__ unsigned join_hash(unsigned long long y) {
  const unsigned x = (unsigned)y ^ ((unsigned)(y >> 32) * 0x9E3779B1u);
  return x * 0x85EBCA6Bu;
}

// A spine without & and | levels inverts every context to v & M == K with M
// a low-bit mask (all ones unless a * level's small value is even), so
// matching a block of contexts against all bottom values is a hash join on
// the low bits Mc that all the block's masks keep: the contexts' K & Mc go
// into a shared-memory filter (one bit per hash) and table (linear probing,
// load <= 1/2), every bottom value tests the filter with v & Mc and, rarely,
// probes the table, and a table entry matches when v & M == K for its own
// mask.  A block with a context of a narrow mask (a small value 0 makes
// M = 0) joins on few bits and probes long chains: slower, still exact.  A
// match is an exact sample-0 match and goes to the match queue like any
// other; contexts whose K has bits outside M can never match and are left
// out.
template <class W, bool FUSED>
__device__ void process_unit_join(const Params<W>& p, const InstDesc<W>& d, Smem& sm, JoinSmem& js,
                                  const Item& it, unsigned long long local, const W* s_in,
                                  const W* s_out) {
  static_assert(kJoinBits == 1 << 14 && kJoinSlots == 1 << 10 && kJoinCtx * 2 <= kJoinSlots,
                "filter and table index widths");
  static_assert(kJoinCtx <= 2 * kThreads, "two contexts per thread at most");
  constexpr int WB = 8 * (int)sizeof(W);
  // value-block major: consecutive units (on other CTAs) share a value
  // block, which then comes from L2 for every context block after the first
  const unsigned long long vblk = local / it.cblocks, cblk = local - vblk * it.cblocks;
  const unsigned long long c0 = cblk * it.cb;
  const int nc = (int)umin64(it.cb, it.nctx - c0);
  // The tables of a context block stay in shared memory for the CTA's next
  // unit: a single search's units of one fused group with one context block
  // (the largest bottom tables) then skip the whole build.
  const unsigned long long tag =
      p.tasks ? ~0ULL : ((unsigned long long)(unsigned)sm.next_item << 40 | cblk);
  if (tag == ~0ULL || js.tag != tag) {
  for (int i = threadIdx.x; i < kJoinSlots; i += blockDim.x) js.ctx[i] = ~0u;
  for (int i = threadIdx.x; i < kJoinBits / 32; i += blockDim.x) js.bits[i] = 0u;
  if (threadIdx.x == 0) js.mc = ~0ULL;
  __syncthreads();
  if (threadIdx.x == 0) js.tag = tag;  // every thread read the old tag before the barrier
  // 1. constraints of this thread's (at most two) contexts; the common mask
  W ms[2], ks[2];
  bool ok[2];
#pragma unroll
  for (int r = 0; r < 2; ++r) {
    const int j = threadIdx.x + r * blockDim.x;
    ok[r] = false;
    if (j >= nc) continue;
    W m = (W)~W(0), k = d.target;
    if (FUSED) {
      const Ctx<W> cx = p.ctxs[it.ctx_off + c0 + j];
      m = cx.M;
      k = cx.K;
    } else {
      W wl[kMaxDepth];
      decode_context<W>(d, it, c0 + j, wl);
      for (int l = 0; l < it.inv; ++l)
        if (!invert_level<W>(it.lv[l], wl[l], m, k)) atomicOr(&p.flags[1], 1);
    }
    ms[r] = m;
    ks[r] = k;
    ok[r] = (W)(k & ~m) == 0;  // otherwise no bottom value can match
    if (ok[r]) atomicAnd(&js.mc, (unsigned long long)m);
  }
  __syncthreads();
  const unsigned long long mc0 = js.mc;
  const bool lo32b = sizeof(W) == 4 || (unsigned)mc0 == 0xFFFFFFFFu;
  // 2. filter bits and table entries, keyed on K & Mc
#pragma unroll
  for (int r = 0; r < 2; ++r) {
    if (!ok[r]) continue;
    const int j = threadIdx.x + r * blockDim.x;
    const unsigned hx = lo32b ? (unsigned)ks[r] * 0x85EBCA6Bu : join_hash((unsigned long long)ks[r] & mc0);
    atomicOr(&js.bits[hx >> 23], 1u << ((hx >> 18) & 31));
    unsigned h = hx >> 22;
    for (int t = 0; t < kJoinSlots; ++t, h = (h + 1) & (kJoinSlots - 1)) {
      if (atomicCAS(&js.ctx[h], ~0u, (unsigned)j) == ~0u) {
        js.key[h] = (unsigned long long)ks[r];
        js.b[h] = (unsigned char)__popcll((unsigned long long)ms[r]);
        break;
      }
    }
  }
  __syncthreads();
  }
  const unsigned long long mc = js.mc;
  // the block joins on at least the low 32 bits (every mask keeps them: the
  // usual case): the hash reads the low word alone, and the exact key
  // compare on a filter hit settles the rest (same hash as join_hash for
  // 32-bit words)
  const bool lo32 = sizeof(W) == 4 || (unsigned)mc == 0xFFFFFFFFu;
  // 3. probe with every bottom value of the block
  constexpr int VW = 16 / sizeof(W);
  const W* V = d.tab[it.bottom];
  const unsigned long long v0 = item_voff(it) + vblk * it.vb;
  const unsigned long long v1 = umin64(v0 + it.vb, item_voff(it) + it.nv);
  const uint4* V4 = reinterpret_cast<const uint4*>(V);
  auto probe = [&](const uint4& raw, unsigned long long q) {
    W xs[VW];
    memcpy(xs, &raw, 16);
#pragma unroll
    for (int e = 0; e < VW; ++e) {
      const unsigned long long v = q * VW + e;
      const unsigned long long y = (unsigned long long)xs[e];
      const unsigned hx = lo32 ? (unsigned)y * 0x85EBCA6Bu : join_hash(y & mc);
      if (!(js.bits[hx >> 23] >> ((hx >> 18) & 31) & 1u)) continue;
      const unsigned long long ym = y & mc;
      unsigned h = hx >> 22;
      for (int t = 0; t < kJoinSlots; ++t, h = (h + 1) & (kJoinSlots - 1)) {
        const unsigned c = js.ctx[h];
        if (c == ~0u) break;
        const unsigned long long key = js.key[h];
        if ((key & mc) != ym) continue;
        const int b = js.b[h];
        const unsigned long long m = b >= WB ? (unsigned long long)(W)~W(0) : ((1ULL << b) - 1);
        if ((y & m) == key && v >= v0 && v < v1) pre_push<W>(p, d, sm, it, c0 + c, v, s_in, s_out);
      }
    }
  };
  // four 16-byte loads in flight per thread
  const unsigned long long q1 = (v1 + VW - 1) / VW, step = blockDim.x;
  unsigned long long q = v0 / VW + threadIdx.x;
  for (; q + 3 * step < q1; q += 4 * step) {
    const uint4 a0 = __ldg(V4 + q);
    const uint4 a1 = __ldg(V4 + q + step);
    const uint4 a2 = __ldg(V4 + q + 2 * step);
    const uint4 a3 = __ldg(V4 + q + 3 * step);
    probe(a0, q);
    probe(a1, q + step);
    probe(a2, q + 2 * step);
    probe(a3, q + 3 * step);
  }
  for (; q < q1; q += step) probe(__ldg(V4 + q), q);
}

template <class W, int XS>
__device__ void dispatch_unit(const Params<W>& p, const InstDesc<W>& d, Smem& sm, JoinSmem* js,
                              const Item& it, unsigned long long local, const W* s_in,
                              const W* s_out) {
  const int e = it.nexp;
  if (it.full == 2) {
    if (!js) {  // a join unit in a launch without join tables: host error
      if (threadIdx.x == 0) atomicOr(&p.flags[1], 2);
      return;
    }
    if (it.fused) return process_unit_join<W, true>(p, d, sm, *js, it, local, s_in, s_out);
    return process_unit_join<W, false>(p, d, sm, *js, it, local, s_in, s_out);
  }
  if (it.fused) {
    if (it.full) return process_unit<W, 0, true, true>(p, d, sm, it, local, s_in, s_out);
    return process_unit<W, 0, false, true>(p, d, sm, it, local, s_in, s_out);
  }
  if (e > kMaxExplicit) return process_unit_generic<W>(p, d, sm, it, local, s_in, s_out);
  if (it.full) {
    switch (e) {
      case 0: return process_unit<W, 0, true, false>(p, d, sm, it, local, s_in, s_out);
      case 1: return process_unit<W, 1, true, false>(p, d, sm, it, local, s_in, s_out);
      default: return process_unit<W, 2, true, false>(p, d, sm, it, local, s_in, s_out);
    }
  }
  switch (e) {
    case 0: return process_unit<W, 0, false, false>(p, d, sm, it, local, s_in, s_out);
    case 1: {  // the explicit level's operator as a template argument
      if (!XS) return process_unit<W, 1, false, false>(p, d, sm, it, local, s_in, s_out);
      const Level& Lx = it.lv[it.inv];
      if (Lx.kind == 1) {
        if (Lx.eps > 0) return process_unit<W, 1, false, false, 7>(p, d, sm, it, local, s_in, s_out);
        return process_unit<W, 1, false, false, 8>(p, d, sm, it, local, s_in, s_out);
      }
      switch (Lx.op) {
        case OP_AND: return process_unit<W, 1, false, false, 0>(p, d, sm, it, local, s_in, s_out);
        case OP_OR: return process_unit<W, 1, false, false, 1>(p, d, sm, it, local, s_in, s_out);
        case OP_XOR: return process_unit<W, 1, false, false, 2>(p, d, sm, it, local, s_in, s_out);
        case OP_ADD: return process_unit<W, 1, false, false, 3>(p, d, sm, it, local, s_in, s_out);
        case OP_SUB:
          if (Lx.small_left) return process_unit<W, 1, false, false, 5>(p, d, sm, it, local, s_in, s_out);
          return process_unit<W, 1, false, false, 4>(p, d, sm, it, local, s_in, s_out);
        case OP_MUL: return process_unit<W, 1, false, false, 6>(p, d, sm, it, local, s_in, s_out);
        default: return process_unit<W, 1, false, false>(p, d, sm, it, local, s_in, s_out);
      }
    }
    default: return process_unit<W, 2, false, false>(p, d, sm, it, local, s_in, s_out);
  }
}

// Stage one instance's count table and samples into shared memory
// (16-byte vector copies; the device arrays are padded to 16 bytes) and
// return where its outputs start.
template <class W>
__device__ W* stage_samples(const InstDesc<W>& d, Smem& sm, W* s_in) {
  for (int i = threadIdx.x; i < (kMaxSize + 1) * kCols; i += blockDim.x) sm.counts[i] = d.counts[i];
  const int nin = (d.S * d.K * (int)sizeof(W) + 15) / 16;
  const int nout = (d.S * (int)sizeof(W) + 15) / 16;
  W* s_out = s_in + nin * (16 / (int)sizeof(W));
  const uint4* gi = reinterpret_cast<const uint4*>(d.in);
  const uint4* go = reinterpret_cast<const uint4*>(d.out);
  uint4* si = reinterpret_cast<uint4*>(s_in);
  uint4* so = reinterpret_cast<uint4*>(s_out);
  for (int i = threadIdx.x; i < nin; i += blockDim.x) si[i] = gi[i];
  for (int i = threadIdx.x; i < nout; i += blockDim.x) so[i] = go[i];
  return s_out;
}

// Copy instance `idx`'s descriptor into shared memory and stage its samples
// (all threads call it; ends with a barrier).
template <class W>
__device__ W* load_instance(const Params<W>& p, Smem& sm, int idx, W* s_in) {
  const uint4* src = reinterpret_cast<const uint4*>(p.insts + idx);
  uint4* dst = reinterpret_cast<uint4*>(sm.desc);
  for (int i = threadIdx.x; i < (int)(sizeof(InstDesc<W>) / 16); i += blockDim.x) dst[i] = src[i];
  __syncthreads();
  W* s_out = stage_samples<W>(*reinterpret_cast<const InstDesc<W>*>(sm.desc), sm, s_in);
  __syncthreads();
  return s_out;
}

// Persistent search kernel: CTAs take work units from an atomic counter.
template <class W, int XS = SIMBA_XOP_SPECIALIZE>
__global__ void SIMBA_SPINE_BOUNDS spine_kernel(Params<W> p) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  Smem& sm = *reinterpret_cast<Smem*>(smem_raw);
  W* s_in = reinterpret_cast<W*>(smem_raw + ((sizeof(Smem) + 15) & ~size_t(15)));
  W* s_out = s_in;
  JoinSmem* js = p.join_off ? reinterpret_cast<JoinSmem*>(smem_raw + p.join_off) : nullptr;
  const InstDesc<W>& d = *reinterpret_cast<const InstDesc<W>*>(sm.desc);
  if (threadIdx.x == 0) {
    sm.one = 1u;
    sm.qn = 0;
    sm.pn = 0;
    sm.item_idx = -1;
    sm.task_idx = -2;
    sm.inst_idx = -1;
    sm.lk_task = -1;
    sm.lk_item = -1;
    if (js) js->tag = ~0ULL;
  }
  __syncthreads();
  for (;;) {
    if (threadIdx.x == 0) {
      const unsigned long long stride = p.unit_stride ? p.unit_stride : 1ULL;
      unsigned long long u = atomicAdd(p.counter, 1ULL);
      u = u < p.total_units ? u * stride + p.unit_offset : ~0ULL;
      if (u >= p.total_units) u = ~0ULL;
      if (u != ~0ULL && p.budget_ns && globaltimer_ns() - *p.start_ns > p.budget_ns) {
        atomicOr(&p.flags[0], 1);
        u = ~0ULL;
      }
      sm.unit = u;
      if (u != ~0ULL) {
        unsigned long long local = u;
        int ilo = 0, ihi = p.nitems - 1, inst = -1, task = -1;
        if (p.tasks) {  // batch: task, then the spine inside its shared list
          int lo = 0, hi = p.ntasks - 1;
          if (sm.lk_task >= 0 && u >= sm.lk_task_lo && u < sm.lk_task_hi) {
            lo = sm.lk_task;  // units of one task are consecutive: usually a hit
          } else {
            while (lo < hi) {
              const int mid = (lo + hi + 1) >> 1;
              if (p.tasks[mid].unit_begin <= u) lo = mid;
              else hi = mid - 1;
            }
            sm.lk_task = lo;
            sm.lk_task_lo = p.tasks[lo].unit_begin;
            sm.lk_task_hi = lo + 1 < p.ntasks ? p.tasks[lo + 1].unit_begin : p.total_units;
            sm.lk_item = -1;
          }
          task = lo;
          const Task tk = p.tasks[lo];
          const TmplDesc td = p.tmpls[tk.tmpl];
          local = u - tk.unit_begin;
          ilo = (int)td.item_off;
          ihi = (int)(td.item_off + td.nitems) - 1;
          inst = (int)tk.inst;
          if (tk.bucket >= 0) {  // guided: one shape-class bucket of the list
            const int b = tk.bucket;
            const TmplBuckets& tb = p.buckets[td.bucket_off];
            local += tb.unit[b];
            ilo = (int)(td.item_off + tb.item[b]);
            ihi = (int)(td.item_off + tb.item[b + 1]) - 1;
          }
        }
        if (sm.lk_item >= ilo && sm.lk_item <= ihi && local >= sm.lk_item_lo && local < sm.lk_item_hi) {
          ilo = sm.lk_item;
        } else {
          while (ilo < ihi) {
            const int mid = (ilo + ihi + 1) >> 1;
            if (p.items[mid].unit_begin <= local) ilo = mid;
            else ihi = mid - 1;
          }
          sm.lk_item = ilo;
          sm.lk_item_lo = p.items[ilo].unit_begin;
          sm.lk_item_hi = sm.lk_item_lo + item_units(p.items[ilo]);
        }
        sm.next_item = ilo;
        sm.next_task = task;
        sm.unit_local = local - p.items[ilo].unit_begin;
        const Item& nx = p.items[ilo];
        if (inst < 0) inst = (int)nx.inst;
        const InstDesc<W>& di = p.insts[inst];
        const unsigned long long cur = *(volatile unsigned long long*)di.best;
        // 1: minimum rank (skip spines above the best match; in RTid order,
        // spines past the best match's operator block); 2: any match
        if (p.stop_on_match == 1)
          sm.skip = di.rtid ? (cur != ~0ULL && nx.base >= rtid_block_end<W>(di, cur)) : nx.base > cur;
        else
          sm.skip = p.stop_on_match == 2 && cur != ~0ULL;
      }
    }
    __syncthreads();
    const unsigned long long u = sm.unit;
    if (u == ~0ULL) break;
    const int ni = sm.next_item;
    const int nt = sm.next_task;
    if (ni != sm.item_idx || nt != sm.task_idx) {
      const uint4* src = reinterpret_cast<const uint4*>(p.items + ni);
      uint4* dst = reinterpret_cast<uint4*>(&sm.item);
      for (int i = threadIdx.x; i < (int)(sizeof(Item) / 16); i += blockDim.x) dst[i] = src[i];
      __syncthreads();
      if (threadIdx.x == 0 && nt >= 0) {
        const Task tk = p.tasks[nt];
        sm.item.inst = tk.inst;
        if (sm.item.fused) sm.item.ctx_off += tk.ctx_base;
      }
    }
    __syncthreads();
    if (!sm.skip) {
      const Item& it = sm.item;
      if ((int)it.inst != sm.inst_idx) {  // uniform: every thread reads the same values
        s_out = load_instance<W>(p, sm, (int)it.inst, s_in);
        if (threadIdx.x == 0) sm.inst_idx = (int)it.inst;
      }
      const unsigned long long local = sm.unit_local;
      unsigned long long cu = local / it.vblocks, vblk = local - cu * it.vblocks;
      if (it.full == 2) {  // join units are value-block major (cpu = 1)
        vblk = local / it.cblocks;
        cu = local - vblk * it.cblocks;
      }
      const unsigned long long cpu = it.cpu ? it.cpu : 1;
      const unsigned long long b0 = cu * cpu, b1 = umin64(b0 + cpu, it.cblocks);
      for (unsigned long long b = b0; b < b1; ++b) {
        const unsigned long long lb = it.full == 2 ? vblk * it.cblocks + b : b * it.vblocks + vblk;
        dispatch_unit<W, XS>(p, d, sm, js, it, lb, s_in, s_out);
        if (threadIdx.x == 0) {
          const unsigned long long c0 = b * it.cb, c1 = umin64(c0 + it.cb, it.nctx);
          const unsigned long long v0 = vblk * it.vb, v1 = umin64(v0 + it.vb, it.nv);  // a count
          atomicAdd(p.evaluated, (c1 - c0) * (v1 - v0));
        }
        if (b + 1 < b1) {  // filter and verify this block's matches before the next one
          __syncthreads();
          if (sm.pn > 0) filter_queue<W>(p, d, sm, s_in, s_out);
          __syncthreads();
          if (sm.qn > 0) verify_queue<W>(d, sm, s_in, s_out);
          __syncthreads();
          if (threadIdx.x == 0) {
            if (p.hits && sm.qn) atomicAdd(p.hits, (unsigned long long)sm.qn);
            sm.qn = 0;
            sm.pn = 0;
          }
          __syncthreads();
        }
      }
    }
    __syncthreads();
    if (sm.pn > 0) filter_queue<W>(p, d, sm, s_in, s_out);
    __syncthreads();
    if (sm.qn > 0) verify_queue<W>(d, sm, s_in, s_out);
    __syncthreads();
    if (threadIdx.x == 0) {
      if (!sm.skip && d.ns) atomicMax(d.ns + 1, globaltimer_ns());
      if (p.hits && sm.qn) atomicAdd(p.hits, (unsigned long long)sm.qn);
      sm.qn = 0;
      sm.pn = 0;
      sm.item_idx = ni;
      sm.task_idx = nt;
    }
  }
}

// One thread per rank: unrank, evaluate sample 0, verify on a match.  This
// is the reference's per-thread algorithm (nocache.cu:85-107) with the
// count table and samples in shared memory, a grid-stride loop (no gridDim
// overflow) and the minimum matching rank.
template <class W>
__global__ void __launch_bounds__(kThreads) naive_kernel(Params<W> p, unsigned long long lo,
                                                         unsigned long long hi) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  Smem& sm = *reinterpret_cast<Smem*>(smem_raw);
  W* s_in = reinterpret_cast<W*>(smem_raw + ((sizeof(Smem) + 15) & ~size_t(15)));
  W* s_out = load_instance<W>(p, sm, 0, s_in);
  const InstDesc<W>& d = *reinterpret_cast<const InstDesc<W>*>(sm.desc);
  const unsigned long long stride = (unsigned long long)gridDim.x * blockDim.x;
  unsigned long long count = 0;
  char post[kMaxSize + 1];
  for (unsigned long long r = lo + (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; r < hi;
       r += stride) {
    if (p.stop_on_match && !d.rtid && r > *(volatile unsigned long long*)d.best) break;
    if ((count & 1023) == 0 && p.budget_ns && globaltimer_ns() - *p.start_ns > p.budget_ns) {
      atomicOr(&p.flags[0], 1);
      break;
    }
    unrank(r, d.size, (const uint64_t(*)[kCols])sm.counts, post);
    ++count;
    if (eval_postfix<W>(post, d.size, s_in) != s_out[0]) continue;
    bool ok = true;
    for (int i = 1; i < d.S && ok; ++i) ok = eval_postfix<W>(post, d.size, s_in + i * d.K) == s_out[i];
    if (ok) note_match<W>(d, r);
  }
  atomicAdd(p.evaluated, count);
  __syncthreads();
  if (threadIdx.x == 0 && d.ns) atomicMax(d.ns + 1, globaltimer_ns());
}

template <class W>
__global__ void build_unary_kernel(W* out, const W* in, unsigned long long n, int op) {
  for (unsigned long long i = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (unsigned long long)gridDim.x * blockDim.x)
    out[i] = un_apply<W>(op, in[i]);
}

template <class W>
__global__ void build_binary_kernel(W* out, const W* A, const W* B, unsigned long long na,
                                    unsigned long long nb, int op) {
  const unsigned long long n = na * nb;
  for (unsigned long long i = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (unsigned long long)gridDim.x * blockDim.x) {
    const unsigned long long a = i / nb;
    out[i] = bin_apply<W>(op, A[a], B[i - a * nb]);
  }
}

// One table-building job of the batch: a unary (nb = 1, B unused) or binary
// operator block of one instance's V_t.
template <class W>
struct BuildJob {
  W* out;
  const W* A;
  const W* B;
  unsigned long long na, nb;
  int op;
  int pad;
  unsigned long long begin;  // first global entry of this job
};

template <class W>
__global__ void build_batch_kernel(const BuildJob<W>* jobs, int njobs, unsigned long long total) {
  int cur = -1;  // the last job found: a thread's strided entries stay in it for a while
  unsigned long long cur_lo = 1, cur_hi = 0;
  for (unsigned long long g = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; g < total;
       g += (unsigned long long)gridDim.x * blockDim.x) {
    if (g < cur_lo || g >= cur_hi) {
      int lo = 0, hi = njobs - 1;
      while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (jobs[mid].begin <= g) lo = mid;
        else hi = mid - 1;
      }
      cur = lo;
      cur_lo = jobs[lo].begin;
      cur_hi = lo + 1 < njobs ? jobs[lo + 1].begin : total;
    }
    const BuildJob<W>& j = jobs[cur];
    const unsigned long long i = g - j.begin;
    if (is_unary(j.op)) {
      j.out[i] = un_apply<W>(j.op, j.A[i]);
    } else {
      const unsigned long long a = i / j.nb;
      j.out[i] = bin_apply<W>(j.op, j.A[a], j.B[i - a * j.nb]);
    }
  }
}

static __global__ void stamp_start_kernel(unsigned long long* t) { *t = globaltimer_ns(); }

// Batch start: instance i's terminals on sample j (row ns*i + j of src, maxK
// wide) go to its V_1 table at byte offset dst[ns*i + j] (~0: no such table).
template <class W>
__global__ void scatter_terminals_kernel(const W* src, const unsigned long long* dst, const int* k,
                                         char* base, int n, int maxK, int ns) {
  const unsigned long long total = (unsigned long long)ns * n * maxK;
  for (unsigned long long g = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; g < total;
       g += (unsigned long long)gridDim.x * blockDim.x) {
    const unsigned long long row = g / maxK;
    const int q = (int)(g - row * maxK);
    const int i = (int)(row / ns);
    if (q >= k[i] || dst[row] == ~0ULL) continue;
    reinterpret_cast<W*>(base + dst[row])[q] = src[g];
  }
}

// ------------------------------------------------------------------ host side

struct ChainClass {
  int eps;
  int64_t c;
  uint64_t off;
};

struct Enumerator {
  const CountTable* ct;
  int T;
  uint64_t mask;
  std::vector<Item>* items;
  bool too_deep = false;

  uint64_t N(int s) const { return ct->n[s][8]; }

  int chain_start = 0;  // size where the current unary chain began

  void emit(int size, std::vector<Level>& lv, uint64_t mult, uint64_t base, const ChainClass& k) {
    if (lv.size() + (k.eps == 1 && k.c == 0 ? 0 : 1) > (size_t)kMaxDepth) {
      too_deep = true;
      return;
    }
    Item it;
    memset(&it, 0, sizeof(it));
    int d = 0;
    for (auto& L : lv) it.lv[d++] = L;
    if (!(k.eps == 1 && k.c == 0)) {
      Level L;
      memset(&L, 0, sizeof(L));
      L.kind = 1;
      L.eps = (int8_t)k.eps;
      L.c = (uint64_t)k.c & mask;
      L.nsmall = 1;
      L.chain_len = (int8_t)(chain_start - size);
      it.lv[d++] = L;
    }
    it.depth = (int8_t)d;
    it.bottom = (int8_t)size;
    it.base = base + k.off;
    it.coefv = mult;
    it.nv = N(size);
    items->push_back(it);
  }

  void rec(int size, std::vector<Level>& lv, uint64_t mult, uint64_t base,
           const std::vector<ChainClass>& cls) {
    if (too_deep) return;
    if (size <= T) {
      for (auto& k : cls) emit(size, lv, mult, base, k);
      return;
    }
    if (lv.size() >= (size_t)kMaxDepth) {
      too_deep = true;
      return;
    }
    // Unary blocks: extend every chain class by ~ (x -> -x - 1) or neg
    // (x -> -x), keeping the smallest rank offset per resulting map.
    const uint64_t off_not = op_offset(ct->n, size, OP_NOT);
    const uint64_t off_neg = op_offset(ct->n, size, OP_NEG);
    std::vector<ChainClass> ncls;
    auto add = [&](int eps, int64_t c, uint64_t off) {
      for (auto& x : ncls)
        if (x.eps == eps && x.c == c) {
          x.off = std::min(x.off, off);
          return;
        }
      ncls.push_back({eps, c, off});
    };
    for (auto& k : cls) {
      add(-k.eps, k.c - k.eps, k.off + off_not * mult);
      add(-k.eps, k.c, k.off + off_neg * mult);
    }
    rec(size - 1, lv, mult, base, ncls);
    const int my_chain_start = chain_start;
    // Binary blocks in rank order.
    const int sub = size - 1;
    for (int op = 0; op < 8; ++op) {
      if (is_unary(op)) continue;
      uint64_t boff = op_offset(ct->n, size, op);
      const int fmax = is_commutative(op) ? sub / 2 : sub - 1;
      for (int f = 1; f <= fmax; ++f) {
        const int i = f, j = sub - f;
        for (auto& k : cls) {
          std::vector<Level> lv2 = lv;
          if (!(k.eps == 1 && k.c == 0)) {
            Level C;
            memset(&C, 0, sizeof(C));
            C.kind = 1;
            C.eps = (int8_t)k.eps;
            C.c = (uint64_t)k.c & mask;
            C.nsmall = 1;
            C.chain_len = (int8_t)(my_chain_start - size);
            lv2.push_back(C);
          }
          Level B;
          memset(&B, 0, sizeof(B));
          B.kind = 0;
          B.op = (int8_t)op;
          uint64_t nmult;
          int big;
          if (j >= i) {  // small = left operand
            B.small_left = 1;
            B.ts = (int8_t)i;
            B.coef = mult * N(j);
            nmult = mult;
            big = j;
          } else {  // small = right operand
            B.small_left = 0;
            B.ts = (int8_t)j;
            B.coef = mult;
            nmult = mult * N(j);
            big = i;
          }
          B.nsmall = N(B.ts);
          lv2.push_back(B);
          if (lv2.size() > (size_t)kMaxDepth) {
            too_deep = true;
            return;
          }
          std::vector<ChainClass> id{{1, 0, 0}};
          chain_start = big;
          rec(big, lv2, nmult, base + k.off + boff * mult, id);
          chain_start = my_chain_start;
        }
        boff += N(i) * N(j);
      }
    }
  }
};

// Structural inversion depth: levels are inverted top-down until the first
// arithmetic level that lies below an & or | (its constraint mask is then
// not of the form 2^n - 1).
static inline void finish_structure(Item& it, uint64_t mask) {
  int inv = it.depth;
  bool andor = false, full = true;
  for (int l = 0; l < it.depth; ++l) {
    const Level& L = it.lv[l];
    const bool notchain = L.kind == 1 && L.eps < 0 && L.c == mask;  // the map x -> ~x
    const bool arith = (L.kind == 0 && (L.op == OP_ADD || L.op == OP_SUB || L.op == OP_MUL)) ||
                       (L.kind == 1 && !notchain);
    if (andor && arith) {
      inv = l;
      break;
    }
    if (L.kind == 0 && (L.op == OP_AND || L.op == OP_OR)) {
      andor = true;
      full = false;
    }
    if (L.kind == 0 && L.op == OP_MUL) full = false;
  }
  it.inv = (int8_t)inv;
  it.nexp = (int8_t)(it.depth - inv);
  it.full = full ? 1 : 0;
  // without & and |, inversion only ever narrows the mask to the low bits
  // (at * levels), so the spine can be joined on those bits
  it.joinable = (!andor && it.nexp == 0) ? 1 : 0;
  uint64_t nctx = 1;
  for (int l = 0; l < it.depth; ++l)
    if (it.lv[l].kind == 0) nctx *= it.lv[l].nsmall;
  it.nctx = nctx;
}

// Thread layout and work units: G groups of kR contexts x L lanes over the
// bottom values, about 2^22 candidates per unit.
static inline void finish_layout(Item& it, int threads, uint64_t unit_target = 1ULL << 22,
                                 int min_lanes = 1, uint64_t max_vals_per_lane = 0) {
  const uint64_t nctx = it.nctx;
  if (it.joinable && nctx >= kJoinMin) {  // hash join (full = 2)
    it.full = 2;
    it.G = 0;
    it.L = 0;
    it.cb = (uint32_t)std::min<uint64_t>(nctx, kJoinCtx);
    it.cblocks = (nctx + it.cb - 1) / it.cb;
    const uint64_t nv_al = (it.nv + 63) / 64 * 64;
    it.vb = std::min<uint64_t>(nv_al, kJoinVals);
    it.vblocks = (it.nv + it.vb - 1) / it.vb;
    it.cpu = 1;
    return;
  }
  uint64_t groups = (nctx + kR - 1) / kR;
  int G = 1;
  // context groups double while they have contexts to take and each keeps
  // at least min_lanes value lanes (the autotuned split of a CTA's threads
  // between contexts and bottom values)
  while (G < threads && (uint64_t)G < groups && threads / (G << 1) >= min_lanes) G <<= 1;
  it.G = (uint16_t)G;
  it.L = (uint16_t)(threads / G);
  it.cb = (uint32_t)(G * kR);
  it.cblocks = (nctx + it.cb - 1) / it.cb;
  uint64_t vb = unit_target / it.cb;  // about unit_target candidates per unit
  const uint64_t align = 64ULL * it.L;
  vb = std::max<uint64_t>(align, (vb + align - 1) / align * align);
  // a cap on the bottom values one lane streams per unit keeps a unit's
  // serial loop short where few contexts leave the thread layout mostly lanes
  if (max_vals_per_lane && vb > max_vals_per_lane * it.L) vb = max_vals_per_lane * it.L;
  const uint64_t nv_al = (it.nv + 63) / 64 * 64;
  if (vb > nv_al) vb = nv_al;
  it.vb = vb;
  it.vblocks = (it.nv + vb - 1) / vb;
  // small bottoms: one context block holds few candidates, so a unit takes
  // several blocks and the per-unit queue and lookup cost is amortised
  it.cpu = 1;
  if (it.vblocks == 1) {
    const uint64_t per = (uint64_t)it.cb * std::max<uint64_t>(it.nv, 1);
    if (per < unit_target)
      it.cpu = (uint16_t)std::min<uint64_t>({unit_target / per, it.cblocks, 65535ULL});
    if (it.cpu == 0) it.cpu = 1;
  }
}

// Integer lane-operations a spine needs.  Nested compares: per candidate
// the masked compare of the bottom value plus every explicitly evaluated
// level (64-bit words take two 32-bit lane operations per bitwise or
// add/sub step and three per multiply).  Hash join: per bottom value and
// context block the hash and the filter test (5), whatever the number of
// contexts the block holds.
static inline double item_alg_ops(const Item& it, size_t wbytes) {
  const double w = wbytes == 8 ? 2.0 : 1.0;
  if (it.full == 2) return (double)it.cblocks * (double)it.nv * 5.0;
  double c = it.full ? w : w + 1.0;
  for (int l = it.inv; l < it.depth; ++l) {
    const Level& L = it.lv[l];
    c += (L.kind == 0 && L.op == OP_MUL) ? (wbytes == 8 ? 3.0 : 1.0) : w;
  }
  return (double)it.nctx * (double)it.nv * c;
}

static inline void finish_item(Item& it, int threads, uint64_t mask) {
  finish_structure(it, mask);
  finish_layout(it, threads);
}

// Shape class of a spine (the guided search's unit of priority): root
// operator x (left operand size, or length of the root's unary chain),
// capped at 7 -- 64 classes.  A unary chain class merges chains that start
// with ~ and with neg, so both root operators are returned.
static inline void spine_classes(const Item& it, int size, int* c0, int* c1) {
  *c0 = *c1 = -1;
  if (it.depth == 0) return;
  const Level& L = it.lv[0];
  if (L.kind == 1) {
    const int m = std::min<int>(std::max<int>(L.chain_len, 1), 7);
    *c0 = OP_NOT * 8 + m;
    *c1 = OP_NEG * 8 + m;
    return;
  }
  const int left = L.small_left ? L.ts : size - 1 - L.ts;
  *c0 = L.op * 8 + std::min(left, 7);
}

// Guided search of a tabled size: the size's rank range (= its value table)
// split into the contiguous ranges of its shape classes -- each operator
// block, and inside a binary block each left size f (N(f) N(s-1-f) ranks,
// class 8 op + min(f, 7)) -- as depth-0 items with their class prior, so that
// the likely classes' ranges are searched first.  A unary block is one range
// whose prior is its best unary-chain class.
static inline void tabled_class_items(const CountTable& ct, int s, const float* prior,
                                      std::vector<Item>* items) {
  auto add = [&](uint64_t a, uint64_t n, float prio) {
    if (n == 0) return;
    Item it;
    memset(&it, 0, sizeof(it));
    it.depth = 0;
    it.bottom = (int8_t)s;
    it.coefv = 1;
    it.nv = n;
    it.lv[0].coef = a;  // item_voff
    it.prio = prio;
    items->push_back(it);
  };
  uint64_t off = 0;
  for (int op = 0; op < 8; ++op) {
    if (is_unary(op)) {
      float p = 0.f;
      for (int m = 1; m < 8; ++m) p = std::max({p, prior[OP_NOT * 8 + m], prior[OP_NEG * 8 + m]});
      add(off, ct.n[s][op], p);
      off += ct.n[s][op];
      continue;
    }
    const int fmax = is_commutative(op) ? (s - 1) / 2 : s - 2;
    for (int f = 1; f <= fmax; ++f) {
      const uint64_t n = ct.n[f][8] * ct.n[s - 1 - f][8];
      add(off, n, prior[op * 8 + std::min(f, 7)]);
      off += n;
    }
  }
}

static inline float spine_prio(const Item& it, int size, const float* prior) {
  int a, b;
  spine_classes(it, size, &a, &b);
  if (a < 0) return 1e30f;  // a whole tabled size: one spine
  float p = prior[a];
  if (b >= 0) p = std::max(p, prior[b]);
  return p;
}

// Fully inverted spines with fewer contexts than one work unit holds would
// each stream their bottom table once; spines sharing a bottom size (and
// mask kind) are fused into one context list instead, materialised on the
// device.  Returns the fused work items; `small` receives the member spines
// with their offsets into the list.  With `nested_all`, every fully inverted
// spine under an & or | is fused whatever its number of contexts (up to
// max_ctxs in all), so that its list can be compacted to the live contexts.
static inline void fuse_small(std::vector<Item>& items, std::vector<Item>* small, uint64_t* nctxs,
                              const CountTable& ct, uint64_t max_ctxs, bool by_prio = false,
                              bool nested_all = false) {
  std::vector<Item> keep;
  std::vector<Item> groups;
  std::vector<std::vector<size_t>> members;
  uint64_t total = 0;
  for (auto& it : items) {
    // a class range of a tabled size covers part of its bottom table: not fused
    const bool fusable = it.nexp == 0 &&
                         (it.nctx < (uint64_t)kThreads * kR || (nested_all && !it.joinable)) &&
                         total + it.nctx <= max_ctxs && item_voff(it) == 0 &&
                         it.nv == ct.n[(int)it.bottom][8];
    if (!fusable) {
      keep.push_back(it);
      continue;
    }
    size_t gi = 0;
    for (; gi < groups.size(); ++gi)
      // joinable spines of one bottom share a group whatever their mask kind
      // (the join reads each context's own mask), so the bottom table is
      // streamed once per block of contexts instead of once per kind
      if (groups[gi].bottom == it.bottom &&
          (groups[gi].full == it.full || (it.joinable && groups[gi].joinable)) &&
          groups[gi].joinable == it.joinable &&
          (!by_prio || groups[gi].prio == it.prio))
        break;
    if (gi == groups.size() && groups.size() >= 127) {  // group indices are int8_t
      keep.push_back(it);
      continue;
    }
    if (gi == groups.size()) {
      Item g;
      memset(&g, 0, sizeof(g));
      g.bottom = it.bottom;
      g.full = it.full;
      g.joinable = it.joinable;
      g.prio = it.prio;
      g.fused = 1;
      g.group = (int8_t)groups.size();
      g.nv = ct.n[(int)it.bottom][8];
      g.base = ~0ULL;
      groups.push_back(g);
      members.emplace_back();
    }
    members[gi].push_back(small->size());
    it.group = (int8_t)gi;
    groups[gi].base = std::min(groups[gi].base, it.base);
    groups[gi].nctx += it.nctx;
    small->push_back(it);
    total += it.nctx;
  }
  uint64_t off = 0;
  for (size_t gi = 0; gi < groups.size(); ++gi) {
    groups[gi].ctx_off = off;
    for (size_t m : members[gi]) {
      (*small)[m].ctx_off = off;
      off += (*small)[m].nctx;
    }
    keep.push_back(groups[gi]);
  }
  // the materialize kernel finds a context's spine by binary search
  std::sort(small->begin(), small->end(),
            [](const Item& a, const Item& b) { return a.ctx_off < b.ctx_off; });
  *nctxs = off;
  items.swap(keep);
}

// Raise (never lower) a kernel's dynamic shared memory limit: sessions,
// batches and the static entry point share the kernel functions, and a
// lower limit set by one would make another's launches fail.
static inline cudaError_t raise_smem_limit(const void* f, size_t bytes) {
  cudaFuncAttributes a;
  cudaError_t e = cudaFuncGetAttributes(&a, f);
  if (e != cudaSuccess) return e;
  if ((size_t)a.maxDynamicSharedSizeBytes >= bytes) return cudaSuccess;
  return cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

template <class W>
class Search final : public SearchSession {
 public:
  Search(const HostInstance& h, const EngineOptions& o) : h_(h), o_(o) {}
  ~Search() override {
    if (stream_ && own_stream_) cudaStreamDestroy(stream_);
    if (ev0_) cudaEventDestroy(ev0_);
    if (evk_) cudaEventDestroy(evk_);
    if (ev1_) cudaEventDestroy(ev1_);
    if (evj_) cudaEventDestroy(evj_);
  }

  int init() {
    SB_CUDA(cudaSetDevice(o_.device));
    if (o_.stream) {
      stream_ = reinterpret_cast<cudaStream_t>(o_.stream);
      own_stream_ = false;
    } else {
      SB_CUDA(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
      own_stream_ = true;
    }
    SB_CUDA(cudaEventCreate(&ev0_));
    SB_CUDA(cudaEventCreate(&evk_));
    SB_CUDA(cudaEventCreate(&ev1_));
    SB_CUDA(cudaEventCreate(&evj_));
    SB_CUDA(cudaDeviceGetAttribute(&sms_, cudaDevAttrMultiProcessorCount, o_.device));
    mask_ = h_.bits == 64 ? ~0ULL : 0xFFFFFFFFULL;
    // count table up to the largest size whose counts fit in 64 bits
    CountTable t;
    int ms = kMaxSize;
    while (ms > 1 && !build_count_table(ms, h_.k, &t)) --ms;
    build_count_table(ms, h_.k, &ct_);
    count_ok_max_ = ms;
    // samples as W words, padded to 16 bytes
    const size_t nin = (size_t)h_.S * h_.k, nout = (size_t)h_.S;
    std::vector<W> win((nin * sizeof(W) + 15) / 16 * 16 / sizeof(W), 0);
    std::vector<W> wout((nout * sizeof(W) + 15) / 16 * 16 / sizeof(W), 0);
    for (size_t i = 0; i < nin; ++i) win[i] = (W)h_.in[i];
    for (size_t i = 0; i < nout; ++i) wout[i] = (W)h_.out[i];
    SB_CUDA(d_in_.reserve(win.size() * sizeof(W)));
    SB_CUDA(d_out_.reserve(wout.size() * sizeof(W)));
    SB_CUDA(cudaMemcpy(d_in_.p, win.data(), win.size() * sizeof(W), cudaMemcpyHostToDevice));
    SB_CUDA(cudaMemcpy(d_out_.p, wout.data(), wout.size() * sizeof(W), cudaMemcpyHostToDevice));
    SB_CUDA(d_counts_.reserve(sizeof(ct_.n)));
    SB_CUDA(cudaMemcpy(d_counts_.p, ct_.n, sizeof(ct_.n), cudaMemcpyHostToDevice));
    SB_CUDA(d_scal_.reserve(256));
    SB_CUDA(d_insts_.reserve(sizeof(InstDesc<W>)));

    // table budget -> largest tabled size
    const int64_t budget = o_.table_bytes > 0 ? o_.table_bytes : (8LL << 30);
    Tcap_ = 0;
    // The filter samples' tables take at most an eighth of the budget
    // (sizes up to Tf_): a single search has large tables and few sparse-
    // mask matches, and building four copies of the largest size would
    // dominate a solve from host buffers.  A spine that needs a table above
    // Tf_ sends its sample-0 matches to verification unfiltered.
    uint64_t cum0 = 0, cumf = 0;
    Tf_ = 0;
    for (int t = 1; t <= count_ok_max_ && t <= 20; ++t) {
      const uint64_t bytes = padded(ct_.n[t][8]) * sizeof(W);
      if (nsamp() > 1 && (cum0 + bytes) * (nsamp() - 1) <= (uint64_t)budget / 8 && Tf_ == t - 1) {
        Tf_ = t;
        cumf = (cum0 + bytes) * (nsamp() - 1);
      }
      if (cum0 + bytes + cumf > (uint64_t)budget) break;
      cum0 += bytes;
      Tcap_ = t;
    }
    if (Tf_ > Tcap_) Tf_ = Tcap_;
    if (Tcap_ < 1) Tcap_ = 1;  // tables are allocated when first built
    built_ = 0;
    smem_bytes_ = ((sizeof(Smem) + 15) & ~size_t(15)) +
                  (((size_t)h_.S * h_.k * sizeof(W) + 15) / 16 + ((size_t)h_.S * sizeof(W) + 15) / 16) * 16;
    join_off_ = (smem_bytes_ + 15) & ~size_t(15);  // join launches: tables after the samples
    smem_join_ = join_off_ + sizeof(JoinSmem);
    SB_CUDA(raise_smem_limit((const void*)spine_kernel<W>, smem_join_));
    SB_CUDA(raise_smem_limit((const void*)naive_kernel<W>, smem_bytes_));
    int occ = 1;
    SB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, spine_kernel<W>, kThreads, smem_bytes_));
    grid_ = sms_ * std::max(occ, 1);
    int occj = 1;
    SB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occj, spine_kernel<W>, kThreads, smem_join_));
    grid_join_ = sms_ * std::max(occj, 1);
    SB_CUDA(d_preq_.reserve((size_t)std::max(grid_, grid_join_) * kPreG * 8));
    int occn = 1;
    SB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occn, naive_kernel<W>, kThreads, smem_bytes_));
    grid_naive_ = sms_ * std::max(occn, 1);
    return 0;
  }

  int solve(int max_size, SolveOutcome* out) override { return run(max_size, 0, 0, true, out); }
  int sweep(int lo, int hi, SolveOutcome* out) override { return run(hi, lo, hi, false, out); }

  // One size over the work units u with u % nshards == shard (the others
  // belong to other GPUs); the caller combines the shards' minima.
  int search_one_size(int s, int shard, int nshards, SizeOutcome* out) override {
    *out = SizeOutcome();
    if (s < 1 || s > count_ok_max_ || nshards < 1 || shard < 0 || shard >= nshards) {
      set_last_error("bad size or shard");
      return SIMBA_E_ARG;
    }
    launches_ = 0;
    kernel_ms_ = 0.0;
    alg_ops_ = 0;
    stamp_start_kernel<<<1, 1, 0, stream_>>>(d_scal_.as<unsigned long long>() + 3);
    ++launches_;
    SB_CUDA(cudaGetLastError());
    uint64_t best = ~0ULL;
    double ms = 0;
    const int rc = search_size(s, true, &best, &out->evaluated, &ms, shard, nshards);
    out->best = best;
    out->candidates = ct_.n[s][8];
    out->device_ms = ms;
    out->kernel_ms = kernel_ms_;
    out->launches = launches_;
    out->status = rc == SIMBA_BUDGET ? SIMBA_BUDGET : (best != ~0ULL ? SIMBA_OK : SIMBA_NOT_FOUND);
    return rc < 0 ? rc : out->status;
  }

 private:
  static uint64_t padded(uint64_t n) { return (n + 63) / 64 * 64 + 64; }

  // V_t on sample j (j = 0, and the filter samples 1..kExtra that exist): one
  // allocation per size t holds the tables of all samples
  W* tab(int t, int j = 0) const { return d_tabs_[t].as<W>() + (size_t)j * padded(ct_.n[t][8]); }
  int nsamp() const { return std::min(h_.S, filter_samples(o_) + 1); }

  // Build V_{built+1} .. V_t (each entry one operator over smaller tables).
  int ensure_tables(int t) {
    for (int s = built_ + 1; s <= t; ++s) {
      const int copies = s <= Tf_ ? nsamp() : 1;
      SB_CUDA(d_tabs_[s].reserve(padded(ct_.n[s][8]) * sizeof(W) * copies));
      // one launch per size: every operator block of every sample's table
      std::vector<BuildJob<W>> jobs;
      uint64_t total = 0;
      for (int j = 0; j < copies; ++j) {
        W* o = tab(s, j);
        if (s == 1) {
          std::vector<W> v(padded(h_.k), 0);
          for (int q = 0; q < h_.k; ++q) v[q] = (W)h_.in[(size_t)j * h_.k + q];
          SB_CUDA(cudaMemcpyAsync(o, v.data(), v.size() * sizeof(W), cudaMemcpyHostToDevice, stream_));
          continue;
        }
        uint64_t off = 0;
        const int sub = s - 1;
        for (int op = 0; op < 8; ++op) {
          const int fmax = is_unary(op) ? 1 : (is_commutative(op) ? sub / 2 : sub - 1);
          for (int f = 1; f <= fmax; ++f) {
            BuildJob<W> b;
            memset(&b, 0, sizeof(b));
            b.out = o + off;
            b.op = op;
            b.begin = total;
            if (is_unary(op)) {
              b.A = tab(sub, j);
              b.na = ct_.n[sub][8];
              b.nb = 1;
            } else {
              b.A = tab(f, j);
              b.B = tab(sub - f, j);
              b.na = ct_.n[f][8];
              b.nb = ct_.n[sub - f][8];
            }
            const uint64_t n = b.na * b.nb;
            if (n == 0) continue;
            jobs.push_back(b);
            off += n;
            total += n;
          }
        }
      }
      if (!jobs.empty()) {
        // stream order keeps the previous size's build ahead of this copy;
        // the copy from pageable memory is staged before the call returns
        SB_CUDA(d_jobs_.reserve(jobs.size() * sizeof(BuildJob<W>)));
        SB_CUDA(cudaMemcpyAsync(d_jobs_.p, jobs.data(), jobs.size() * sizeof(BuildJob<W>),
                                cudaMemcpyHostToDevice, stream_));
        const int blocks = (int)std::min<uint64_t>((total + 255) / 256, (uint64_t)sms_ * 16);
        build_batch_kernel<W><<<blocks, 256, 0, stream_>>>(d_jobs_.as<BuildJob<W>>(), (int)jobs.size(),
                                                            total);
        ++launches_;
      }
      SB_CUDA(cudaGetLastError());
      built_ = s;
    }
    return 0;
  }

  // Kernel parameters for size s; uploads the instance descriptor.
  Params<W> params(int s) {
    InstDesc<W> d;
    memset(&d, 0, sizeof(d));
    for (int t = 1; t <= built_; ++t) {
      d.tab[t] = tab(t);
      if (t <= Tf_)
        for (int j = 1; j < nsamp(); ++j) d.tabx[j - 1][t] = tab(t, j);
    }
    for (int j = 1; j < nsamp(); ++j) d.targetx[j - 1] = (W)h_.out[j];
    d.in = d_in_.as<W>();
    d.out = d_out_.as<W>();
    d.counts = d_counts_.as<unsigned long long>();
    unsigned long long* sc = d_scal_.as<unsigned long long>();
    d.best = sc + 1;
    d.target = (W)h_.out[0];
    d.size = s;
    d.S = h_.S;
    d.K = h_.k;
    d.rtid = o_.rank_order == 1 && s > 1;
    if (d.rtid)
      for (int op = 0; op < 8; ++op)
        if (ct_.n[s][op]) d.rt_inv[op] = inverse_mod(rtid_multiplier(ct_.n[s][op]), ct_.n[s][op]);
    cudaMemcpyAsync(d_insts_.p, &d, sizeof(d), cudaMemcpyHostToDevice, stream_);
    Params<W> p;
    memset(&p, 0, sizeof(p));
    p.insts = d_insts_.as<InstDesc<W>>();
    p.counter = sc + 0;
    p.evaluated = sc + 2;
    p.start_ns = sc + 3;
    p.flags = reinterpret_cast<int*>(sc + 4);
    p.hits = sc + 6;
    p.live = sc + 8;
    p.preq = d_preq_.as<unsigned long long>();
    p.maxS = h_.S;
    p.maxK = h_.k;
    p.budget_ns = o_.budget_s > 0 ? (unsigned long long)(o_.budget_s * 1e9) : 0;
    return p;
  }

  // Search one size; writes the minimum matching rank (or ~0) and the number
  // of candidates evaluated.  status: 0 ok, SIMBA_BUDGET on budget expiry.

  int search_size(int s, bool stop, uint64_t* best, uint64_t* evaluated, double* ms, int shard = 0,
                  int nshards = 1) {
    dead_ = 0;
    double alg_total = 0;
    // reset counter, best, evaluated, flags
    unsigned long long init[8] = {0, ~0ULL, 0, 0, 0, 0, 0, 0};
    SB_CUDA(cudaMemcpyAsync(d_scal_.p, init, 3 * sizeof(unsigned long long), cudaMemcpyHostToDevice, stream_));
    SB_CUDA(cudaMemsetAsync(d_scal_.as<unsigned long long>() + 4, 0, 5 * sizeof(unsigned long long), stream_));
    const bool spine_ok = o_.engine == 0 && s <= count_ok_max_;
    int T = std::min(Tcap_, s);
    bool use_naive = !spine_ok || (s > T && (s - 1) / 2 > T);
    std::vector<Item> items;
    if (!use_naive) {
      if (s <= T && o_.class_prior && s >= 2) {
        tabled_class_items(ct_, s, o_.class_prior, &items);
      } else if (s <= T) {
        Item it;
        memset(&it, 0, sizeof(it));
        it.depth = 0;
        it.bottom = (int8_t)s;
        it.base = 0;
        it.coefv = 1;
        it.nv = ct_.n[s][8];
        items.push_back(it);
      } else {
        Enumerator en;
        en.ct = &ct_;
        en.T = T;
        en.mask = mask_;
        en.items = &items;
        std::vector<Level> lv;
        std::vector<ChainClass> top{{1, 0, 0}};
        en.rec(s, lv, 1, 0, top);
        if (en.too_deep) use_naive = true;
      }
    }
    SB_CUDA(cudaEventRecord(ev0_, stream_));
    if (!use_naive) {
      int rc = ensure_tables(std::min(T, s));
      if (rc) return rc;
      for (auto& it : items) {
        for (int l = 0; l < it.depth; ++l)
          if (it.lv[l].kind == 1) it.lv[l].c &= mask_;
        finish_structure(it, mask_);
      }
      const bool guided = o_.class_prior != nullptr;
      if (guided)  // class ranges of a tabled size carry their prior already
        for (auto& it : items)
          if (it.depth > 0) it.prio = spine_prio(it, s, o_.class_prior);
      std::vector<Item> small;
      uint64_t nctxs = 0;
      fuse_small(items, &small, &nctxs, ct_, 1ULL << 22, guided, true);
      for (auto& it : items) {  // planned work of the two launch kinds (every joinable spine joins)
        const double c = (double)it.nctx * (double)it.nv;
        if (it.joinable) join_cand_ += c;
        else nested_cand_ += c;
      }
      Params<W> p = params(s);
      SB_CUDA(cudaEventRecord(evk_, stream_));
      double dead = 0;  // candidates of contexts left out of the compacted lists
      if (nctxs) {
        // Materialise the fused spines' contexts, keeping per group only the
        // live ones (some bottom value may complete them on sample 0), and
        // read the live counts back: the work units are laid out over those.
        SB_CUDA(d_small_.reserve(small.size() * sizeof(Item)));
        SB_CUDA(cudaMemcpyAsync(d_small_.p, small.data(), small.size() * sizeof(Item),
                                cudaMemcpyHostToDevice, stream_));
        SB_CUDA(d_ctx_.reserve(nctxs * sizeof(Ctx<W>)));
        for (auto& it : items)
          if (it.fused) {
            h_glive_[2 * it.group] = 0;
            h_glive_[2 * it.group + 1] = it.ctx_off;
          }
        SB_CUDA(d_glive_.reserve(sizeof(h_glive_)));
        SB_CUDA(cudaMemcpyAsync(d_glive_.p, h_glive_, sizeof(h_glive_), cudaMemcpyHostToDevice, stream_));
        p.sitems = d_small_.as<Item>();
        p.nsitems = (int)small.size();
        p.nctxs = nctxs;
        p.ctx_live = d_glive_.as<unsigned long long>();
        const int mb = (int)std::min<uint64_t>((nctxs + 255) / 256, (uint64_t)sms_ * 8);
        materialize_kernel<W><<<mb, 256, 0, stream_>>>(p, d_ctx_.as<Ctx<W>>());
        ++launches_;
        SB_CUDA(cudaGetLastError());
        SB_CUDA(cudaMemcpyAsync(h_glive_, d_glive_.p, sizeof(h_glive_), cudaMemcpyDeviceToHost, stream_));
        SB_CUDA(cudaStreamSynchronize(stream_));
        p.ctx_live = nullptr;
        p.ctxs = d_ctx_.as<Ctx<W>>();
        std::vector<Item> kept;
        for (auto& it : items) {
          if (it.fused) {
            const uint64_t live = h_glive_[2 * it.group];
            dead += (double)(it.nctx - live) * (double)it.nv;
            it.nctx = live;
            it.fused = 2;
            if (live == 0) continue;
          }
          kept.push_back(it);
        }
        items.swap(kept);
      }
      uint64_t unit_target = 1ULL << (o_.unit_log2 > 0 ? std::min(o_.unit_log2, 40) : 22);
      if (o_.unit_log2 <= 0) {
        // By default the nested-compare units shrink (down to 2^16
        // candidates) until the launch has four units per resident CTA: the
        // compacted lists leave a size little work, and a few large units
        // would run as long serial loops on a few SMs.
        double nested = 0;
        for (auto& it : items)
          if (!it.joinable) nested += (double)it.nctx * (double)it.nv;
        while (unit_target > (1ULL << 16) && nested < 4.0 * grid_ * (double)unit_target) unit_target >>= 1;
      }
      for (auto& it : items) {
        // Nested spines left out of the compacted lists (explicit levels)
        // find most of their contexts dead in each unit: units an eighth
        // the size spread the live ones' streaming over more CTAs.
        const bool listless = !it.joinable && !it.fused && it.depth > 0 && o_.unit_log2 <= 0;
        const uint64_t ut = listless ? std::max<uint64_t>(unit_target >> 3, 1ULL << 16) : unit_target;
        finish_layout(it, kThreads, ut, 1 << std::min(o_.lanes_log2, 8), o_.unit_log2 <= 0 ? 256 : 0);
      }
      if (guided)  // most likely shape classes first; ties in rank order
        std::stable_sort(items.begin(), items.end(), [](const Item& a, const Item& b) {
          return a.prio != b.prio ? a.prio > b.prio : a.base < b.base;
        });
      else
        std::stable_sort(items.begin(), items.end(),
                         [](const Item& a, const Item& b) { return a.base < b.base; });
      // join units run in a launch of their own (with the join tables in
      // shared memory), the nested-compare units in another
      std::stable_partition(items.begin(), items.end(), [](const Item& a) { return a.full == 2; });
      size_t nj = 0;
      while (nj < items.size() && items[nj].full == 2) ++nj;
      uint64_t units = 0, units_join = 0;
      for (size_t q = 0; q < items.size(); ++q) {
        if (q == nj) {
          units_join = units;
          units = 0;
        }
        items[q].unit_begin = units;
        units += item_units(items[q]);
      }
      if (nj == items.size()) {
        units_join = units;
        units = 0;
      }
      if (!items.empty()) {
        SB_CUDA(d_items_.reserve(items.size() * sizeof(Item)));
        SB_CUDA(cudaMemcpyAsync(d_items_.p, items.data(), items.size() * sizeof(Item),
                                cudaMemcpyHostToDevice, stream_));
      }
      for (auto& it : items) alg_total += item_alg_ops(it, sizeof(W));
      {  // what the join launch streams
        bool seen[kMaxSize + 1] = {};
        for (size_t q = 0; q < nj; ++q) {
          const Item& it = items[q];
          join_streamed_ += (double)it.nv * sizeof(W) * (double)it.cblocks;
          if (!seen[(int)it.bottom]) {
            seen[(int)it.bottom] = true;
            join_table_ += (double)it.nv * sizeof(W);
          }
        }
      }
      if (shard == 0) dead_ = dead;
      p.items = d_items_.as<Item>() + nj;
      p.nitems = (int)(items.size() - nj);
      p.total_units = units;
      p.unit_offset = (unsigned long long)shard;
      p.unit_stride = (unsigned long long)nshards;
      p.stop_on_match = stop ? (guided ? 2 : 1) : 0;
      if (nj) {
        Params<W> pj = p;
        pj.items = d_items_.as<Item>();
        pj.nitems = (int)nj;
        pj.total_units = units_join;
        pj.join_off = (unsigned)join_off_;
        spine_kernel<W><<<grid_join_, kThreads, smem_join_, stream_>>>(pj);
        ++launches_;
      }
      SB_CUDA(cudaEventRecord(evj_, stream_));
      if (nj < items.size()) {
        p.counter = d_scal_.as<unsigned long long>() + 7;  // zeroed with the flags
        spine_kernel<W><<<grid_, kThreads, smem_bytes_, stream_>>>(p);
        ++launches_;
      }
      SB_CUDA(cudaGetLastError());
    } else {
      Params<W> p = params(s);
      p.stop_on_match = stop ? 1 : 0;
      alg_total = (double)ct_.n[s][8] * (double)s * (sizeof(W) == 8 ? 2.0 : 1.0);
      SB_CUDA(cudaEventRecord(evk_, stream_));
      SB_CUDA(cudaEventRecord(evj_, stream_));  // no join launch
      nested_cand_ += (double)ct_.n[s][8];
      const unsigned __int128 n = ct_.n[s][8];
      const uint64_t lo = (uint64_t)(n * (unsigned)shard / (unsigned)nshards);
      const uint64_t hi = (uint64_t)(n * (unsigned)(shard + 1) / (unsigned)nshards);
      naive_kernel<W><<<grid_naive_, kThreads, smem_bytes_, stream_>>>(p, lo, hi);
      ++launches_;
      SB_CUDA(cudaGetLastError());
    }
    SB_CUDA(cudaEventRecord(ev1_, stream_));
    SB_CUDA(cudaMemcpyAsync(h_scal_, d_scal_.p, 9 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, stream_));
    SB_CUDA(cudaStreamSynchronize(stream_));
    float e = 0, ek = 0, ej = 0;
    SB_CUDA(cudaEventElapsedTime(&e, ev0_, ev1_));
    SB_CUDA(cudaEventElapsedTime(&ek, evk_, ev1_));
    SB_CUDA(cudaEventElapsedTime(&ej, evk_, evj_));
    *ms += e;
    kernel_ms_ += ek;
    join_ms_ += ej;
    nested_ms_ += ek - ej;
    const unsigned long long* hs = static_cast<unsigned long long*>(h_scal_);
    *best = hs[1];
    // the candidates the compaction decided count with a size swept to the
    // end; where a match stopped the search early, only the units that ran
    *evaluated += hs[2] + (hs[1] == ~0ULL ? (uint64_t)dead_ : 0);
    nested_live_ += hs[8];
    const double cand_total = use_naive ? (double)ct_.n[s][8] : [&] {
      double c = 0;
      for (auto& it : items) c += (double)it.nctx * (double)it.nv;
      return c;
    }();
    if (cand_total > 0) alg_ops_ += (uint64_t)(alg_total * ((double)hs[2] / cand_total));
    const int* fl = reinterpret_cast<const int*>(hs + 4);
    last_T_ = use_naive ? 0 : T;
    if (fl[1]) {
      set_last_error("inversion failed on a level marked invertible");
      return SIMBA_E_INTERNAL;
    }
    if (o_.verbose)
      fprintf(stderr, "size %2d | %s | items %zu | evaluated %llu | sample-0 hits %llu | %.3f ms\n", s,
              use_naive ? "naive" : "spine", items.size(), (unsigned long long)hs[2],
              (unsigned long long)hs[6], e);
    return fl[0] ? SIMBA_BUDGET : 0;
  }

  int run(int max_size, int lo, int hi, bool stop, SolveOutcome* out) {
    *out = SolveOutcome();
    int first, last;
    if (stop) {
      first = o_.size_range ? 1 : 2;
      last = o_.size_range ? max_size : max_size - 1;
    } else {
      first = lo;
      last = hi;
    }
    if (last > count_ok_max_) {
      set_last_error("candidate counts exceed 64 bits at this size");
      return SIMBA_E_OVERFLOW;
    }
    launches_ = 0;
    kernel_ms_ = 0.0;
    join_ms_ = nested_ms_ = join_cand_ = nested_cand_ = join_streamed_ = join_table_ = 0.0;
    nested_live_ = 0;
    alg_ops_ = 0;
    stamp_start_kernel<<<1, 1, 0, stream_>>>(d_scal_.as<unsigned long long>() + 3);
    ++launches_;
    SB_CUDA(cudaGetLastError());
    const auto t0 = std::chrono::steady_clock::now();
    for (int s = first; s <= last; ++s) {
      if (o_.budget_s > 0) {
        const double el = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        if (el > o_.budget_s) {
          out->status = SIMBA_BUDGET;
          return SIMBA_BUDGET;
        }
      }
      uint64_t best = ~0ULL;
      int rc = search_size(s, stop, &best, &out->evaluated, &out->device_ms);
      if (best != ~0ULL && o_.rank_order == 1 && s > 1) best = rtid_rank(ct_.n, s, best);
      out->launches = launches_;
      out->kernel_ms = kernel_ms_;
      out->join_ms = join_ms_;
      out->nested_ms = nested_ms_;
      out->join_candidates = (uint64_t)join_cand_;
      out->nested_candidates = (uint64_t)nested_cand_;
      out->nested_live_candidates = nested_live_;
      out->join_bytes_streamed = join_streamed_;
      out->join_table_bytes = join_table_;
      out->alg_ops = alg_ops_;
      out->max_size_searched = s;
      out->table_size = std::max(out->table_size, last_T_);
      if (rc == SIMBA_BUDGET) {
        out->status = SIMBA_BUDGET;
        return SIMBA_BUDGET;
      }
      if (rc) return rc;
      if (best != ~0ULL && stop) {
        const int op = s == 1 ? 8 : op_of_rank(ct_.n, s, best);
        uint64_t c = 0;
        if (s == 1) c = best + 1;
        else
          for (int q = 0; q <= op; ++q) c += ct_.n[s][q];
        out->per_size[s] = c;
        out->candidates += c;
        char buf[kMaxSize + 1];
        unrank(best, s, ct_.n, buf);
        buf[s] = 0;
        out->postfix = buf;
        out->size = s;
        out->op = op;
        out->rank = best;
        if (!host_check(out->postfix, h_)) {
          set_last_error("device match failed the host re-check");
          return SIMBA_E_INTERNAL;
        }
        out->status = SIMBA_OK;
        return SIMBA_OK;
      }
      out->per_size[s] = ct_.n[s][8];
      out->candidates += ct_.n[s][8];
      if (!stop && best != ~0ULL && out->status != SIMBA_OK) {
        // sweeps report the first size with a match but keep going
        char buf[kMaxSize + 1];
        unrank(best, s, ct_.n, buf);
        buf[s] = 0;
        out->postfix = buf;
        out->size = s;
        out->op = s == 1 ? 8 : op_of_rank(ct_.n, s, best);
        out->rank = best;
        out->status = SIMBA_OK;
      }
    }
    if (out->status != SIMBA_OK) out->status = SIMBA_NOT_FOUND;
    return out->status;
  }

  HostInstance h_;
  EngineOptions o_;
  CountTable ct_;
  int count_ok_max_ = 0;
  uint64_t mask_ = 0;
  cudaStream_t stream_ = nullptr;
  cudaEvent_t ev0_ = nullptr, evk_ = nullptr, ev1_ = nullptr, evj_ = nullptr;
  bool own_stream_ = true;
  int launches_ = 0;
  double kernel_ms_ = 0.0;
  double join_ms_ = 0.0, nested_ms_ = 0.0, join_cand_ = 0.0, nested_cand_ = 0.0;
  uint64_t nested_live_ = 0;  // candidates of live nested-compare contexts
  double join_streamed_ = 0.0, join_table_ = 0.0;
  uint64_t alg_ops_ = 0;
  int sms_ = 0, grid_ = 0, grid_naive_ = 0, grid_join_ = 0;
  size_t smem_bytes_ = 0, join_off_ = 0, smem_join_ = 0;
  DevBuf d_in_, d_out_, d_counts_, d_scal_, d_items_, d_small_, d_ctx_, d_insts_, d_preq_, d_jobs_;
  DevBuf d_glive_;                       // per fused group: live count, first slot
  unsigned long long h_glive_[2 * 128] = {};
  double dead_ = 0;  // candidates of this size decided by the list compaction
  DevBuf d_tabs_[kMaxSize + 1];  // V_t of every sample, allocated when size t is first built
  unsigned long long h_scal_[16] = {};
  int Tcap_ = 0, Tf_ = 0, built_ = 0, last_T_ = 0;
};

// ------------------------------------------------------------------ batch

// Fused spine list of one (terms, tabled size, size): spine shapes depend
// only on these, not on an instance's values, so every instance with the
// same key shares them (contexts are materialised per instance).
struct ItemTemplate {
  std::vector<Item> items;   // fused groups + unfused spines (ctx_off relative)
  std::vector<Item> small;   // fused members (ctx_off relative)
  uint64_t nctxs = 0;
  uint64_t units = 0;
  double alg = 0;            // algorithmic lane-operations of the whole size
  double cand = 0;           // candidates evaluated for the whole size
  bool ok = true;            // false: spines too deep, use per-rank kernel
  int id = -1;               // index of its TmplDesc on the device
  uint64_t bucket_units[64] = {};  // guided lists: units per shape class
};

// Batched plain search: many independent instances advance size by size in
// rounds; one persistent spine_kernel launch per round serves the work
// units of every active instance (an atomic work queue across instances),
// and an instance whose size produced a match retires at the end of that
// round.  Value tables are per instance, built by one batched launch per
// round.  All instances share the word width W.
template <class W>
class Batch {
 public:
  struct Out {
    int status = SIMBA_NOT_FOUND;
    int size = 0, op = -1;
    uint64_t rank = 0;
    std::string postfix;
    double seconds = 0;
    uint64_t candidates = 0;
  };

  Batch(const std::vector<HostInstance>& hs, const EngineOptions& o, int64_t inst_table_bytes,
        uint64_t unit_target)
      : hs_(hs), o_(o), inst_budget_(inst_table_bytes), unit_target_(unit_target) {}
  ~Batch() {
    if (stream_ && own_stream_) cudaStreamDestroy(stream_);
    if (e0_) cudaEventDestroy(e0_);
    if (e1_) cudaEventDestroy(e1_);
  }

  int run(int max_size, std::vector<Out>* outs, double* device_ms, int* rounds, int* launches,
          uint64_t* evaluated, uint64_t* candidates, double* alg_ops, double* kernel_ms) {
    const int n = (int)hs_.size();
    outs->assign(n, Out());
    SB_CUDA(cudaSetDevice(o_.device));
    if (o_.stream) {
      stream_ = reinterpret_cast<cudaStream_t>(o_.stream);
      own_stream_ = false;
    } else {
      SB_CUDA(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
    }
    SB_CUDA(cudaEventCreate(&e0_));
    SB_CUDA(cudaEventCreate(&e1_));
    int sms = 0;
    SB_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, o_.device));
    const uint64_t mask = sizeof(W) == 8 ? ~0ULL : 0xFFFFFFFFULL;
    // count tables per distinct terminal count
    int maxS = 1, maxK = 1;
    std::vector<int> ct_of(n);
    for (int i = 0; i < n; ++i) {
      maxS = std::max(maxS, hs_[i].S);
      maxK = std::max(maxK, hs_[i].k);
      int j = 0;
      for (; j < (int)cts_.size(); ++j)
        if (cts_[j].terms == hs_[i].k) break;
      if (j == (int)cts_.size()) {
        CountTable t;
        int ms = kMaxSize;
        while (ms > 1 && !build_count_table(ms, hs_[i].k, &t)) --ms;
        build_count_table(ms, hs_[i].k, &t);
        cts_.push_back(t);
      }
      ct_of[i] = j;
    }
    for (auto& t : cts_)
      if (max_size > t.max_size) {
        set_last_error("candidate counts exceed 64 bits at this size");
        return SIMBA_E_OVERFLOW;
      }
    // per-instance tabled size and device layout
    std::vector<int> T(n);
    std::vector<uint64_t> tab_off(n), in_off(n), out_off(n);
    std::vector<std::array<uint64_t, kMaxSize + 1>> toff(n);
    uint64_t tab_total = 0, smp_total = 0;
    auto padded = [](uint64_t x) { return (x + 63) / 64 * 64 + 64; };
    std::vector<uint64_t> tab_sz(n);
    std::vector<int> nsamp(n);
    for (int i = 0; i < n; ++i) {
      const CountTable& ct = cts_[ct_of[i]];
      nsamp[i] = std::min(hs_[i].S, filter_samples(o_) + 1);  // sample-0 tables and the filter samples'
      const uint64_t ns = (uint64_t)nsamp[i];
      uint64_t tot = 0;  // every tabled size has the tables of all samples
      T[i] = 0;
      for (int t = 1; t <= ct.max_size && t <= 16; ++t) {
        const uint64_t b = padded(ct.n[t][8]) * sizeof(W);
        if (t > 1 && (tot + b) * ns > (uint64_t)inst_budget_) break;
        toff[i][t] = tot;
        tot += b;
        T[i] = t;
      }
      tab_off[i] = tab_total;
      tab_sz[i] = tot;
      tab_total += tot * ns;
      in_off[i] = smp_total;
      smp_total += ((uint64_t)hs_[i].S * hs_[i].k * sizeof(W) + 15) / 16 * 16;
      out_off[i] = smp_total;
      smp_total += ((uint64_t)hs_[i].S * sizeof(W) + 15) / 16 * 16;
    }
    SB_CUDA(d_tab_.reserve(tab_total + 256));
    SB_CUDA(d_smp_.reserve(smp_total + 256));
    SB_CUDA(d_cts_.reserve(cts_.size() * sizeof(cts_[0].n)));
    SB_CUDA(d_best_.reserve((size_t)n * 8));
    SB_CUDA(d_desc_.reserve((size_t)n * sizeof(InstDesc<W>)));
    SB_CUDA(d_scal_.reserve(256));
    {
      std::vector<unsigned char> smp(smp_total, 0);
      for (int i = 0; i < n; ++i) {
        W* a = reinterpret_cast<W*>(smp.data() + in_off[i]);
        W* b = reinterpret_cast<W*>(smp.data() + out_off[i]);
        for (size_t q = 0; q < hs_[i].in.size(); ++q) a[q] = (W)hs_[i].in[q];
        for (size_t q = 0; q < hs_[i].out.size(); ++q) b[q] = (W)hs_[i].out[q];
      }
      SB_CUDA(cudaMemcpy(d_smp_.p, smp.data(), smp_total, cudaMemcpyHostToDevice));
      std::vector<uint64_t> cta(cts_.size() * (kMaxSize + 1) * kCols);
      for (size_t j = 0; j < cts_.size(); ++j)
        memcpy(cta.data() + j * (kMaxSize + 1) * kCols, cts_[j].n, sizeof(cts_[j].n));
      SB_CUDA(cudaMemcpy(d_cts_.p, cta.data(), cta.size() * 8, cudaMemcpyHostToDevice));
      // V_1 of every instance: the terminals on samples 0 and 1, gathered
      // into one upload and scattered to the instances' tables on the device
      constexpr int NS = kExtra + 1;
      std::vector<W> v1((size_t)NS * n * maxK, 0);
      std::vector<unsigned long long> dst((size_t)NS * n, ~0ULL);
      std::vector<int> kk(n);
      for (int i = 0; i < n; ++i) {
        kk[i] = hs_[i].k;
        for (int j = 0; j < nsamp[i]; ++j) {
          dst[(size_t)NS * i + j] = tab_off[i] + (uint64_t)j * tab_sz[i] + toff[i][1];
          for (int q = 0; q < hs_[i].k; ++q)
            v1[((size_t)NS * i + j) * maxK + q] = (W)hs_[i].in[(size_t)j * hs_[i].k + q];
        }
      }
      DevBuf d_v1, d_dst, d_kk;
      SB_CUDA(d_v1.reserve(v1.size() * sizeof(W)));
      SB_CUDA(d_dst.reserve(dst.size() * 8));
      SB_CUDA(d_kk.reserve(kk.size() * sizeof(int) + 16));
      SB_CUDA(cudaMemcpy(d_v1.p, v1.data(), v1.size() * sizeof(W), cudaMemcpyHostToDevice));
      SB_CUDA(cudaMemcpy(d_dst.p, dst.data(), dst.size() * 8, cudaMemcpyHostToDevice));
      SB_CUDA(cudaMemcpy(d_kk.p, kk.data(), kk.size() * sizeof(int), cudaMemcpyHostToDevice));
      const unsigned long long nw = (unsigned long long)NS * n * maxK;
      scatter_terminals_kernel<W><<<(int)std::min<unsigned long long>((nw + 255) / 256, 65535), 256, 0,
                                    stream_>>>(d_v1.as<W>(), d_dst.as<unsigned long long>(),
                                               d_kk.as<int>(), d_tab_.as<char>(), n, maxK, NS);
      SB_CUDA(cudaGetLastError());
      SB_CUDA(cudaStreamSynchronize(stream_));
    }
    std::vector<int> size(n), built(n, 1);
    const int first = o_.size_range ? 1 : 2;
    const int last = o_.size_range ? max_size : max_size - 1;
    for (int i = 0; i < n; ++i) size[i] = first;
    std::vector<char> active(n, 1), inround(n, 0), ran(n, 0);
    std::vector<double> swept(n, 0.0);  // candidates of the sizes already searched
    if (first > last)
      for (int i = 0; i < n; ++i) active[i] = 0, (*outs)[i].status = SIMBA_NOT_FOUND;
    auto tabp = [&](int i, int t, int j = 0) {  // sample j's V_t of instance i
      return reinterpret_cast<const W*>(d_tab_.as<char>() + tab_off[i] + (uint64_t)j * tab_sz[i] +
                                        toff[i][t]);
    };
    auto next_cost = [&](int i) { return swept[i] + (double)cts_[ct_of[i]].n[size[i]][8]; };
    const size_t smem_base = ((sizeof(Smem) + 15) & ~size_t(15)) +
                             (((size_t)maxS * maxK * sizeof(W) + 15) / 16 + ((size_t)maxS * sizeof(W) + 15) / 16) * 16;
    const size_t join_off = (smem_base + 15) & ~size_t(15);  // one launch: join tables included
    const size_t smem = join_off + sizeof(JoinSmem);
    SB_CUDA(raise_smem_limit((const void*)spine_kernel<W>, smem));
    SB_CUDA(raise_smem_limit((const void*)naive_kernel<W>, smem));
    int occ = 1;
    SB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, spine_kernel<W>, kThreads, smem));
    const int grid = sms * std::max(occ, 1);
    SB_CUDA(d_preq_.reserve((size_t)grid * kPreG * 8));
    SB_CUDA(d_ns_.reserve((size_t)n * 16 + 16));
    SB_CUDA(cudaMemsetAsync(d_ns_.p, 0, (size_t)n * 16, stream_));
    std::vector<unsigned long long> ns(2 * (size_t)n + 2);
    const double growth = round_growth();
    const auto t0 = std::chrono::steady_clock::now();
    SB_CUDA(cudaEventRecord(e0_, stream_));
    stamp_start_kernel<<<1, 1, 0, stream_>>>(d_scal_.as<unsigned long long>() + 3);
    *launches = 1;
    *rounds = 0;
    *evaluated = 0;
    *candidates = 0;
    *alg_ops = 0;
    *kernel_ms = 0;
    std::vector<InstDesc<W>> desc(n);
    std::vector<unsigned long long> best(n);
    std::vector<int> order;
    unsigned long long start_ns = 0;
    for (;;) {
      // Rounds in order of cost: an instance searches its next size in this
      // round when the candidates it will then have swept are within
      // `growth` times the cheapest such total, so instances that are cheap
      // to solve reach their sizes first instead of waiting for every
      // instance's sweep of each size.
      double lo = std::numeric_limits<double>::infinity();
      for (int i = 0; i < n; ++i)
        if (active[i]) lo = std::min(lo, next_cost(i));
      if (!(lo < std::numeric_limits<double>::infinity())) break;
      const double el = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
      if (o_.budget_s > 0 && el > o_.budget_s) {
        for (int i = 0; i < n; ++i)
          if (active[i]) {
            active[i] = 0;
            (*outs)[i].status = SIMBA_BUDGET;
            (*outs)[i].seconds = el;
          }
        break;
      }
      const double theta = lo * growth;
      order.clear();
      for (int i = 0; i < n; ++i) {
        inround[i] = active[i] && next_cost(i) <= theta;
        if (inround[i]) order.push_back(i);
      }
      std::stable_sort(order.begin(), order.end(),
                       [&](int a, int b) { return next_cost(a) < next_cost(b); });
      ++*rounds;
      // 1. value tables: instances whose current size is tabled build it now
      build_jobs_.clear();
      for (int i : order) {
        const int want = std::min(size[i], T[i]);
        const CountTable& ct = cts_[ct_of[i]];
        for (int t = built[i] + 1; t <= want; ++t) {
          const int sub = t - 1;
          for (int j = 0; j < nsamp[i]; ++j) {
            uint64_t off = 0;
            W* o = const_cast<W*>(tabp(i, t, j));
            for (int op = 0; op < 8; ++op) {
              if (is_unary(op)) {
                build_jobs_.push_back({o + off, tabp(i, sub, j), nullptr, ct.n[sub][8], 1, op, 0});
                off += ct.n[sub][8];
                continue;
              }
              const int fmax = is_commutative(op) ? sub / 2 : sub - 1;
              for (int f = 1; f <= fmax; ++f) {
                const uint64_t na = ct.n[f][8], nb = ct.n[sub - f][8];
                build_jobs_.push_back({o + off, tabp(i, f, j), tabp(i, sub - f, j), na, nb, op, 0});
                off += na * nb;
              }
            }
          }
          built[i] = t;
        }
      }
      if (!build_jobs_.empty()) {
        uint64_t acc = 0;
        for (auto& j : build_jobs_) {
          j.begin = acc;
          acc += j.na * j.nb;
        }
        SB_CUDA(d_jobs_.reserve(build_jobs_.size() * sizeof(BuildJob<W>)));
        SB_CUDA(cudaMemcpyAsync(d_jobs_.p, build_jobs_.data(), build_jobs_.size() * sizeof(BuildJob<W>),
                                cudaMemcpyHostToDevice, stream_));
        const int blocks = (int)std::min<uint64_t>((acc + 255) / 256, (uint64_t)sms * 16);
        build_batch_kernel<W><<<blocks, 256, 0, stream_>>>(d_jobs_.as<BuildJob<W>>(),
                                                          (int)build_jobs_.size(), acc);
        ++*launches;
        SB_CUDA(cudaGetLastError());
      }
      // 2. tasks on the shared spine lists, instances cheapest first.  Plain:
      // one task per instance.  Guided: one per (instance, shape-class
      // bucket), an instance's buckets by prior probability per unit of
      // work, so each instance reaches its likeliest spines first and no
      // instance waits for another's guesses.
      tasks_.clear();
      mtasks_.clear();
      const float* priors = o_.class_prior;  // n x 64 in batch mode
      const bool guided = priors != nullptr;
      uint64_t ctx_base = 0, units = 0;
      std::vector<int> naive_insts;
      struct Pending {
        double key;
        int inst, bucket;
        unsigned tmpl;
        uint64_t ctx_base, units;
      };
      std::vector<Pending> pend;
      // materialised contexts must fit in free memory: the most expensive
      // instances of the round wait for a later round if they do not
      size_t mem_free = 0, mem_total = 0;
      SB_CUDA(cudaMemGetInfo(&mem_free, &mem_total));
      const uint64_t room = mem_free + d_ctx_.bytes + pool_cached_bytes(o_.device);
      const uint64_t ctx_room = room > (1ULL << 30) ? (room - (1ULL << 30)) / sizeof(Ctx<W>) : 0;
      for (int i : order) {
        ran[i] = 0;
        const CountTable& ct = cts_[ct_of[i]];
        const int ul = hs_[i].unit_log2 > 0 ? std::min(hs_[i].unit_log2, 40) : 0;
        const ItemTemplate& tp = get_template(ct, std::min(T[i], size[i]), size[i], mask,
                                              ul ? 1ULL << ul : unit_target_, guided);
        if (!tp.ok || tp.units == 0) {
          naive_insts.push_back(i);
          ran[i] = 1;
          continue;
        }
        if (ctx_base + tp.nctxs > ctx_room && !pend.empty()) continue;  // deferred
        ran[i] = 1;
        Task mt;
        memset(&mt, 0, sizeof(mt));
        mt.ctx_base = ctx_base;
        mt.inst = (unsigned)i;
        mt.tmpl = (unsigned)tp.id;
        mt.bucket = -1;
        if (tp.nctxs) mtasks_.push_back(mt);
        if (guided) {  // this instance's buckets, likeliest per unit of work first
          const float* pr = priors + (size_t)i * 64;
          const size_t first = pend.size();
          for (int b = 0; b < 64; ++b) {
            if (tp.bucket_units[b] == 0) continue;
            // a unary-chain bucket holds both ~- and neg-rooted chains
            const double pb = b < 8 ? (double)pr[b] + (double)pr[32 + b] : (double)pr[b];
            pend.push_back({-(std::max(pb, 1e-12) / (double)tp.bucket_units[b]), i, b,
                            (unsigned)tp.id, ctx_base, tp.bucket_units[b]});
          }
          std::stable_sort(pend.begin() + first, pend.end(),
                           [](const Pending& a, const Pending& b) { return a.key < b.key; });
        } else {
          pend.push_back({0.0, i, -1, (unsigned)tp.id, ctx_base, tp.units});
        }
        ctx_base += tp.nctxs;
        *alg_ops += tp.alg;
      }
      for (const Pending& q : pend) {
        Task tk;
        memset(&tk, 0, sizeof(tk));
        tk.unit_begin = units;
        tk.ctx_base = q.ctx_base;
        tk.inst = (unsigned)q.inst;
        tk.tmpl = q.tmpl;
        tk.bucket = q.bucket;
        tasks_.push_back(tk);
        units += q.units;
      }
      if (tmpl_dirty_) {  // upload the spine lists created since the last round
        SB_CUDA(d_items_.reserve(std::max<size_t>(1, all_items_.size()) * sizeof(Item)));
        SB_CUDA(cudaMemcpyAsync(d_items_.p, all_items_.data(), all_items_.size() * sizeof(Item),
                                cudaMemcpyHostToDevice, stream_));
        SB_CUDA(d_small_.reserve(std::max<size_t>(1, all_small_.size()) * sizeof(Item)));
        SB_CUDA(cudaMemcpyAsync(d_small_.p, all_small_.data(), all_small_.size() * sizeof(Item),
                                cudaMemcpyHostToDevice, stream_));
        SB_CUDA(d_tdesc_.reserve(std::max<size_t>(1, tdescs_.size()) * sizeof(TmplDesc)));
        SB_CUDA(cudaMemcpyAsync(d_tdesc_.p, tdescs_.data(), tdescs_.size() * sizeof(TmplDesc),
                                cudaMemcpyHostToDevice, stream_));
        SB_CUDA(d_buckets_.reserve(std::max<size_t>(1, all_buckets_.size()) * sizeof(TmplBuckets)));
        SB_CUDA(cudaMemcpyAsync(d_buckets_.p, all_buckets_.data(),
                                all_buckets_.size() * sizeof(TmplBuckets), cudaMemcpyHostToDevice,
                                stream_));
        tmpl_dirty_ = false;
      }
      // 3. descriptors and per-instance best
      for (int i = 0; i < n; ++i) {
        InstDesc<W>& d = desc[i];
        memset(&d, 0, sizeof(d));
        for (int t = 1; t <= built[i]; ++t) {
          d.tab[t] = tabp(i, t);
          for (int j = 1; j < nsamp[i]; ++j) d.tabx[j - 1][t] = tabp(i, t, j);
        }
        for (int j = 1; j < nsamp[i]; ++j) d.targetx[j - 1] = (W)hs_[i].out[j];
        d.in = reinterpret_cast<const W*>(d_smp_.as<char>() + in_off[i]);
        d.out = reinterpret_cast<const W*>(d_smp_.as<char>() + out_off[i]);
        d.counts = d_cts_.as<unsigned long long>() + (size_t)ct_of[i] * (kMaxSize + 1) * kCols;
        d.best = d_best_.as<unsigned long long>() + i;
        d.ns = d_ns_.as<unsigned long long>() + 2 * (size_t)i;
        d.target = (W)hs_[i].out[0];
        d.size = size[i];
        d.S = hs_[i].S;
        d.K = hs_[i].k;
      }
      SB_CUDA(cudaMemcpyAsync(d_desc_.p, desc.data(), n * sizeof(InstDesc<W>), cudaMemcpyHostToDevice, stream_));
      SB_CUDA(cudaMemsetAsync(d_best_.p, 0xFF, (size_t)n * 8, stream_));
      unsigned long long init[3] = {0, 0, 0};
      SB_CUDA(cudaMemcpyAsync(d_scal_.p, init, sizeof(init), cudaMemcpyHostToDevice, stream_));
      SB_CUDA(cudaMemsetAsync(d_scal_.as<unsigned long long>() + 4, 0, 32, stream_));
      Params<W> p;
      memset(&p, 0, sizeof(p));
      p.insts = d_desc_.as<InstDesc<W>>();
      unsigned long long* sc = d_scal_.as<unsigned long long>();
      p.counter = sc + 0;
      p.evaluated = sc + 2;
      p.start_ns = sc + 3;
      p.flags = reinterpret_cast<int*>(sc + 4);
      p.hits = sc + 6;
      p.preq = d_preq_.as<unsigned long long>();
      p.join_off = (unsigned)join_off;
      p.maxS = maxS;
      p.maxK = maxK;
      p.stop_on_match = guided ? 2 : 1;  // guided: any verified match of the size
      p.budget_ns = o_.budget_s > 0 ? (unsigned long long)(o_.budget_s * 1e9) : 0;
      float kms = 0;
      cudaEvent_t ka, kb;
      SB_CUDA(cudaEventCreate(&ka));
      SB_CUDA(cudaEventCreate(&kb));
      SB_CUDA(cudaEventRecord(ka, stream_));
      if (!tasks_.empty()) {
        SB_CUDA(d_tasks_.reserve(tasks_.size() * sizeof(Task)));
        SB_CUDA(cudaMemcpyAsync(d_tasks_.p, tasks_.data(), tasks_.size() * sizeof(Task),
                                cudaMemcpyHostToDevice, stream_));
        p.tasks = d_tasks_.as<Task>();
        p.ntasks = (int)tasks_.size();
        p.buckets = d_buckets_.as<TmplBuckets>();
        p.tmpls = d_tdesc_.as<TmplDesc>();
        p.items = d_items_.as<Item>();
        p.nitems = (int)all_items_.size();
        p.total_units = units;
        if (ctx_base) {  // contexts of the fused spines, one task per instance
          SB_CUDA(d_ctx_.reserve(ctx_base * sizeof(Ctx<W>)));
          SB_CUDA(d_mtasks_.reserve(mtasks_.size() * sizeof(Task)));
          SB_CUDA(cudaMemcpyAsync(d_mtasks_.p, mtasks_.data(), mtasks_.size() * sizeof(Task),
                                  cudaMemcpyHostToDevice, stream_));
          p.sitems = d_small_.as<Item>();
          p.nsitems = (int)all_small_.size();
          p.nctxs = ctx_base;
          Params<W> m = p;
          m.tasks = d_mtasks_.as<Task>();
          m.ntasks = (int)mtasks_.size();
          const int mb = (int)std::min<uint64_t>((ctx_base + 255) / 256, (uint64_t)sms * 8);
          materialize_kernel<W><<<mb, 256, 0, stream_>>>(m, d_ctx_.as<Ctx<W>>());
          ++*launches;
          p.ctxs = d_ctx_.as<Ctx<W>>();
        }
        spine_kernel<W><<<grid, kThreads, smem, stream_>>>(p);
        ++*launches;
        SB_CUDA(cudaGetLastError());
      }
      for (int i : naive_insts) {  // spines too deep for this instance's tables
        Params<W> q = p;
        q.tasks = nullptr;
        q.insts = d_desc_.as<InstDesc<W>>() + i;
        const CountTable& ct = cts_[ct_of[i]];
        naive_kernel<W><<<grid, kThreads, smem, stream_>>>(q, 0, ct.n[size[i]][8]);
        ++*launches;
        SB_CUDA(cudaGetLastError());
      }
      SB_CUDA(cudaEventRecord(kb, stream_));
      SB_CUDA(cudaMemcpyAsync(best.data(), d_best_.p, (size_t)n * 8, cudaMemcpyDeviceToHost, stream_));
      SB_CUDA(cudaMemcpyAsync(ns.data(), d_ns_.p, (size_t)n * 16, cudaMemcpyDeviceToHost, stream_));
      unsigned long long hs[8];
      SB_CUDA(cudaMemcpyAsync(hs, d_scal_.p, sizeof(hs), cudaMemcpyDeviceToHost, stream_));
      SB_CUDA(cudaStreamSynchronize(stream_));
      SB_CUDA(cudaEventElapsedTime(&kms, ka, kb));
      cudaEventDestroy(ka);
      cudaEventDestroy(kb);
      *kernel_ms += kms;
      *evaluated += hs[2];
      start_ns = hs[3];
      const int* fl = reinterpret_cast<const int*>(hs + 4);
      if (fl[1]) {
        set_last_error("inversion failed on a level marked invertible");
        return SIMBA_E_INTERNAL;
      }
      const double now = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
      // 4. retire solved instances, advance the others
      for (int i : order) {
        if (!ran[i]) continue;
        Out& r = (*outs)[i];
        const CountTable& ct = cts_[ct_of[i]];
        const int s = size[i];
        if (best[i] != ~0ULL) {
          const int op = s == 1 ? 8 : op_of_rank(ct.n, s, best[i]);
          uint64_t c = 0;
          if (s == 1) c = best[i] + 1;
          else
            for (int q = 0; q <= op; ++q) c += ct.n[s][q];
          r.candidates += c;
          char buf[kMaxSize + 1];
          unrank(best[i], s, ct.n, buf);
          buf[s] = 0;
          r.postfix = buf;
          r.size = s;
          r.op = op;
          r.rank = best[i];
          r.status = host_check(r.postfix, hs_[i]) ? SIMBA_OK : SIMBA_E_INTERNAL;
          // device time of the solution: the first verified match (guided:
          // the search stops there), or the last unit of the instance that
          // ran (plain: every rank below the answer is then searched)
          const unsigned long long t = guided ? ns[2 * i] : std::max(ns[2 * i], ns[2 * i + 1]);
          r.seconds = t > start_ns ? (double)(t - start_ns) * 1e-9 : now;
          active[i] = 0;
        } else if (fl[0]) {
          r.status = SIMBA_BUDGET;
          r.seconds = now;
          active[i] = 0;
        } else {
          r.candidates += ct.n[s][8];
          swept[i] += (double)ct.n[s][8];
          if (++size[i] > last) {
            r.status = SIMBA_NOT_FOUND;
            r.seconds = now;
            active[i] = 0;
          }
        }
      }
      if (o_.verbose) {
        int solved = 0, smin = kMaxSize, smax = 0, nran = 0;
        for (int i : order) {
          if (!ran[i]) continue;
          ++nran;
          solved += best[i] != ~0ULL;
          smin = std::min(smin, size[i] - (best[i] == ~0ULL ? 1 : 0));
          smax = std::max(smax, size[i] - (best[i] == ~0ULL ? 1 : 0));
        }
        fprintf(stderr,
                "round %3d | t %8.3f s | insts %6zu (sizes %d-%d) | tasks %7zu | units %10llu | "
                "ctxs %10llu | naive %4zu | evaluated %.3e | hits %.3e | kernels %9.3f ms | "
                "solved %5d%s\n",
                *rounds, now, (size_t)nran, smin, smax, tasks_.size(), (unsigned long long)units,
                (unsigned long long)ctx_base, naive_insts.size(), (double)hs[2], (double)hs[6], kms,
                solved, fl[0] ? " | budget" : "");
      }
    }
    SB_CUDA(cudaEventRecord(e1_, stream_));
    SB_CUDA(cudaEventSynchronize(e1_));
    float ms = 0;
    SB_CUDA(cudaEventElapsedTime(&ms, e0_, e1_));
    *device_ms = ms;
    for (auto& r : *outs) *candidates += r.candidates;
    return 0;
  }

 private:
  // Width of a cost-ordered round: instances whose swept total after their
  // next size is within this factor of the cheapest one run in the round
  // (SIMBA_ROUND_GROWTH overrides; 0 or less means every active instance,
  // i.e. all instances step through the sizes together).
  static double round_growth() {
    const char* e = getenv("SIMBA_ROUND_GROWTH");
    const double g = e ? atof(e) : 64.0;
    return g > 0 ? std::max(g, 1.0) : std::numeric_limits<double>::infinity();
  }

  // Bucket of a spine in a guided list: its (primary) shape class.
  static int bucket_of(const Item& it, int s) {
    int a, b;
    spine_classes(it, s, &a, &b);
    return a < 0 ? 0 : a;
  }

  const ItemTemplate& get_template(const CountTable& ct, int T, int s, uint64_t mask,
                                   uint64_t unit_target, bool guided = false) {
    int ul = 0;
    while ((1ULL << ul) < unit_target && ul < 63) ++ul;
    const uint64_t key = ((uint64_t)guided << 32) | ((uint64_t)ul << 24) |
                         ((uint64_t)ct.terms << 16) | ((uint64_t)T << 8) | (uint64_t)s;
    auto f = templates_.find(key);
    if (f != templates_.end()) return f->second;
    ItemTemplate tp;
    std::vector<Item> items;
    if (s <= T) {
      Item it;
      memset(&it, 0, sizeof(it));
      it.bottom = (int8_t)s;
      it.coefv = 1;
      it.nv = ct.n[s][8];
      items.push_back(it);
    } else if ((s - 1) / 2 > T) {
      tp.ok = false;
    } else {
      Enumerator en;
      en.ct = &ct;
      en.T = T;
      en.mask = mask;
      en.items = &items;
      std::vector<Level> lv;
      std::vector<ChainClass> top{{1, 0, 0}};
      en.rec(s, lv, 1, 0, top);
      if (en.too_deep) tp.ok = false;
    }
    if (tp.ok) {
      for (auto& it : items) {
        for (int l = 0; l < it.depth; ++l)
          if (it.lv[l].kind == 1) it.lv[l].c &= mask;
        finish_structure(it, mask);
      }
      if (guided)  // fused groups stay inside one bucket
        for (auto& it : items) it.prio = (float)bucket_of(it, s);
      fuse_small(items, &tp.small, &tp.nctxs, ct, 1ULL << 22, guided);
      for (auto& it : items) finish_layout(it, kThreads, unit_target, 1 << std::min(o_.lanes_log2, 8));
      // Spines of one kernel variant (fused / full compare / explicit
      // levels) run together: CTAs of a round work through a few lists at a
      // time, and mixing variants there thrashes the instruction cache.
      auto variant = [](const Item& a) {
        return (a.full == 2 ? 0 : 32) + (a.fused ? 0 : 16) + (a.full ? 0 : 8) +
               std::min<int>(a.nexp, kMaxExplicit + 1);
      };
      if (guided)
        std::stable_sort(items.begin(), items.end(), [&](const Item& a, const Item& b) {
          if (a.prio != b.prio) return a.prio < b.prio;
          if (variant(a) != variant(b)) return variant(a) < variant(b);
          return a.base < b.base;
        });
      else
        std::stable_sort(items.begin(), items.end(), [&](const Item& a, const Item& b) {
          if (variant(a) != variant(b)) return variant(a) < variant(b);
          return a.base < b.base;
        });
      for (auto& it : items) {
        tp.units += item_units(it);
        tp.cand += (double)it.nctx * (double)it.nv;
        tp.alg += item_alg_ops(it, sizeof(W));
      }
      uint64_t ub = 0;
      for (auto& it : items) {  // unit_begin relative to the list
        it.unit_begin = ub;
        ub += item_units(it);
      }
      TmplDesc td;
      td.item_off = all_items_.size();
      td.nitems = (unsigned)items.size();
      td.small_off = all_small_.size();
      td.nsmall = (unsigned)tp.small.size();
      td.bucket_off = 0;
      if (guided) {
        TmplBuckets tb;
        memset(&tb, 0, sizeof(tb));
        size_t q = 0;
        uint64_t uacc = 0;
        for (int b = 0; b < 64; ++b) {
          tb.item[b] = (unsigned)q;
          tb.unit[b] = uacc;
          for (; q < items.size() && (int)items[q].prio == b; ++q) uacc += item_units(items[q]);
        }
        tb.item[64] = (unsigned)q;
        tb.unit[64] = uacc;
        td.bucket_off = all_buckets_.size();
        all_buckets_.push_back(tb);
        for (int b = 0; b < 64; ++b) tp.bucket_units[b] = tb.unit[b + 1] - tb.unit[b];
      }
      all_items_.insert(all_items_.end(), items.begin(), items.end());
      all_small_.insert(all_small_.end(), tp.small.begin(), tp.small.end());
      tp.id = (int)tdescs_.size();
      tdescs_.push_back(td);
      tmpl_dirty_ = true;
      tp.items = std::move(items);
    }
    return templates_.emplace(key, std::move(tp)).first->second;
  }

  std::vector<HostInstance> hs_;
  EngineOptions o_;
  int64_t inst_budget_;
  uint64_t unit_target_;
  cudaStream_t stream_ = nullptr;
  bool own_stream_ = true;
  cudaEvent_t e0_ = nullptr, e1_ = nullptr;
  std::vector<CountTable> cts_;
  std::map<uint64_t, ItemTemplate> templates_;
  std::vector<Item> all_items_, all_small_;  // every spine list, concatenated
  std::vector<TmplDesc> tdescs_;
  std::vector<TmplBuckets> all_buckets_;
  std::vector<Task> mtasks_;  // one per instance with fused spines (materialisation)
  bool tmpl_dirty_ = false;
  std::vector<Task> tasks_;
  std::vector<BuildJob<W>> build_jobs_;
  DevBuf d_tab_, d_smp_, d_cts_, d_best_, d_desc_, d_scal_, d_items_, d_small_, d_ctx_, d_jobs_,
      d_tasks_, d_tdesc_, d_buckets_, d_mtasks_, d_ns_, d_preq_;
};

template <class W>
int batch_typed(const std::vector<HostInstance>& hs, int max_size, const EngineOptions& o,
                int64_t inst_table_bytes, BatchOutcome* out) {
  const uint64_t unit_target = 1ULL << (o.unit_log2 > 0 ? std::min(o.unit_log2, 40) : 22);
  Batch<W> b(hs, o, inst_table_bytes > 0 ? inst_table_bytes : (8LL << 20), unit_target);
  std::vector<typename Batch<W>::Out> r;
  const int rc = b.run(max_size, &r, &out->device_ms, &out->rounds, &out->launches, &out->evaluated,
                       &out->candidates, &out->alg_ops, &out->kernel_ms);
  if (rc) return rc;
  out->items.resize(r.size());
  for (size_t i = 0; i < r.size(); ++i) {
    BatchItemOutcome& d = out->items[i];
    d.status = r[i].status;
    d.size = r[i].size;
    d.op = r[i].op;
    d.rank = r[i].rank;
    d.postfix = r[i].postfix;
    d.seconds = r[i].seconds;
    d.candidates = r[i].candidates;
  }
  return 0;
}

// Creates and initialises a session for word type W (search_u32.cu / search_u64.cu).
template <class W>
int make_search_typed(const HostInstance& h, const EngineOptions& o, SearchSession** out) {
  auto s = std::make_unique<Search<W>>(h, o);
  const int rc = s->init();
  if (rc) return rc;
  *out = s.release();
  return 0;
}

}  // namespace simba
