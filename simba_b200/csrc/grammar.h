// Grammar, count table and rank <-> expression bijection shared by host and
// device code.
//
// Rank space (the contract of the reference search): for a size s the ranks
// [0, N(s)) are ordered by root operator in the order ~ & | ^ neg + - *
// (simba/src/globals.cuh:13-15).  Inside a binary operator block the ranks
// are ordered by left size f = 1, 2, ... and inside a split by
// (left rank) * N(s-1-f) + (right rank) (simba/src/nocache.cu:53-79).
// Commutative operators only enumerate left size <= right size
// (nocache.cu:137-140); '-' enumerates every split (:141-144).
#pragma once
#include <cstdint>

#if defined(__CUDACC__)
#define SB_HD __host__ __device__ __forceinline__
#else
#define SB_HD inline
#endif

namespace simba {

constexpr int kMaxSize = 32;     // largest expression size (reference limit)
constexpr int kMaxTerms = 16;    // terminals (variables incl. a constant)
constexpr int kMaxSamples = 256; // samples staged in shared memory
constexpr int kCols = 9;         // 8 operator columns + total

enum Op : int { OP_NOT = 0, OP_AND, OP_OR, OP_XOR, OP_NEG, OP_ADD, OP_SUB, OP_MUL };

SB_HD bool is_unary(int op) { return op == OP_NOT || op == OP_NEG; }
SB_HD bool is_commutative(int op) { return op != OP_SUB; }

// Postfix token characters: the reference writes terminals as '0' + index and
// operators as these characters (globals.cuh:13-15, '#' = unary minus).
SB_HD char op_char(int op) {
  const char c[8] = {'~', '&', '|', '^', '#', '+', '-', '*'};
  return c[op];
}

SB_HD int char_op(char c) {
  switch (c) {
    case '~': return OP_NOT;
    case '&': return OP_AND;
    case '|': return OP_OR;
    case '^': return OP_XOR;
    case '#': return OP_NEG;
    case '+': return OP_ADD;
    case '-': return OP_SUB;
    case '*': return OP_MUL;
  }
  return -1;
}

// numForm[size][op] with column 8 = total; N(1) = k, N(2) = 2k
// (nocache.cu:117-160).  Computed with 128-bit sums; returns false when a
// count needs more than 64 bits (the reference would wrap silently).
struct CountTable {
  uint64_t n[kMaxSize + 1][kCols];
  int max_size;
  int terms;
};

inline bool build_count_table(int max_size, int k, CountTable* t) {
  bool ok = true;
  for (int s = 0; s <= kMaxSize; ++s)
    for (int c = 0; c < kCols; ++c) t->n[s][c] = 0;
  t->max_size = max_size;
  t->terms = k;
  if (max_size >= 1) t->n[1][8] = (uint64_t)k;
  if (max_size >= 2) {
    t->n[2][OP_NOT] = (uint64_t)k;
    t->n[2][OP_NEG] = (uint64_t)k;
    t->n[2][8] = 2 * (uint64_t)k;
  }
  for (int s = 3; s <= max_size; ++s) {
    unsigned __int128 u = t->n[s - 1][8], c = 0, nc = 0;
    for (int j = 1; j <= s - 2; ++j) {
      unsigned __int128 p = (unsigned __int128)t->n[j][8] * t->n[s - 1 - j][8];
      nc += p;
      if (j <= (s - 1) / 2) c += p;
    }
    unsigned __int128 tot = 2 * u + 5 * c + nc;
    if ((tot >> 64) != 0) ok = false;
    for (int op = 0; op < 8; ++op)
      t->n[s][op] = is_unary(op) ? (uint64_t)u : (op == OP_SUB ? (uint64_t)nc : (uint64_t)c);
    t->n[s][8] = (uint64_t)tot;
  }
  return ok;
}

// First rank of operator block `op` inside size s.
SB_HD uint64_t op_offset(const uint64_t (*n)[kCols], int s, int op) {
  uint64_t o = 0;
  for (int i = 0; i < op; ++i) o += n[s][i];
  return o;
}

// Root operator block containing `rank` of size s.
SB_HD int op_of_rank(const uint64_t (*n)[kCols], int s, uint64_t rank) {
  uint64_t o = 0;
  for (int op = 0; op < 8; ++op) {
    if (rank < o + n[s][op]) return op;
    o += n[s][op];
  }
  return -1;
}

// rank -> postfix (size characters, no terminator).  Same bijection as the
// reference's numberToFormula (nocache.cu:23-83), written as an explicit
// work stack so that it also runs on the device without recursion.
SB_HD void unrank(uint64_t rank, int size, const uint64_t (*n)[kCols], char* out) {
  struct Ent { uint64_t r; int size; int pos; };
  Ent st[kMaxSize];
  int sp = 0;
  st[0] = {rank, size, 0};
  while (sp >= 0) {
    Ent e = st[sp--];
    if (e.size == 1) {
      out[e.pos] = (char)('0' + (int)(e.r % n[1][8]));
      continue;
    }
    // Both scans are bounded: a rank outside [0, N(size)) yields some
    // well-formed expression instead of reading past the table.
    int op = 0;
    while (op < 7 && e.r >= n[e.size][op]) e.r -= n[e.size][op++];
    const int sub = e.size - 1;
    out[e.pos + sub] = op_char(op);
    if (is_unary(op) || sub < 2) {
      if (!is_unary(op)) out[e.pos + sub] = op_char(OP_NOT);
      st[++sp] = {e.r, sub, e.pos};
      continue;
    }
    int f = 1;
    for (;;) {
      uint64_t blk = n[f][8] * n[sub - f][8];
      if (e.r < blk || f >= sub - 1) break;
      e.r -= blk;
      ++f;
    }
    const uint64_t nr = n[sub - f][8];
    st[++sp] = {e.r / nr, f, e.pos};
    st[++sp] = {e.r % nr, sub - f, e.pos + f};
  }
}

// (a * b) mod n for any 64-bit a, b < n: shift-and-add, so it needs no
// 128-bit division (used only when a match is recorded, never per candidate).
SB_HD uint64_t mulmod64(uint64_t a, uint64_t b, uint64_t n) {
  uint64_t r = 0;
  a %= n;
  b %= n;
  while (b) {
    if (b & 1) {
      const uint64_t t = r + a;
      r = (t < r || t >= n) ? t - n : t;
    }
    const uint64_t d = a + a;
    a = (d < a || d >= n) ? d - n : d;
    b >>= 1;
  }
  return r;
}

// RTid order (the simba_rtid build, nocache_rtid.cu:85-95): position t of
// an operator block of N ranks visits the rank (t * C) mod N of the block,
// C = 2246822507.  That C = 15809 * 142123, and t * C wraps 64 bits for
// t > 8.2e9, so the reference's map misses ranks for some N; here the
// multiplier is the smallest c >= C coprime to N, and the product is taken
// exactly, which makes the order a bijection of the block.
constexpr uint64_t kRtidMultiplier = 2246822507ULL;

inline uint64_t gcd64(uint64_t a, uint64_t b) {
  while (b) {
    const uint64_t t = a % b;
    a = b;
    b = t;
  }
  return a;
}

inline uint64_t rtid_multiplier(uint64_t n) {
  uint64_t c = kRtidMultiplier;
  while (n > 1 && gcd64(c % n, n) != 1) ++c;
  return c;
}

// Inverse of c modulo n (gcd(c, n) = 1), by the extended Euclidean algorithm.
inline uint64_t inverse_mod(uint64_t c, uint64_t n) {
  if (n <= 1) return 0;
  __int128 t = 0, nt = 1, r = (__int128)n, nr = (__int128)(c % n);
  while (nr != 0) {
    const __int128 q = r / nr, a = t - q * nt, b = r - q * nr;
    t = nt;
    nt = a;
    r = nr;
    nr = b;
  }
  if (t < 0) t += (__int128)n;
  return (uint64_t)t;
}

// RTid position (as off + t) of `rank` in its operator block of size s, and
// back.  Keys of one block lie in the block's rank interval, so the minimum
// key of a size sits in its first operator block with a match.
inline uint64_t rtid_key(const uint64_t (*n)[kCols], int s, uint64_t rank) {
  const int op = op_of_rank(n, s, rank);
  const uint64_t off = op_offset(n, s, op), N = n[s][op];
  return off + mulmod64(rank - off, inverse_mod(rtid_multiplier(N), N), N);
}

inline uint64_t rtid_rank(const uint64_t (*n)[kCols], int s, uint64_t key) {
  const int op = op_of_rank(n, s, key);
  const uint64_t off = op_offset(n, s, op), N = n[s][op];
  return off + mulmod64(key - off, rtid_multiplier(N), N);
}

// postfix -> rank (inverse of unrank), used to check the bijection and to
// locate a known expression in the rank space.  Returns false on a malformed
// string or if a binary node's split is not enumerated (commutative with
// left size > right size).
inline bool rank_of(const char* p, int len, const uint64_t (*n)[kCols], int k, uint64_t* out) {
  if (len <= 0) return false;
  if (len == 1) {
    int t = p[0] - '0';
    if (t < 0 || t >= k) return false;
    *out = (uint64_t)t;
    return true;
  }
  const int op = char_op(p[len - 1]);
  if (op < 0) return false;
  const int sub = len - 1;
  uint64_t r = op_offset(n, len, op);
  if (is_unary(op)) {
    uint64_t c;
    if (!rank_of(p, sub, n, k, &c)) return false;
    *out = r + c;
    return true;
  }
  // The right operand is the complete subtree that ends just before the
  // operator: scan backwards counting open operand slots.
  int need = 1, f = -1;
  for (int i = sub - 1; i >= 0; --i) {
    int o = char_op(p[i]);
    need -= 1;
    if (o >= 0) need += is_unary(o) ? 1 : 2;
    if (need == 0) { f = i; break; }
  }
  if (f <= 0) return false;
  if (is_commutative(op) && f > sub - f) return false;
  for (int g = 1; g < f; ++g) r += n[g][8] * n[sub - g][8];
  uint64_t a, b;
  if (!rank_of(p, f, n, k, &a) || !rank_of(p + f, sub - f, n, k, &b)) return false;
  *out = r + a * n[sub - f][8] + b;
  return true;
}

}  // namespace simba
