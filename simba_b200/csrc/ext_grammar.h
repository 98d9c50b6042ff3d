// Extended grammar: the operator set the reference declares but leaves
// switched off -- its Op enum (vfb/src/full-cache.cu:166-179) lists
//   ~ & | ^ << >> neg + - * / %
// and the enumeration table (:460-472) comments out <<, >>, / and %;
// evaluateRPN (simba/src/mba.cuh:71-131) evaluates '<' '>' '/' '%' but has
// no caller.  Here the grammar is an option (simba_options.grammar = 1) of
// simba_solve and vfb_solve.
//
// Rank space (plain search): sizes in increasing order, the twelve operator
// blocks of a size in the order above, the SIMBA count recurrence with the
// four new operators counted like '-' (none is commutative: every left size
// is enumerated).  Postfix characters: ~ & | ^ < > # + - * / %.
//
// Semantics on w-bit words: x << y and x >> y (logical) give 0 when y >= w
// (the GPU's clamped shift of the reference's `L[i] << R[i]`,
// full-cache.cu:215-220); x / y and x % y follow VFB's zero-divisor rule
// (full-cache.cu:230-256): VFB composes whole vectors and takes the
// dividend vector when any divisor element is 0; the plain search decides a
// candidate one sample at a time and applies the same fallback per sample
// (x / 0 = x % 0 = x).
//
// Operator codes in results: the base codes 0..7 (grammar.h), then
// 9 '<<', 10 '>>', 11 '/', 12 '%' (8 stays "a variable").  Terminals are
// '0' + index with at most 10 terminals ('<' and '>' follow '9').
#pragma once
#include <cstdint>

#include "grammar.h"

namespace simba {

constexpr int kExtOps = 12;
constexpr int kExtCols = 13;  // 12 operator columns + total
constexpr int kExtMaxTerms = 10;
enum ExtCode : int { OP_SHL = 9, OP_SHR = 10, OP_DIV = 11, OP_MOD = 12 };

// position in the extended order -> operator code, character
SB_HD int ext_code(int e) {
  const int c[kExtOps] = {OP_NOT, OP_AND, OP_OR, OP_XOR, OP_SHL, OP_SHR,
                          OP_NEG, OP_ADD, OP_SUB, OP_MUL, OP_DIV, OP_MOD};
  return c[e];
}
SB_HD char ext_char(int e) {
  const char c[kExtOps] = {'~', '&', '|', '^', '<', '>', '#', '+', '-', '*', '/', '%'};
  return c[e];
}
SB_HD bool ext_unary(int e) { return e == 0 || e == 6; }
SB_HD bool ext_commutative(int e) { return e == 1 || e == 2 || e == 3 || e == 7 || e == 9; }

// character -> operator code (base and extended), -1 for a terminal
SB_HD int ext_char_code(char ch) {
  switch (ch) {
    case '<': return OP_SHL;
    case '>': return OP_SHR;
    case '/': return OP_DIV;
    case '%': return OP_MOD;
  }
  return char_op(ch);
}

// operator code -> postfix character (base and extended codes)
SB_HD char code_char(int code) {
  switch (code) {
    case OP_SHL: return '<';
    case OP_SHR: return '>';
    case OP_DIV: return '/';
    case OP_MOD: return '%';
  }
  return op_char(code);
}

// character -> position in the extended order, -1 for a terminal
SB_HD int ext_char_pos(char ch) {
  for (int e = 0; e < kExtOps; ++e)
    if (ext_char(e) == ch) return e;
  return -1;
}

struct ExtCountTable {
  uint64_t n[kMaxSize + 1][kExtCols];
};

inline bool build_ext_count_table(int max_size, int k, ExtCountTable* t) {
  bool ok = true;
  for (int s = 0; s <= kMaxSize; ++s)
    for (int c = 0; c < kExtCols; ++c) t->n[s][c] = 0;
  if (max_size >= 1) t->n[1][kExtOps] = (uint64_t)k;
  if (max_size >= 2) {
    t->n[2][0] = t->n[2][6] = (uint64_t)k;
    t->n[2][kExtOps] = 2 * (uint64_t)k;
  }
  for (int s = 3; s <= max_size; ++s) {
    unsigned __int128 u = t->n[s - 1][kExtOps], c = 0, nc = 0, tot = 0;
    for (int j = 1; j <= s - 2; ++j) {
      const unsigned __int128 p = (unsigned __int128)t->n[j][kExtOps] * t->n[s - 1 - j][kExtOps];
      nc += p;
      if (j <= (s - 1) / 2) c += p;
    }
    for (int e = 0; e < kExtOps; ++e) {
      const unsigned __int128 v = ext_unary(e) ? u : (ext_commutative(e) ? c : nc);
      if ((v >> 64) != 0) ok = false;
      t->n[s][e] = (uint64_t)v;
      tot += v;
    }
    if ((tot >> 64) != 0) ok = false;
    t->n[s][kExtOps] = (uint64_t)tot;
  }
  return ok;
}

// rank -> postfix in the extended rank space (the unranking of grammar.h
// with twelve operator blocks); an explicit stack, host and device.
SB_HD void ext_unrank(uint64_t rank, int size, const uint64_t (*n)[kExtCols], char* out) {
  struct Ent { uint64_t r; int size; int pos; };
  Ent st[kMaxSize];
  int sp = 0;
  st[0] = {rank, size, 0};
  while (sp >= 0) {
    Ent e = st[sp--];
    if (e.size == 1) {
      out[e.pos] = (char)('0' + (int)(e.r % n[1][kExtOps]));
      continue;
    }
    int op = 0;
    while (op < kExtOps - 1 && e.r >= n[e.size][op]) e.r -= n[e.size][op++];
    const int sub = e.size - 1;
    out[e.pos + sub] = ext_char(op);
    if (ext_unary(op) || sub < 2) {
      if (!ext_unary(op)) out[e.pos + sub] = '~';  // only for ranks out of range
      st[++sp] = {e.r, sub, e.pos};
      continue;
    }
    int f = 1;
    for (;;) {
      const uint64_t blk = n[f][kExtOps] * n[sub - f][kExtOps];
      if (e.r < blk || f >= sub - 1) break;
      e.r -= blk;
      ++f;
    }
    const uint64_t nr = n[sub - f][kExtOps];
    st[++sp] = {e.r / nr, f, e.pos};
    st[++sp] = {e.r % nr, sub - f, e.pos + f};
  }
}

// postfix -> rank in the extended rank space (inverse of ext_unrank).
inline bool ext_rank_of(const char* p, int len, const uint64_t (*n)[kExtCols], int k, uint64_t* out) {
  if (len <= 0) return false;
  if (len == 1) {
    const int t = p[0] - '0';
    if (t < 0 || t >= k || t > 9) return false;
    *out = (uint64_t)t;
    return true;
  }
  const int e = ext_char_pos(p[len - 1]);
  if (e < 0) return false;
  const int sub = len - 1;
  uint64_t r = 0;
  for (int q = 0; q < e; ++q) r += n[len][q];
  if (ext_unary(e)) {
    uint64_t c;
    if (!ext_rank_of(p, sub, n, k, &c)) return false;
    *out = r + c;
    return true;
  }
  int need = 1, f = -1;
  for (int i = sub - 1; i >= 0; --i) {
    const int o = ext_char_pos(p[i]);
    need -= 1;
    if (o >= 0) need += ext_unary(o) ? 1 : 2;
    if (need == 0) {
      f = i;
      break;
    }
  }
  if (f <= 0) return false;
  if (ext_commutative(e) && f > sub - f) return false;
  for (int g = 1; g < f; ++g) r += n[g][kExtOps] * n[sub - g][kExtOps];
  uint64_t a, b;
  if (!ext_rank_of(p, f, n, k, &a) || !ext_rank_of(p + f, sub - f, n, k, &b)) return false;
  *out = r + a * n[sub - f][kExtOps] + b;
  return true;
}

// One operator (by code) on one sample of W-bit words, per-sample rule.
template <class W>
SB_HD W ext_apply(int code, W l, W r) {
  constexpr W kBits = (W)(8 * sizeof(W));
  switch (code) {
    case OP_NOT: return (W)~r;
    case OP_NEG: return (W)(W(0) - r);
    case OP_AND: return l & r;
    case OP_OR: return l | r;
    case OP_XOR: return l ^ r;
    case OP_ADD: return (W)(l + r);
    case OP_SUB: return (W)(l - r);
    case OP_MUL: return (W)(l * r);
    case OP_SHL: return r >= kBits ? W(0) : (W)(l << r);
    case OP_SHR: return r >= kBits ? W(0) : (W)(l >> r);
    case OP_DIV: return r == 0 ? l : (W)(l / r);
    default: return r == 0 ? l : (W)(l % r);  // OP_MOD
  }
}

}  // namespace simba
