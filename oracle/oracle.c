/*
 * CPU oracle for the SIMBA / VFB search -- TEST INFRASTRUCTURE ONLY.
 *
 * Restates the reference's algorithms in plain C so that the CUDA product
 * can be checked against them; only tests/, the smoke check and bench.py's
 * CPU-baseline leg call this code, never the product.  Every function cites
 * the reference lines it follows (paths relative to the reference project).
 *
 * Word width: the reference computes in uint32_t (simba/src/mba.cuh:8); the
 * oracle takes word_bits = 32 or 64 and wraps every result to that width.
 */
#include "oracle.h"

#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

static const char OP_CHARS[8] = {'~', '&', '|', '^', '#', '+', '-', '*'};

int orc_max_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

/* Count table numForm[size][op], column 8 = total of the size.
 * simba/src/nocache.cu:117-160.  Unary columns (0 '~', 4 '#') hold N(s-1);
 * commutative binary columns sum N(j) N(s-1-j) over j <= (s-1)/2; column 6
 * ('-') sums over every j in 1..s-2.  Returns -1 if a count overflows 64 bits
 * (the reference would wrap silently). */
int orc_count_table(int max_size, int n_terms, uint64_t *t) {
  int overflow = 0;
  memset(t, 0, sizeof(uint64_t) * 9 * (size_t)(max_size + 1));
  if (max_size >= 1) t[1 * 9 + 8] = (uint64_t)n_terms;
  if (max_size >= 2) {
    t[2 * 9 + 0] = (uint64_t)n_terms;
    t[2 * 9 + 4] = (uint64_t)n_terms;
    t[2 * 9 + 8] = 2 * (uint64_t)n_terms;
  }
  for (int i = 3; i <= max_size; ++i) {
    unsigned __int128 u = t[(i - 1) * 9 + 8], c = 0, n = 0;
    for (int j = 1; j <= (i - 1) / 2; ++j)
      c += (unsigned __int128)t[j * 9 + 8] * t[(i - j - 1) * 9 + 8];
    for (int j = 1; j <= i - 2; ++j)
      n += (unsigned __int128)t[j * 9 + 8] * t[(i - j - 1) * 9 + 8];
    unsigned __int128 tot = 2 * u + 5 * c + n;
    if (tot >> 64) overflow = 1;
    t[i * 9 + 0] = (uint64_t)u;
    t[i * 9 + 1] = t[i * 9 + 2] = t[i * 9 + 3] = (uint64_t)c;
    t[i * 9 + 4] = (uint64_t)u;
    t[i * 9 + 5] = (uint64_t)c;
    t[i * 9 + 6] = (uint64_t)n;
    t[i * 9 + 7] = (uint64_t)c;
    t[i * 9 + 8] = (uint64_t)tot;
  }
  return overflow ? -1 : 0;
}

/* Rank -> postfix string, simba/src/nocache.cu:23-83.  The root operator is
 * found by a prefix scan over the op columns (:53-57), the left size by a
 * prefix scan over N(f) N(size-1-f) for f = 1, 2, ... (:71-75), then the
 * left rank is n / N(right) and the right rank n % N(right) (:77-79).  The
 * operator is written at the last position of the subtree (:59-60). */
static void unrank_rec(uint64_t n, int size, const uint64_t *t, char *out) {
  if (size == 1) {
    out[0] = (char)('0' + (int)n);
    return;
  }
  uint64_t part = 0;
  int op = 0;
  while (n >= part + t[size * 9 + op]) part += t[size * 9 + op++];
  n -= part;
  int sub = size - 1;
  out[sub] = OP_CHARS[op];
  if (op == ORC_NOT || op == ORC_NEG) {
    unrank_rec(n, sub, t, out);
    return;
  }
  uint64_t fpart = 0;
  int f = 1;
  while (n >= fpart + t[f * 9 + 8] * t[(sub - f) * 9 + 8]) {
    fpart += t[f * 9 + 8] * t[(sub - f) * 9 + 8];
    f++;
  }
  n -= fpart;
  uint64_t r = t[(sub - f) * 9 + 8];
  unrank_rec(n / r, f, t, out);
  unrank_rec(n % r, sub - f, t, out + f);
}

void orc_unrank(uint64_t rank, int size, const uint64_t *t, char *postfix) {
  unrank_rec(rank, size, t, postfix);
}

static inline uint64_t wmask(int bits) { return bits == 64 ? ~0ULL : 0xFFFFFFFFULL; }

static inline uint64_t apply_op(char c, uint64_t l, uint64_t r, uint64_t m) {
  switch (c) {
    case '~': return ~r & m;
    case '#': return (0 - r) & m;
    case '&': return l & r;
    case '|': return l | r;
    case '^': return l ^ r;
    case '+': return (l + r) & m;
    case '-': return (l - r) & m;
    case '*': return (l * r) & m;
  }
  return 0;
}

/* Evaluate a postfix expression on one sample (one input row of k words),
 * following the token interpreter of simba/src/mba.cuh:11-61. */
uint64_t orc_eval1(const char *p, int len, int bits, const uint64_t *row) {
  uint64_t st[ORC_MAX_SIZE + 8];
  int sp = -1;
  const uint64_t m = wmask(bits);
  for (int j = 0; j < len; ++j) {
    char c = p[j];
    if (c == '~' || c == '#') {
      st[sp] = apply_op(c, 0, st[sp], m);
    } else if (c == '&' || c == '|' || c == '^' || c == '+' || c == '-' || c == '*') {
      uint64_t r = st[sp--];
      st[sp] = apply_op(c, st[sp], r, m);
    } else {
      st[++sp] = row[c - '0'] & m;
    }
  }
  return st[0];
}

/* is_solution_rpn, simba/src/mba.cuh:6-69: every sample must match, and the
 * test stops at the first mismatching sample. */
int orc_check(const char *p, int len, int bits, int k, int S, const uint64_t *in,
              const uint64_t *out) {
  const uint64_t m = wmask(bits);
  for (int i = 0; i < S; ++i)
    if (orc_eval1(p, len, bits, in + (size_t)i * k) != (out[i] & m)) return 0;
  return 1;
}

static inline void atomic_min_u64(uint64_t *p, uint64_t v) {
  uint64_t cur = __atomic_load_n(p, __ATOMIC_RELAXED);
  while (v < cur && !__atomic_compare_exchange_n(p, &cur, v, 0, __ATOMIC_RELAXED,
                                                 __ATOMIC_RELAXED)) {
  }
}

#define ORC_CHUNK 2048

/* Scan ranks [lo, hi) of one size; returns the number of ranks evaluated,
 * the minimum matching rank in *best (unchanged if none).  Chunks above the
 * best match found so far are skipped, which never changes the minimum. */
static int64_t scan(int bits, int k, int S, const uint64_t *in, const uint64_t *out,
                    const uint64_t *t, int size, uint64_t lo, uint64_t hi, int nth,
                    uint64_t *best, uint64_t *hits) {
  if (hi <= lo) return 0;
  const uint64_t n = hi - lo;
  const int64_t nchunks = (int64_t)((n + ORC_CHUNK - 1) / ORC_CHUNK);
  int64_t evaluated = 0;
  uint64_t nh = 0;
#ifdef _OPENMP
#pragma omp parallel for schedule(dynamic, 4) num_threads(nth) reduction(+ : evaluated, nh)
#endif
  for (int64_t c = 0; c < nchunks; ++c) {
    uint64_t a = lo + (uint64_t)c * ORC_CHUNK;
    uint64_t b = a + ORC_CHUNK < hi ? a + ORC_CHUNK : hi;
    if (a > __atomic_load_n(best, __ATOMIC_RELAXED)) continue;
    char p[ORC_MAX_SIZE + 1];
    for (uint64_t r = a; r < b; ++r) {
      orc_unrank(r, size, t, p);
      evaluated++;
      if (orc_check(p, size, bits, k, S, in, out)) {
        nh++;
        atomic_min_u64(best, r);
        break;
      }
    }
  }
  (void)nth;
  if (hits) *hits += nh;
  return evaluated;
}

int64_t orc_scan_range(int bits, int k, int S, const uint64_t *in, const uint64_t *out,
                       int size, uint64_t lo, uint64_t hi, int nth, uint64_t *min_rank,
                       uint64_t *n_hits) {
  uint64_t t[(ORC_MAX_SIZE + 1) * 9];
  if (size < 2 || size > ORC_MAX_SIZE) return -1;
  orc_count_table(size, k, t);
  uint64_t best = ~0ULL, nh = 0;
  if (nth <= 0) nth = orc_max_threads();
  int64_t e = scan(bits, k, S, in, out, t, size, lo, hi, nth, &best, &nh);
  if (min_rank) *min_rank = best;
  if (n_hits) *n_hits = nh;
  return e;
}

/* NoCache::solve, simba/src/nocache.cu:197-289: sizes 1 .. max_size-1 in
 * order, operators 0..7 within a size, a whole (size, op) block at a time,
 * stop after the first block that holds a match.  Size 1 has no operator
 * blocks (numForm[1][0..7] = 0), so a bare variable is never returned unless
 * include_edges is set, which also searches size 1 and max_size itself.
 * Where the reference returns whichever thread of the block wins its
 * atomicCAS (:102-105), the oracle returns the minimum matching rank. */
int orc_search(int bits, int k, int S, const uint64_t *in, const uint64_t *out, int max_size,
               int include_edges, int nth, orc_result *res) {
  memset(res, 0, sizeof(*res));
  if (max_size > ORC_MAX_SIZE || k > ORC_MAX_TERMS || k < 1 || S < 1) return -2;
  uint64_t t[(ORC_MAX_SIZE + 1) * 9];
  if (orc_count_table(max_size, k, t) != 0) return -3;
  if (nth <= 0) nth = orc_max_threads();
  const uint64_t m = wmask(bits);
  if (include_edges) {
    for (int v = 0; v < k; ++v) {
      res->candidates++;
      res->per_size[1]++;
      int ok = 1;
      for (int i = 0; i < S && ok; ++i) ok = (in[(size_t)i * k + v] & m) == (out[i] & m);
      if (ok) {
        res->found = 1;
        res->size = 1;
        res->op = 8;
        res->rank = (uint64_t)v;
        res->postfix[0] = (char)('0' + v);
        return 1;
      }
    }
  }
  const int last = include_edges ? max_size : max_size - 1;
  for (int s = 2; s <= last; ++s) {
    uint64_t off = 0;
    for (int op = 0; op < 8; ++op) {
      uint64_t N = t[s * 9 + op];
      res->candidates += N;
      res->per_size[s] += N;
      uint64_t best = ~0ULL;
      if (N) scan(bits, k, S, in, out, t, s, off, off + N, nth, &best, NULL);
      if (best != ~0ULL) {
        res->found = 1;
        res->size = s;
        res->op = op;
        res->rank = best;
        orc_unrank(best, s, t, res->postfix);
        res->postfix[s] = 0;
        return 1;
      }
      off += N;
    }
  }
  return 0;
}

/* ---------------------------------------------------------------------------
 * RTid order: simba/src/nocache_rtid.cu:85-95.  Thread t of an operator
 * block of N ranks (grid ceil(N/1024)*1024) evaluates rank (t * C) % N with
 * C = 2246822507 in 64-bit arithmetic.  mode 1 restates exactly that map,
 * over every launched t (the reference's own visiting set: C = 15809 *
 * 142123 is not coprime to every N, and t * C wraps for t > 8.2e9, so some
 * ranks may be skipped and others visited twice).  mode 0 is the bijection
 * the product implements: multiplier c = the smallest c >= C with
 * gcd(c, N) = 1, exact product, t in [0, N).  Both return the match with the
 * smallest t (the reference returns whichever thread wins its atomicCAS).
 * ------------------------------------------------------------------------- */
static uint64_t orc_mulmod(uint64_t a, uint64_t b, uint64_t n) {
  return (uint64_t)(((unsigned __int128)a * b) % n);
}

static uint64_t orc_gcd(uint64_t a, uint64_t b) {
  while (b) {
    uint64_t t = a % b;
    a = b;
    b = t;
  }
  return a;
}

uint64_t orc_rtid_multiplier(uint64_t n) {
  uint64_t c = 2246822507ULL;
  while (n > 1 && orc_gcd(c % n, n) != 1) ++c;
  return c;
}

static uint64_t rtid_map(uint64_t t, uint64_t n, uint64_t c, int mode) {
  if (mode == 1) return (t * 2246822507ULL) % n; /* wraps mod 2^64 like the reference */
  return orc_mulmod(t, c, n);
}

int orc_search_rtid(int bits, int k, int S, const uint64_t *in, const uint64_t *out, int max_size,
                    int include_edges, int mode, int nth, orc_result *res) {
  memset(res, 0, sizeof(*res));
  if (max_size > ORC_MAX_SIZE || k > ORC_MAX_TERMS || k < 1 || S < 1 || mode < 0 || mode > 1)
    return -2;
  uint64_t t[(ORC_MAX_SIZE + 1) * 9];
  if (orc_count_table(max_size, k, t) != 0) return -3;
  if (nth <= 0) nth = orc_max_threads();
  const uint64_t m = wmask(bits);
  if (include_edges) {
    for (int v = 0; v < k; ++v) {
      res->candidates++;
      res->per_size[1]++;
      int ok = 1;
      for (int i = 0; i < S && ok; ++i) ok = (in[(size_t)i * k + v] & m) == (out[i] & m);
      if (ok) {
        res->found = 1;
        res->size = 1;
        res->op = 8;
        res->rank = (uint64_t)v;
        res->postfix[0] = (char)('0' + v);
        return 1;
      }
    }
  }
  const int last = include_edges ? max_size : max_size - 1;
  for (int s = 2; s <= last; ++s) {
    uint64_t off = 0;
    for (int op = 0; op < 8; ++op) {
      const uint64_t N = t[s * 9 + op];
      res->candidates += N;
      res->per_size[s] += N;
      if (!N) continue;
      const uint64_t c = orc_rtid_multiplier(N);
      const uint64_t T = mode == 1 ? (N + 1023) / 1024 * 1024 : N;
      const int64_t nchunks = (int64_t)((T + ORC_CHUNK - 1) / ORC_CHUNK);
      uint64_t best = ~0ULL;
#ifdef _OPENMP
#pragma omp parallel for schedule(dynamic, 4) num_threads(nth)
#endif
      for (int64_t ch = 0; ch < nchunks; ++ch) {
        const uint64_t a = (uint64_t)ch * ORC_CHUNK;
        const uint64_t b = a + ORC_CHUNK < T ? a + ORC_CHUNK : T;
        if (a > __atomic_load_n(&best, __ATOMIC_RELAXED)) continue;
        char p[ORC_MAX_SIZE + 1];
        for (uint64_t x = a; x < b; ++x) {
          orc_unrank(off + rtid_map(x, N, c, mode), s, t, p);
          if (orc_check(p, s, bits, k, S, in, out)) {
            atomic_min_u64(&best, x);
            break;
          }
        }
      }
      if (best != ~0ULL) {
        res->found = 1;
        res->size = s;
        res->op = op;
        res->rank = off + rtid_map(best, N, c, mode);
        orc_unrank(res->rank, s, t, res->postfix);
        res->postfix[s] = 0;
        return 1;
      }
      off += N;
    }
  }
  return 0;
}

/* ---------------------------------------------------------------------------
 * VFB: bottom-up enumeration with observational-equivalence dedup.
 * vfb/src/full-cache.cu:665-774 (driver), :568-663 (per-operator loops),
 * :333-372 (candidate order, Minus also tries the swapped pair), :460-472
 * (operator order ~ & | ^ neg + - *).
 * ------------------------------------------------------------------------- */

/* Fingerprint of a uint32 characteristic vector, full-cache.cu:113-134. */
static uint32_t simple_hash(uint32_t x) {
  x ^= x >> 16;
  x *= 0x85ebca6bU;
  x ^= x >> 13;
  x *= 0xc2b2ae35U;
  x ^= x >> 16;
  return x;
}

uint64_t orc_vfb_fingerprint32(const uint32_t *cs, int n) {
  uint64_t seed = 0;
  for (int i = 0; i < n; ++i) {
    uint64_t val = (uint64_t)simple_hash(cs[i]) + 0x9e3779b9ULL + (seed << 6) + (seed >> 2);
    val = (i & 1) ? (val >> 32 | val << 32) : val;
    seed ^= val;
  }
  return seed;
}

typedef struct {
  uint64_t *vecs; /* pool of vectors, S words each */
  int64_t n, cap;
  int64_t *slots; /* open addressing over pool indices, -1 = empty */
  uint64_t nslots;
  int S;
} vecset;

static uint64_t vhash(const uint64_t *v, int S) {
  uint64_t h = 0x243F6A8885A308D3ULL;
  for (int i = 0; i < S; ++i) {
    h ^= v[i] + 0x9E3779B97F4A7C15ULL + (h << 6) + (h >> 2);
    h *= 0xff51afd7ed558ccdULL;
    h ^= h >> 33;
  }
  return h;
}

static int vs_init(vecset *s, int S) {
  s->S = S;
  s->n = 0;
  s->cap = 1024;
  s->vecs = (uint64_t *)malloc(sizeof(uint64_t) * S * s->cap);
  s->nslots = 4096;
  s->slots = (int64_t *)malloc(sizeof(int64_t) * s->nslots);
  if (!s->vecs || !s->slots) return -1;
  for (uint64_t i = 0; i < s->nslots; ++i) s->slots[i] = -1;
  return 0;
}

static void vs_free(vecset *s) {
  free(s->vecs);
  free(s->slots);
}

static int vs_grow(vecset *s) {
  uint64_t ns = s->nslots * 2;
  int64_t *sl = (int64_t *)malloc(sizeof(int64_t) * ns);
  if (!sl) return -1;
  for (uint64_t i = 0; i < ns; ++i) sl[i] = -1;
  for (int64_t i = 0; i < s->n; ++i) {
    uint64_t h = vhash(s->vecs + i * s->S, s->S) & (ns - 1);
    while (sl[h] >= 0) h = (h + 1) & (ns - 1);
    sl[h] = i;
  }
  free(s->slots);
  s->slots = sl;
  s->nslots = ns;
  return 0;
}

/* Returns 1 if v was new (and inserts it), 0 if already present, -1 on OOM. */
static int vs_insert(vecset *s, const uint64_t *v) {
  if ((uint64_t)(s->n + 1) * 2 > s->nslots && vs_grow(s)) return -1;
  uint64_t h = vhash(v, s->S) & (s->nslots - 1);
  while (s->slots[h] >= 0) {
    if (!memcmp(s->vecs + s->slots[h] * s->S, v, sizeof(uint64_t) * s->S)) return 0;
    h = (h + 1) & (s->nslots - 1);
  }
  if (s->n == s->cap) {
    uint64_t *nv = (uint64_t *)realloc(s->vecs, sizeof(uint64_t) * s->S * s->cap * 2);
    if (!nv) return -1;
    s->vecs = nv;
    s->cap *= 2;
  }
  memcpy(s->vecs + s->n * s->S, v, sizeof(uint64_t) * s->S);
  s->slots[h] = s->n++;
  return 1;
}

typedef struct {
  uint64_t *vec; /* rows x S */
  int8_t *op;
  int64_t *l, *r;
  int64_t n, cap;
  int S;
} rowstore;

static int rs_push(rowstore *rs, const uint64_t *v, int op, int64_t l, int64_t r) {
  if (rs->n == rs->cap) {
    int64_t nc = rs->cap ? rs->cap * 2 : 1024;
    uint64_t *nv = (uint64_t *)realloc(rs->vec, sizeof(uint64_t) * rs->S * nc);
    int8_t *no = (int8_t *)realloc(rs->op, nc);
    int64_t *nl = (int64_t *)realloc(rs->l, sizeof(int64_t) * nc);
    int64_t *nr = (int64_t *)realloc(rs->r, sizeof(int64_t) * nc);
    if (!nv || !no || !nl || !nr) return -1;
    rs->vec = nv;
    rs->op = no;
    rs->l = nl;
    rs->r = nr;
    rs->cap = nc;
  }
  memcpy(rs->vec + rs->n * rs->S, v, sizeof(uint64_t) * rs->S);
  rs->op[rs->n] = (int8_t)op;
  rs->l[rs->n] = l;
  rs->r[rs->n] = r;
  rs->n++;
  return 0;
}

static int row_postfix(const rowstore *rs, int64_t row, char *out, int pos, int maxlen) {
  if (pos >= maxlen - 1) return -1;
  int op = rs->op[row];
  if (op < 0) {
    out[pos] = (char)('0' + (int)rs->l[row]);
    return pos + 1;
  }
  pos = row_postfix(rs, rs->l[row], out, pos, maxlen);
  if (pos < 0) return -1;
  if (op != ORC_NOT && op != ORC_NEG) {
    pos = row_postfix(rs, rs->r[row], out, pos, maxlen);
    if (pos < 0) return -1;
  }
  if (pos >= maxlen - 1) return -1;
  out[pos] = OP_CHARS[op];
  return pos + 1;
}

/* Candidate handling: insertInCache + processUniqueCS (full-cache.cu:277-321).
 * ref_inverted = 1 reproduces the reference's test as written: warpcore's
 * HashSet::insert returns a positive value for a key that is already present
 * (vfb/include/warpcore/hash_set.cuh:210-214,230-233) and a negative one for
 * a fresh insert (:235-238), and `insert(...) > 0` is taken as "unique", so
 * the reference stores the 2nd, 3rd, ... occurrence of a vector.  With 0,
 * the first occurrence is stored and later ones dropped (the documented
 * intent).  Vectors are compared in full, not by fingerprint. */
typedef struct {
  vecset seen;
  rowstore rows;
  const uint64_t *target;
  int S, inverted;
  int64_t cap_rows;
  int64_t found_row;
  int full;
} vfb_state;

static int vfb_offer(vfb_state *st, const uint64_t *v, int op, int64_t l, int64_t r) {
  int fresh = vs_insert(&st->seen, v);
  if (fresh < 0) return -1;
  int keep = st->inverted ? !fresh : fresh;
  if (!keep) return 0;
  if (st->rows.n >= st->cap_rows) {
    st->full = 1;
    return 0;
  }
  if (rs_push(&st->rows, v, op, l, r)) return -1;
  if (st->found_row < 0 && !memcmp(v, st->target, sizeof(uint64_t) * st->S))
    st->found_row = st->rows.n - 1;
  return 0;
}

int orc_vfb(int bits, int k, int S, const uint64_t *in, const uint64_t *out, int max_len,
            int64_t cap_rows, int inverted, orc_vfb_result *res) {
  memset(res, 0, sizeof(*res));
  if (max_len < 1 || max_len > 100 || S < 1 || k < 1) return -2;
  const uint64_t m = wmask(bits);
  vfb_state st;
  memset(&st, 0, sizeof(st));
  st.S = S;
  st.inverted = inverted;
  st.cap_rows = cap_rows > 0 ? cap_rows : ((int64_t)1 << 40);
  st.found_row = -1;
  st.rows.S = S;
  uint64_t *tgt = (uint64_t *)malloc(sizeof(uint64_t) * S);
  uint64_t *v = (uint64_t *)malloc(sizeof(uint64_t) * S);
  if (!tgt || !v || vs_init(&st.seen, S)) return -1;
  for (int i = 0; i < S; ++i) tgt[i] = out[i] & m;
  st.target = tgt;
  int rc = 0;
  int64_t start[102];
  memset(start, 0, sizeof(start));
  /* size 1: the variables, checked on the host (full-cache.cu:694-707) and
   * inserted into the hash set (hashSetInit, :142-157, :748) */
  start[1] = 0;
  for (int j = 0; j < k; ++j) {
    for (int i = 0; i < S; ++i) v[i] = in[(size_t)i * k + j] & m;
    res->candidates++;
    rs_push(&st.rows, v, -1, j, -1);
    if (!memcmp(v, tgt, sizeof(uint64_t) * S)) {
      res->found = 1;
      res->size = 1;
      res->op = 8;
      res->postfix[0] = (char)('0' + j);
      goto done;
    }
  }
  for (int j = 0; j < k; ++j)
    if (vs_insert(&st.seen, st.rows.vec + (size_t)j * S) < 0) {
      rc = -1;
      goto done;
    }
  res->rows_per_size[1] = k;
  start[2] = st.rows.n;
  for (int L = 2; L <= max_len; ++L) {
    for (int op = 0; op < 8 && st.found_row < 0 && !st.full; ++op) {
      if (op == ORC_NOT || op == ORC_NEG) {
        for (int64_t x = start[L - 1]; x < start[L]; ++x) {
          const uint64_t *a = st.rows.vec + x * S;
          for (int i = 0; i < S; ++i) v[i] = apply_op(OP_CHARS[op], 0, a[i], m);
          res->candidates++;
          if (vfb_offer(&st, v, op, x, 0)) {
            rc = -1;
            goto done;
          }
          a = NULL;
        }
      } else {
        for (int i = 1; 2 * i <= L - 1; ++i) {
          int j = L - 1 - i;
          for (int64_t x = start[i]; x < start[i + 1]; ++x) {
            for (int64_t y = start[j]; y < start[j + 1]; ++y) {
              const uint64_t *a = st.rows.vec + x * S;
              const uint64_t *b = st.rows.vec + y * S;
              for (int q = 0; q < S; ++q) v[q] = apply_op(OP_CHARS[op], a[q], b[q], m);
              res->candidates++;
              if (vfb_offer(&st, v, op, x, y)) {
                rc = -1;
                goto done;
              }
              if (op == ORC_SUB) {
                a = st.rows.vec + x * S;
                b = st.rows.vec + y * S;
                for (int q = 0; q < S; ++q) v[q] = apply_op('-', b[q], a[q], m);
                res->candidates++;
                if (vfb_offer(&st, v, op, y, x)) {
                  rc = -1;
                  goto done;
                }
              }
            }
          }
        }
      }
      if (st.found_row >= 0) {
        res->found = 1;
        res->size = L;
        res->op = op;
        if (row_postfix(&st.rows, st.found_row, res->postfix, 0, 256) < 0)
          res->postfix[0] = 0;
        break;
      }
    }
    start[L + 1] = st.rows.n;
    res->rows_per_size[L] = st.rows.n - start[L];
    if (st.found_row >= 0) break;
    if (st.full) {
      res->cache_full = 1;
      break;
    }
  }
done:
  res->rows_total = st.rows.n;
  vs_free(&st.seen);
  free(st.rows.vec);
  free(st.rows.op);
  free(st.rows.l);
  free(st.rows.r);
  free(tgt);
  free(v);
  return rc < 0 ? rc : res->found;
}

/* ---------------------------------------------------------------------------
 * Extended grammar: the operator set of the reference's Op enum with the
 * shifts, division and modulo that its builds leave switched off
 * (vfb/src/full-cache.cu:166-179 declares Not And Or Xor LShift RShift Neg
 * Plus Minus Mul Div Mod; :460-472 comments LShift, RShift, Div and Mod out
 * of the enumeration; simba/src/mba.cuh:71-131 evaluates '<' '>' '/' '%' in
 * evaluateRPN, which nothing calls).  Operator order, as declared:
 *   ~ & | ^ << >> neg + - * / %     (postfix chars ~ & | ^ < > # + - * / %)
 * Rank space: the SIMBA count recurrence with the four new binary operators
 * counted like '-' (every left size; none is commutative).
 * Semantics on w-bit words: x << y and x >> y (logical) are 0 when y >= w,
 * as the GPU's clamped shifts give for the reference's `L[i] << R[i]`
 * (full-cache.cu:215-220).  Division and modulo follow VFB's zero-divisor
 * rule (full-cache.cu:230-256): in VFB, where whole vectors are composed, a
 * divisor vector with any zero element makes the result the dividend vector;
 * the SIMBA rank-space search evaluates one sample at a time and applies the
 * same fallback per sample (x / 0 = x % 0 = x).
 * Operator codes in results: the base codes 0..7, 9 '<<', 10 '>>', 11 '/',
 * 12 '%' (8 stays "a variable").
 * ------------------------------------------------------------------------- */

#define EXT_OPS 12
#define EXT_COLS 13
static const char EXT_CHARS[EXT_OPS] = {'~', '&', '|', '^', '<', '>', '#', '+', '-', '*', '/', '%'};
static const int EXT_CODE[EXT_OPS] = {0, 1, 2, 3, 9, 10, 4, 5, 6, 7, 11, 12};

static int ext_unary(int e) { return e == 0 || e == 6; }
static int ext_comm(int e) { return e == 1 || e == 2 || e == 3 || e == 7 || e == 9; }

static char code_char(int code) {
  switch (code) {
    case 9: return '<';
    case 10: return '>';
    case 11: return '/';
    case 12: return '%';
  }
  return OP_CHARS[code];
}

int orc_ext_count_table(int max_size, int n_terms, uint64_t *t) {
  int overflow = 0;
  memset(t, 0, sizeof(uint64_t) * EXT_COLS * (size_t)(max_size + 1));
  if (max_size >= 1) t[1 * EXT_COLS + EXT_OPS] = (uint64_t)n_terms;
  if (max_size >= 2) {
    t[2 * EXT_COLS + 0] = (uint64_t)n_terms;
    t[2 * EXT_COLS + 6] = (uint64_t)n_terms;
    t[2 * EXT_COLS + EXT_OPS] = 2 * (uint64_t)n_terms;
  }
  for (int i = 3; i <= max_size; ++i) {
    unsigned __int128 u = t[(i - 1) * EXT_COLS + EXT_OPS], c = 0, n = 0, tot = 0;
    for (int j = 1; j <= (i - 1) / 2; ++j)
      c += (unsigned __int128)t[j * EXT_COLS + EXT_OPS] * t[(i - j - 1) * EXT_COLS + EXT_OPS];
    for (int j = 1; j <= i - 2; ++j)
      n += (unsigned __int128)t[j * EXT_COLS + EXT_OPS] * t[(i - j - 1) * EXT_COLS + EXT_OPS];
    for (int e = 0; e < EXT_OPS; ++e) {
      const unsigned __int128 v = ext_unary(e) ? u : (ext_comm(e) ? c : n);
      if (v >> 64) overflow = 1;
      t[i * EXT_COLS + e] = (uint64_t)v;
      tot += v;
    }
    if (tot >> 64) overflow = 1;
    t[i * EXT_COLS + EXT_OPS] = (uint64_t)tot;
  }
  return overflow ? -1 : 0;
}

static void ext_unrank_rec(uint64_t n, int size, const uint64_t *t, char *out) {
  if (size == 1) {
    out[0] = (char)('0' + (int)n);
    return;
  }
  uint64_t part = 0;
  int e = 0;
  while (n >= part + t[size * EXT_COLS + e]) part += t[size * EXT_COLS + e++];
  n -= part;
  const int sub = size - 1;
  out[sub] = EXT_CHARS[e];
  if (ext_unary(e)) {
    ext_unrank_rec(n, sub, t, out);
    return;
  }
  uint64_t fpart = 0;
  int f = 1;
  while (n >= fpart + t[f * EXT_COLS + EXT_OPS] * t[(sub - f) * EXT_COLS + EXT_OPS]) {
    fpart += t[f * EXT_COLS + EXT_OPS] * t[(sub - f) * EXT_COLS + EXT_OPS];
    f++;
  }
  n -= fpart;
  const uint64_t r = t[(sub - f) * EXT_COLS + EXT_OPS];
  ext_unrank_rec(n / r, f, t, out);
  ext_unrank_rec(n % r, sub - f, t, out + f);
}

void orc_ext_unrank(uint64_t rank, int size, const uint64_t *t, char *postfix) {
  ext_unrank_rec(rank, size, t, postfix);
}

/* One operator on one sample (the per-sample form of the rules above). */
static inline uint64_t ext_apply(char c, uint64_t l, uint64_t r, int bits) {
  const uint64_t m = wmask(bits);
  switch (c) {
    case '<': return r >= (uint64_t)bits ? 0 : (l << r) & m;
    case '>': return r >= (uint64_t)bits ? 0 : l >> r;
    case '/': return r == 0 ? l : l / r;
    case '%': return r == 0 ? l : l % r;
  }
  return apply_op(c, l, r, m);
}

uint64_t orc_ext_eval1(const char *p, int len, int bits, const uint64_t *row) {
  uint64_t st[ORC_MAX_SIZE + 8];
  int sp = -1;
  const uint64_t m = wmask(bits);
  for (int j = 0; j < len; ++j) {
    const char c = p[j];
    if (c == '~' || c == '#') {
      st[sp] = ext_apply(c, 0, st[sp], bits);
    } else if (c >= '0' && c <= '9') {  /* at most 10 terminals: '<' and '>' follow '9' */
      st[++sp] = row[c - '0'] & m;
    } else {
      const uint64_t r = st[sp--];
      st[sp] = ext_apply(c, st[sp], r, bits);
    }
  }
  return st[0];
}

int orc_ext_check(const char *p, int len, int bits, int k, int S, const uint64_t *in,
                  const uint64_t *out) {
  const uint64_t m = wmask(bits);
  for (int i = 0; i < S; ++i)
    if (orc_ext_eval1(p, len, bits, in + (size_t)i * k) != (out[i] & m)) return 0;
  return 1;
}

/* The plain search in the extended grammar: sizes 2 .. max_size-1 (1 and
 * max_size too with include_edges), the twelve operator blocks of a size in
 * order, stop after the first block with a match, minimum matching rank of
 * that block (the rules of orc_search).  res->op is the operator's code. */
int orc_ext_search(int bits, int k, int S, const uint64_t *in, const uint64_t *out, int max_size,
                   int include_edges, int nth, orc_result *res) {
  memset(res, 0, sizeof(*res));
  if (max_size > ORC_MAX_SIZE || k > 10 || k < 1 || S < 1) return -2;
  uint64_t t[(ORC_MAX_SIZE + 1) * EXT_COLS];
  if (orc_ext_count_table(max_size, k, t) != 0) return -3;
  if (nth <= 0) nth = orc_max_threads();
  const uint64_t m = wmask(bits);
  if (include_edges) {
    for (int v = 0; v < k; ++v) {
      res->candidates++;
      res->per_size[1]++;
      int ok = 1;
      for (int i = 0; i < S && ok; ++i) ok = (in[(size_t)i * k + v] & m) == (out[i] & m);
      if (ok) {
        res->found = 1;
        res->size = 1;
        res->op = 8;
        res->rank = (uint64_t)v;
        res->postfix[0] = (char)('0' + v);
        return 1;
      }
    }
  }
  const int last = include_edges ? max_size : max_size - 1;
  for (int s = 2; s <= last; ++s) {
    uint64_t off = 0;
    for (int e = 0; e < EXT_OPS; ++e) {
      const uint64_t N = t[s * EXT_COLS + e];
      res->candidates += N;
      res->per_size[s] += N;
      uint64_t best = ~0ULL;
      if (N) {
        const int64_t nchunks = (int64_t)((N + ORC_CHUNK - 1) / ORC_CHUNK);
#ifdef _OPENMP
#pragma omp parallel for schedule(dynamic, 4) num_threads(nth)
#endif
        for (int64_t c = 0; c < nchunks; ++c) {
          const uint64_t a = off + (uint64_t)c * ORC_CHUNK;
          const uint64_t b = a + ORC_CHUNK < off + N ? a + ORC_CHUNK : off + N;
          if (a > __atomic_load_n(&best, __ATOMIC_RELAXED)) continue;
          char p[ORC_MAX_SIZE + 1];
          for (uint64_t r = a; r < b; ++r) {
            orc_ext_unrank(r, s, t, p);
            if (orc_ext_check(p, s, bits, k, S, in, out)) {
              atomic_min_u64(&best, r);
              break;
            }
          }
        }
      }
      if (best != ~0ULL) {
        res->found = 1;
        res->size = s;
        res->op = EXT_CODE[e];
        res->rank = best;
        orc_ext_unrank(best, s, t, res->postfix);
        res->postfix[s] = 0;
        return 1;
      }
      off += N;
    }
  }
  return 0;
}

/* Whole-vector composition in the extended grammar (full-cache.cu:182-262):
 * '/' and '%' copy the dividend vector when any divisor element is zero. */
static void ext_compose(char c, const uint64_t *a, const uint64_t *b, uint64_t *v, int S, int bits) {
  if (c == '/' || c == '%') {
    int zero = 0;
    for (int i = 0; i < S && !zero; ++i) zero = b[i] == 0;
    if (zero) {
      memcpy(v, a, sizeof(uint64_t) * S);
      return;
    }
  }
  for (int i = 0; i < S; ++i) v[i] = ext_apply(c, a[i], b[i], bits);
}

static int ext_row_postfix(const rowstore *rs, int64_t row, char *out, int pos, int maxlen) {
  if (pos >= maxlen - 1) return -1;
  const int op = rs->op[row];
  if (op < 0) {
    out[pos] = (char)('0' + (int)rs->l[row]);
    return pos + 1;
  }
  pos = ext_row_postfix(rs, rs->l[row], out, pos, maxlen);
  if (pos < 0) return -1;
  if (op != ORC_NOT && op != ORC_NEG) {
    pos = ext_row_postfix(rs, rs->r[row], out, pos, maxlen);
    if (pos < 0) return -1;
  }
  if (pos >= maxlen - 1) return -1;
  out[pos] = code_char(op);
  return pos + 1;
}

/* VFB in the extended grammar: the driver of orc_vfb with the twelve
 * operators in declaration order (the reference's generateMBAs, full-cache.cu:
 * 568-663, with LShift, RShift, Div and Mod enabled; every non-commutative
 * operator -- '-', '<<', '>>', '/', '%' -- also composes the swapped pair,
 * :573-575), exact dedup (the documented intent; no as-written mode). */
int orc_ext_vfb(int bits, int k, int S, const uint64_t *in, const uint64_t *out, int max_len,
                int64_t cap_rows, orc_vfb_result *res) {
  memset(res, 0, sizeof(*res));
  if (max_len < 1 || max_len > 100 || S < 1 || k < 1 || k > 10) return -2;
  const uint64_t m = wmask(bits);
  vfb_state st;
  memset(&st, 0, sizeof(st));
  st.S = S;
  st.cap_rows = cap_rows > 0 ? cap_rows : ((int64_t)1 << 40);
  st.found_row = -1;
  st.rows.S = S;
  uint64_t *tgt = (uint64_t *)malloc(sizeof(uint64_t) * S);
  uint64_t *v = (uint64_t *)malloc(sizeof(uint64_t) * S);
  if (!tgt || !v || vs_init(&st.seen, S)) return -1;
  for (int i = 0; i < S; ++i) tgt[i] = out[i] & m;
  st.target = tgt;
  int rc = 0;
  int64_t start[102];
  memset(start, 0, sizeof(start));
  for (int j = 0; j < k; ++j) {
    for (int i = 0; i < S; ++i) v[i] = in[(size_t)i * k + j] & m;
    res->candidates++;
    rs_push(&st.rows, v, -1, j, -1);
    if (!memcmp(v, tgt, sizeof(uint64_t) * S)) {
      res->found = 1;
      res->size = 1;
      res->op = 8;
      res->postfix[0] = (char)('0' + j);
      goto done;
    }
  }
  for (int j = 0; j < k; ++j)
    if (vs_insert(&st.seen, st.rows.vec + (size_t)j * S) < 0) {
      rc = -1;
      goto done;
    }
  res->rows_per_size[1] = k;
  start[2] = st.rows.n;
  for (int L = 2; L <= max_len; ++L) {
    for (int e = 0; e < EXT_OPS && st.found_row < 0 && !st.full; ++e) {
      const char c = EXT_CHARS[e];
      const int code = EXT_CODE[e];
      if (ext_unary(e)) {
        for (int64_t x = start[L - 1]; x < start[L]; ++x) {
          const uint64_t *a = st.rows.vec + x * S;
          for (int i = 0; i < S; ++i) v[i] = ext_apply(c, 0, a[i], bits);
          res->candidates++;
          if (vfb_offer(&st, v, code, x, 0)) {
            rc = -1;
            goto done;
          }
        }
        continue;
      }
      const int swap = !ext_comm(e);
      /* the reference stops after the chunk (here: the split) that produced
       * the target (generateMBAs, full-cache.cu:636-640) */
      for (int i = 1; 2 * i <= L - 1 && st.found_row < 0; ++i) {
        const int j = L - 1 - i;
        for (int64_t x = start[i]; x < start[i + 1]; ++x) {
          for (int64_t y = start[j]; y < start[j + 1]; ++y) {
            /* rows may move when the store grows: index them afresh */
            ext_compose(c, st.rows.vec + x * S, st.rows.vec + y * S, v, S, bits);
            res->candidates++;
            if (vfb_offer(&st, v, code, x, y)) {
              rc = -1;
              goto done;
            }
            if (swap) {
              ext_compose(c, st.rows.vec + y * S, st.rows.vec + x * S, v, S, bits);
              res->candidates++;
              if (vfb_offer(&st, v, code, y, x)) {
                rc = -1;
                goto done;
              }
            }
          }
        }
      }
      if (st.found_row >= 0) {
        res->found = 1;
        res->size = L;
        res->op = code;
        if (ext_row_postfix(&st.rows, st.found_row, res->postfix, 0, 256) < 0)
          res->postfix[0] = 0;
        break;
      }
    }
    if (st.found_row >= 0 && !res->found) { /* found by a unary block */
      res->found = 1;
      res->size = L;
      res->op = st.rows.op[st.found_row];
      if (ext_row_postfix(&st.rows, st.found_row, res->postfix, 0, 256) < 0)
        res->postfix[0] = 0;
    }
    start[L + 1] = st.rows.n;
    res->rows_per_size[L] = st.rows.n - start[L];
    if (st.found_row >= 0) break;
    if (st.full) {
      res->cache_full = 1;
      break;
    }
  }
done:
  res->rows_total = st.rows.n;
  vs_free(&st.seen);
  free(st.rows.vec);
  free(st.rows.op);
  free(st.rows.l);
  free(st.rows.r);
  free(tgt);
  free(v);
  return rc < 0 ? rc : res->found;
}
