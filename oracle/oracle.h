/*
 * CPU oracle for the SIMBA / VFB search -- TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C (+OpenMP) restatement of the reference's algorithms, used by the
 * tests, by the smoke check and as the timed CPU baseline of bench.py.  The
 * product (libsimba_b200.so, the simba / vfb executables) never links or
 * calls it.
 *
 * Pinned against: the reference generator's own outputs
 * (tests/golden/ref_instances_u32.json, produced by the reference's
 * scripts/generate.py + scripts/sample.py) and the reference CUDA
 * executables rebuilt for sm_100a (tests/golden/ref_results_u32.json).
 */
#ifndef SIMBA_ORACLE_H
#define SIMBA_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ORC_MAX_SIZE 32
#define ORC_MAX_TERMS 32
#define ORC_MAX_SAMPLES 1024

/* Operator order of the rank space: simba/src/globals.cuh:13-15 */
enum { ORC_NOT = 0, ORC_AND, ORC_OR, ORC_XOR, ORC_NEG, ORC_ADD, ORC_SUB, ORC_MUL };

typedef struct {
  int found;                 /* 1 if an expression was found */
  int size;                  /* its size (number of nodes) */
  int op;                    /* root operator block it was found in */
  uint64_t rank;             /* minimum matching rank in that block's size */
  char postfix[ORC_MAX_SIZE + 1];
  uint64_t candidates;       /* sum of block counts launched (reference rule) */
  uint64_t per_size[ORC_MAX_SIZE + 1];
} orc_result;

typedef struct {
  int found;
  int size;
  int op;
  char postfix[256];
  int cache_full;
  uint64_t candidates;       /* allMBAs as counted by the reference */
  int64_t rows_per_size[101];/* rows stored at each size (PRINT_CACHE_SIZE) */
  int64_t rows_total;
} orc_vfb_result;

int orc_count_table(int max_size, int n_terms, uint64_t *table);
void orc_unrank(uint64_t rank, int size, const uint64_t *table, char *postfix);
uint64_t orc_eval1(const char *postfix, int len, int word_bits, const uint64_t *row);
int orc_check(const char *postfix, int len, int word_bits, int n_terms, int n_samples,
              const uint64_t *inputs, const uint64_t *outputs);
int orc_search(int word_bits, int n_terms, int n_samples, const uint64_t *inputs,
               const uint64_t *outputs, int max_size, int include_edges, int n_threads,
               orc_result *res);
int orc_search_rtid(int word_bits, int n_terms, int n_samples, const uint64_t *inputs,
                    const uint64_t *outputs, int max_size, int include_edges, int mode,
                    int n_threads, orc_result *res);
uint64_t orc_rtid_multiplier(uint64_t n);
int64_t orc_scan_range(int word_bits, int n_terms, int n_samples, const uint64_t *inputs,
                       const uint64_t *outputs, int size, uint64_t rank_lo, uint64_t rank_hi,
                       int n_threads, uint64_t *min_rank, uint64_t *n_hits);
int orc_vfb(int word_bits, int n_terms, int n_samples, const uint64_t *inputs,
            const uint64_t *outputs, int max_len, int64_t cap_rows, int ref_inverted,
            orc_vfb_result *res);
uint64_t orc_vfb_fingerprint32(const uint32_t *cs, int n);

/* Extended grammar (~ & | ^ << >> neg + - * / %; see oracle.c): count table
 * of (max_size + 1) rows x 13 columns (column 12 = total), unranking,
 * per-sample evaluation, the plain search and VFB.  At most 10 terminals. */
int orc_ext_count_table(int max_size, int n_terms, uint64_t *table);
void orc_ext_unrank(uint64_t rank, int size, const uint64_t *table, char *postfix);
uint64_t orc_ext_eval1(const char *postfix, int len, int word_bits, const uint64_t *row);
int orc_ext_check(const char *postfix, int len, int word_bits, int n_terms, int n_samples,
                  const uint64_t *inputs, const uint64_t *outputs);
int orc_ext_search(int word_bits, int n_terms, int n_samples, const uint64_t *inputs,
                   const uint64_t *outputs, int max_size, int include_edges, int n_threads,
                   orc_result *res);
int orc_ext_vfb(int word_bits, int n_terms, int n_samples, const uint64_t *inputs,
                const uint64_t *outputs, int max_len, int64_t cap_rows, orc_vfb_result *res);
int orc_max_threads(void);

#ifdef __cplusplus
}
#endif
#endif
