/*
 * simba_b200 -- C ABI of the B200-native SIMBA / VFB search library
 * (libsimba_b200.so).  Plain C types only; every buffer is owned by the
 * caller; no call throws or aborts across this boundary.
 *
 * The reference exposes no library API: its only interface is the two
 * executables `simba <instance.json> <maxLen>` (simba/src/nocache.cu:291-342)
 * and `vfb <instance.json> <maxLen>` (vfb/src/full-cache.cu:776-854).  Each
 * entry point below names the reference code it replaces.
 */
#ifndef SIMBA_B200_H
#define SIMBA_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SIMBA_ABI_VERSION 2

/* Status codes (return value of the solve calls and result.status). */
#define SIMBA_OK 0           /* an expression was found                      */
#define SIMBA_NOT_FOUND 1    /* every size searched, no match: "Not found !" */
#define SIMBA_BUDGET 2       /* time budget exhausted before a match         */
#define SIMBA_CACHE_FULL 3   /* VFB cache capacity reached: "Not found !"    */
#define SIMBA_E_ARG (-1)     /* bad argument or limit exceeded               */
#define SIMBA_E_CUDA (-2)    /* CUDA runtime error                           */
#define SIMBA_E_NOMEM (-3)   /* device or host allocation failed             */
#define SIMBA_E_NODEV (-4)   /* no usable CUDA device                        */
#define SIMBA_E_OVERFLOW (-5)/* a candidate count exceeds 64 bits            */
#define SIMBA_E_INTERNAL (-6)/* internal consistency check failed            */
#define SIMBA_E_IO (-7)      /* instance file unreadable or malformed        */

/* One MBA learning instance.  Mirrors MbaInstance (simba/src/instance.h:10-30):
 * inputs are sample-major, inputs[i * num_variables + j] = variable j on
 * sample i.  A constant terminal 1 is an extra variable equal to 1 on every
 * sample.  word_bits selects the arithmetic: 32 (the reference's uint32_t,
 * simba/src/mba.cuh:8) or 64 (exact uint64, mod 2^64). */
typedef struct {
  int32_t num_variables;
  int32_t num_examples;
  int32_t word_bits;
  int32_t unit_log2;     /* batch only: work-unit size chosen by the autotuner
                            for this instance's bucket, 0 = opt->unit_log2   */
  const uint64_t *inputs;
  const uint64_t *outputs;
} simba_instance;

/* Options; a zero-filled struct (or NULL) gives the reference behaviour. */
typedef struct {
  int32_t device;        /* CUDA device ordinal                                  */
  int32_t size_range;    /* 0: sizes 2..max-1 like the reference (nocache.cu:246);
                            1: sizes 1..max                                       */
  int32_t verbose;       /* progress lines on stderr                             */
  int32_t engine;        /* 0: tabled spine engine; 1: one thread per rank       */
  double budget_seconds; /* 0 = unlimited                                        */
  int64_t table_bytes;   /* cap on the value tables, 0 = default (8 GiB); the
                            tables are kept for sample 0 and, as match
                            filters, for samples 1..3 (instances with fewer
                            samples keep fewer), all inside this cap         */
  uint64_t stream;       /* cudaStream_t to launch on (0 = library-owned stream)  */
  int64_t vfb_cache_rows;/* VFB row capacity, 0 = the reference's rule
                            (max pitch / (4 * samples), full-cache.cu:713-718)  */
  int32_t vfb_reference_dedup; /* 1: VFB keeps the reference's uniqueness test
                            as written (stores repeated vectors)                */
  int32_t unit_log2;     /* log2 of candidates per work unit, 0 = 22 (autotuned
                            per bucket by the Python autotuner)                  */
  const float *class_prior; /* guided search: 64 shape-class priors (see
                            simba_shape_class).  Sizes are still searched in
                            order and every candidate of the sizes below the
                            answer is evaluated; inside a size the spines run
                            in decreasing prior and the search stops at the
                            first verified match, which has the minimal size
                            but need not have the minimum rank.  NULL = plain */
  int32_t rank_order;    /* simba_solve only.  0: the minimum matching rank of
                            the first operator block with a match; 1: RTid
                            order (the reference's simba_rtid build,
                            nocache_rtid.cu:85-95): the block's ranks are
                            visited as (t * c) mod N, t = 0, 1, ..., and the
                            match with the smallest t is returned; c is the
                            smallest integer >= 2246822507 coprime to N, so
                            every rank is visited exactly once            */
  int32_t grammar;       /* simba_solve and vfb_solve only.  0: the reference's
                            operators ~ & | ^ neg + - *.  1: the extended set
                            the reference declares but leaves switched off
                            (vfb/src/full-cache.cu:166-179,460-472):
                            ~ & | ^ << >> neg + - * / % in that order, postfix
                            characters < > / %, result op codes 9..12 for
                            << >> / %; shifts by >= the word width give 0;
                            VFB takes the dividend vector when any divisor
                            element is 0 (full-cache.cu:230-256), the plain
                            search the dividend per sample (x/0 = x%0 = x);
                            at most 10 terminals.  The plain search runs one
                            thread per rank in this grammar.               */
  int32_t lanes_log2;    /* spine kernel layout: each group of contexts keeps at
                            least 2^lanes_log2 of a CTA's 256 threads on its
                            bottom values (0 = as many context groups as there
                            are contexts); tuned by the Python autotuner      */
  int32_t filter_samples;/* match filters: samples 1..filter_samples get value
                            tables (1..3; 0 = 3)                               */
} simba_options;

typedef struct {
  int32_t status;
  int32_t size;          /* size of the expression found                         */
  int32_t op;            /* root-operator block 0..7 (~ & | ^ neg + - *), 8 = leaf */
  int32_t table_size;    /* largest tabled size used by the engine               */
  uint64_t rank;         /* minimum matching rank of that size                   */
  char postfix[64];      /* reference encoding: '0'+var and ~ & | ^ # + - *      */
  char expr[512];        /* SIMBA syntax, e.g. (v0 + (~v1))  (nocache.cu:162-195) */
  double seconds;        /* wall time of the call                                */
  double device_ms;      /* GPU time of the search kernels                       */
  uint64_t candidates;   /* candidates in the blocks searched (reference rule)   */
  uint64_t evaluated;    /* candidates the kernels evaluated                     */
  uint64_t per_size[33]; /* candidates per size (reference rule)                 */
  int32_t max_size_searched;
  int32_t launches;      /* kernels launched by the call                         */
  double kernel_ms;      /* GPU time of the search kernel launches alone         */
  uint64_t alg_ops;      /* integer lane-operations the algorithm needs for the
                            candidates evaluated (see simba_int_peak)            */
  /* The spine kernel runs up to two launches per size: the hash-join units
   * (spines without & and |) and the nested-compare units.  Their GPU time
   * and candidates, summed over the sizes searched: */
  double join_ms;
  double nested_ms;
  uint64_t join_candidates;
  uint64_t nested_candidates;
  double join_bytes_streamed; /* bottom-table bytes the join units read: each
                            table once per block of contexts                    */
  double join_table_bytes;    /* the bottom tables the join launches read, each
                            counted once per size: the algorithmic minimum     */
  uint64_t nested_live_candidates; /* nested-compare candidates whose context can
                            match sample 0 and were compared one by one; the
                            rest were decided by their context's constraint   */
} simba_result;

/* Plain cache-free unranking search of one instance: replaces NoCache::solve
 * (simba/src/nocache.cu:197-289).  Searches sizes in increasing order and
 * operator blocks in the reference order, stops after the first block that
 * holds a match and returns the minimum matching rank of that block.
 * Returns result.status. */
int simba_solve(const simba_instance *inst, int max_size, const simba_options *opt,
                simba_result *result);

/* VFB bottom-up search result. */
typedef struct {
  int32_t status;
  int32_t size;
  int32_t op;            /* operator block of the answer, 8 = a variable         */
  int32_t max_size_searched;
  char postfix[256];
  char expr[2048];       /* VFB syntax, e.g. (v0)+(~(v1)) (full-cache.cu:483-509) */
  double seconds;
  double device_ms;
  uint64_t candidates;   /* allMBAs as the reference counts it                   */
  int64_t rows_total;    /* cached characteristic vectors                        */
  int64_t rows_per_size[101];
  uint64_t cache_bytes;  /* bytes of the row cache                               */
  uint64_t table_bytes;  /* bytes of the dedup hash table                        */
  double bytes_moved;    /* algorithmic HBM bytes of the composition kernels     */
  int32_t launches;
  int32_t reserved;
} vfb_result;

/* VFB bottom-up enumeration with observational-equivalence dedup: replaces
 * MBA() / generateMBAs (vfb/src/full-cache.cu:568-774).  Sizes 1..max_len,
 * operators ~ & | ^ neg + - *, stop after the operator block that produces
 * the target; "Not found !" when max_len is reached or the cache fills. */
int vfb_solve(const simba_instance *inst, int max_len, const simba_options *opt,
              vfb_result *result);

/* simba_solve without any device allocation, for callers that cannot call
 * cudaMalloc while they run: a plugin inside a host application that owns
 * the GPU memory budget (its own pool allocator must not be bypassed), or
 * work issued while another stream of the process is being captured into a
 * CUDA graph, where an allocation would invalidate that capture.  No
 * counterpart in the reference.  All scratch lives in one 64 MiB __device__
 * array that every GPU loading the library holds until exit; sizes whose
 * value tables or spine list do not fit it are rejected with SIMBA_E_ARG.
 * The first call on a device looks up that array's address, so make it
 * before any stream capture starts; the address is cached per device
 * ordinal and is not valid after cudaDeviceReset.  Calls share the array:
 * calls that overlap on the GPU race and must be serialised.  Runs on
 * opt->stream; while another stream is being captured, pass a non-blocking
 * stream (cudaStreamNonBlocking or the per-thread default stream), since
 * work on the legacy default stream (stream 0) synchronises with blocking
 * streams, and capture that other stream in relaxed or thread-local mode.
 * Plain spine search only: opt->engine must be 0 and opt->class_prior NULL
 * (SIMBA_E_ARG otherwise); opt->table_bytes and opt->unit_log2 are ignored.
 * Creates no stream or event and reports only host-clock seconds. */
int simba_solve_noalloc(const simba_instance *inst, int max_size, const simba_options *opt,
                        simba_result *result);

/* Per-instance result of a batch. */
typedef struct {
  int32_t status;
  int32_t size;
  int32_t op;
  int32_t reserved;
  uint64_t rank;
  char postfix[64];
  double seconds;        /* time to solution on the device clock, from the batch's
                            first kernel: the first verified match (guided) or
                            the end of the instance's last unit (plain); for
                            unsolved instances the host time of retirement     */
  uint64_t candidates;   /* reference-rule candidates of this instance           */
} simba_batch_result;

typedef struct {
  double seconds;
  double device_ms;
  double kernel_ms;      /* spine / build kernels of all rounds                  */
  double alg_ops;        /* integer lane-operations of the candidates evaluated  */
  uint64_t candidates;
  uint64_t evaluated;
  int32_t rounds;        /* one persistent launch per round                      */
  int32_t launches;
  int32_t solved;
  int32_t reserved;
} simba_batch_stats;

/* Batched plain search of n independent instances of one word width (no
 * counterpart in the reference, which runs one process per instance,
 * run_all.sh:20-43).  Instances advance size by size in rounds; each round
 * is one persistent kernel whose work queue spans the instances of the
 * round, and an instance whose size produced a match retires.  Rounds are
 * cost-ordered: an instance searches its next size in a round when the
 * candidates it will then have swept are within 64x (environment
 * SIMBA_ROUND_GROWTH; 0 = every active instance) of the cheapest active
 * instance's, and the round's queue runs the cheapest instances first.
 * opt->table_bytes caps each instance's value tables, filter samples
 * included (0 = 8 MiB);
 * opt->budget_seconds bounds the whole batch.  With opt->class_prior set it
 * points to n x 64 priors (one row per instance, e.g. from
 * simba_mlp_predict) and the batch is guided: the queue holds one entry per
 * (instance, shape class), instances cheapest first and each instance's
 * classes by prior per unit of work, and an instance retires at its first
 * verified match. */
int simba_solve_batch(const simba_instance *insts, int n, int max_size, const simba_options *opt,
                      simba_batch_result *results, simba_batch_stats *stats);

/* Resident session: samples and value tables stay on the device between
 * calls (used by the benchmark to time the search with inputs in HBM). */
typedef struct simba_session simba_session;
int simba_session_create(const simba_instance *inst, const simba_options *opt,
                         simba_session **session);
int simba_session_solve(simba_session *session, int max_size, simba_result *result);
/* Evaluate every candidate of sizes lo..hi with no early stop (throughput). */
int simba_session_sweep(simba_session *session, int lo, int hi, simba_result *result);
void simba_session_destroy(simba_session *session);

/* One size of the plain search over the work units u with
 * u % nshards == shard: the building block of a search spread over several
 * GPUs, where each GPU takes one shard and the minimum of the shards'
 * best_rank decides the size (no counterpart in the reference, which uses
 * one GPU). */
typedef struct {
  int32_t status;        /* SIMBA_OK if this shard holds a match                 */
  int32_t launches;
  uint64_t best_rank;    /* minimum matching rank in this shard, ~0 if none      */
  uint64_t candidates;   /* candidates of the whole size                         */
  uint64_t evaluated;    /* candidates this shard evaluated                      */
  double device_ms;
  double kernel_ms;
} simba_size_result;
int simba_session_search_size(simba_session *session, int size, int shard, int nshards,
                              simba_size_result *result);

/* Count table numForm[size][op] (simba/src/nocache.cu:117-160), written as
 * (max_size + 1) rows of 9 columns, column 8 = total.  Host only. */
int simba_count_table(int max_size, int n_terms, uint64_t *table);
/* Rank -> postfix (simba/src/nocache.cu:23-83); writes size chars + NUL. */
int simba_unrank(uint64_t rank, int size, int n_terms, char *postfix);
/* Postfix -> rank (inverse of simba_unrank). */
int simba_rank_of(const char *postfix, int n_terms, uint64_t *rank);
/* Postfix -> infix; style 0 = SIMBA (nocache.cu:162-195), 1 = VFB
 * (vfb/src/full-cache.cu:483-509); add 2 to read '<' '>' '/' '%' as the
 * extended grammar's << >> / %.  Returns the length or a negative code. */
int simba_format(const char *postfix, int style, char *out, int cap);

/* Instance file reader: the reference JSON schema (simba/src/instance.cpp:7-27,
 * vfb/src/utils.h:15-44); "size": 64 on the values selects 64-bit words.
 * The arrays are owned by the library until simba_instance_free. */
int simba_instance_load(const char *path, simba_instance *inst);
void simba_instance_free(simba_instance *inst);

/* Measured integer-ALU issue rate of the device: independent 32-bit
 * LOP3/IADD3 chains over every SM, in lane-operations per second.  The
 * denominator of the search kernels' roofline (no counterpart in the
 * reference, which reports no roofline). */
int simba_int_peak(int device, double *lane_ops_per_s);
/* The same with LOP3 only: the rate of the ALU pipe alone, which bounds
 * kernels whose instructions are all bitwise/compare operations. */
int simba_alu_peak(int device, double *lane_ops_per_s);

/* Shape class of an expression (the guided search's unit of priority and
 * the label the proposal learns): 8 * root operator + min(left operand size,
 * 7) for a binary root, 8 * root operator + min(length of the unary chain at
 * the root, 7) for a unary root.  Returns 0..63 or a negative code. */
int simba_shape_class(const char *postfix);

/* Learned proposal: a 3-layer MLP (8192 -> 512 -> 512 -> 64) over bit-level
 * features of an instance's samples, predicting the shape class of its
 * minimal expression; BF16 tensor-core GEMMs with FP32 accumulation,
 * hand-written backward pass and Adam.  No counterpart in the reference.
 * Parameters are flattened W1[8192x512], b1[512], W2[512x512], b2[512],
 * W3[512x64], b3[64] (row-major, input x output). */
typedef struct simba_mlp simba_mlp;
int64_t simba_mlp_param_count(void);
int simba_mlp_create(int device, uint64_t seed, simba_mlp **mlp);
void simba_mlp_destroy(simba_mlp *mlp);
/* One Adam step on a minibatch; *loss = mean cross-entropy before the step. */
int simba_mlp_train_step(simba_mlp *mlp, const simba_instance *insts, int n, const int32_t *labels,
                         float lr, float *loss);
/* Gradients of the mean cross-entropy (param_count floats), no update. */
int simba_mlp_gradients(simba_mlp *mlp, const simba_instance *insts, int n, const int32_t *labels,
                        float *grads, float *loss);
/* One Adam step with the given gradients (param_count floats): data-parallel
 * training applies the ranks' all-reduced mean gradient on every rank. */
int simba_mlp_apply(simba_mlp *mlp, const float *grads, float lr);
/* Class probabilities, n x 64. */
int simba_mlp_predict(simba_mlp *mlp, const simba_instance *insts, int n, float *probs);
/* The features the network reads, n x 8192 (values -1, 0, +1). */
int simba_mlp_features(simba_mlp *mlp, const simba_instance *insts, int n, float *features);
int simba_mlp_get_params(simba_mlp *mlp, float *params);
int simba_mlp_set_params(simba_mlp *mlp, const float *params);

/* Device memory released by the calls above is kept in a process-wide cache
 * (up to SIMBA_DEVICE_CACHE_BYTES, default 32 GiB per process, 0 = off) and
 * reused by later calls, so that repeated searches do not allocate and free
 * gigabytes of value tables each time (no counterpart in the reference,
 * which allocates per run).  This returns every cached block to the device.
 * Do not call it while another thread's call is running. */
int simba_release_device_cache(void);

const char *simba_version(void);
const char *simba_status_string(int status);
const char *simba_last_error(void);
int simba_device_count(void);

#ifdef __cplusplus
}
#endif
#endif /* SIMBA_B200_H */
