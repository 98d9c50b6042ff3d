// Internal C++ interface between the C ABI (capi.cpp) and the CUDA engines
// (search_impl.cuh via search_u32.cu / search_u64.cu, search_static.cu,
// vfb.cu, mlp.cu).  Nothing here crosses the library boundary.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

#include "../../include/simba_b200.h"
#include "grammar.h"

namespace simba {

// An instance with its words already reduced to the word width.
struct HostInstance {
  int k = 0;          // terminals
  int S = 0;          // samples
  int bits = 32;      // 32 or 64
  std::vector<uint64_t> in;   // S*k sample-major
  std::vector<uint64_t> out;  // S
  int unit_log2 = 0;          // batch: autotuned work-unit size, 0 = options
};

struct EngineOptions {
  int device = 0;
  int size_range = 0;        // 0 reference (2..max-1), 1 complete (1..max)
  int verbose = 0;
  double budget_s = 0.0;     // 0 = unlimited
  int64_t table_bytes = 0;   // 0 = default cap
  int engine = 0;            // 0 spine (auto), 1 naive per-rank kernel
  int stop_on_match = 1;     // 0: evaluate whole sizes (throughput sweeps)
  uint64_t stream = 0;       // caller's cudaStream_t, 0 = own stream
  int unit_log2 = 0;         // log2 candidates per work unit, 0 = 22
  const float* class_prior = nullptr;  // guided search: 64 shape-class priors
  int rank_order = 0;        // 0 rank order, 1 RTid order (single-instance solve only)
  int grammar = 0;           // 0 the reference grammar, 1 extended (ext_grammar.h)
  int lanes_log2 = 0;        // spine kernel: at least 2^lanes_log2 value lanes per context group
  int filter_samples = 0;    // match-filter samples with value tables, 1..3 (0 = 3)
};

// Per-solve outcome filled by the engines (capi.cpp formats the strings).
struct SolveOutcome {
  int status = SIMBA_NOT_FOUND;
  int size = 0;
  int op = -1;
  uint64_t rank = 0;
  std::string postfix;
  double device_ms = 0.0;
  uint64_t candidates = 0;
  uint64_t evaluated = 0;
  uint64_t per_size[kMaxSize + 1] = {};
  int table_size = 0;
  int max_size_searched = 0;
  int launches = 0;
  double kernel_ms = 0.0;
  uint64_t alg_ops = 0;
  // the two launch kinds of the spine kernel (single-instance searches)
  double join_ms = 0.0, nested_ms = 0.0;
  uint64_t join_candidates = 0, nested_candidates = 0;
  uint64_t nested_live_candidates = 0;  // of those, candidates of contexts that can match
  double join_bytes_streamed = 0.0, join_table_bytes = 0.0;
};

std::string last_error();
void set_last_error(const std::string& e);

// Limits check shared by every entry point (the reference's own limits are
// 10 variables / 100 samples / size 32: simba/src/globals.cuh:5-7; this
// build allows kMaxTerms / kMaxSamples / kMaxSize).
int validate(const HostInstance& h, int max_size);

// Plain SIMBA search on one instance.  Session objects keep the samples and
// value tables resident between calls.
struct SizeOutcome {
  int status = SIMBA_NOT_FOUND;
  uint64_t best = ~0ULL;
  uint64_t candidates = 0;
  uint64_t evaluated = 0;
  double device_ms = 0.0;
  double kernel_ms = 0.0;
  int launches = 0;
};

class SearchSession {
 public:
  virtual ~SearchSession() = default;
  virtual int search_one_size(int size, int shard, int nshards, SizeOutcome* out) = 0;
  virtual int solve(int max_size, SolveOutcome* out) = 0;
  // Evaluate every candidate of sizes [lo, hi] with no early stop.
  virtual int sweep(int lo, int hi, SolveOutcome* out) = 0;
};

int make_search_session(const HostInstance& h, const EngineOptions& o,
                        SearchSession** out);

// Plain search in the extended grammar (ext.cu) and its host re-check.
int ext_solve(const HostInstance& h, int max_size, const EngineOptions& o, SolveOutcome* out);
bool ext_check_host(const std::string& postfix, const HostInstance& h);
// The same check with VFB's whole-vector rule for / and % (a divisor vector
// with a zero element yields the dividend vector).
bool ext_vector_check(const std::string& postfix, const HostInstance& h);

// Plain search with all scratch in a static __device__ array (search_static.cu).
int solve_static(const HostInstance& h, int max_size, const EngineOptions& o, SolveOutcome* out);

struct BatchItemOutcome {
  int status = SIMBA_NOT_FOUND;
  int size = 0, op = -1;
  uint64_t rank = 0;
  std::string postfix;
  double seconds = 0.0;
  uint64_t candidates = 0;
};

struct BatchOutcome {
  std::vector<BatchItemOutcome> items;
  double device_ms = 0.0, kernel_ms = 0.0, alg_ops = 0.0;
  int rounds = 0, launches = 0;
  uint64_t evaluated = 0, candidates = 0;
};

// Batched plain search of independent instances of one word width
// (search_impl.cuh: Batch).  inst_table_bytes caps each instance's tables.
int batch_solve(const std::vector<HostInstance>& hs, int max_size, const EngineOptions& o,
                int64_t inst_table_bytes, BatchOutcome* out);

// Learned proposal (mlp.cu).
class Mlp;
long long mlp_param_count();
int mlp_create(int device, unsigned long long seed, Mlp** out);
void mlp_destroy(Mlp* m);
int mlp_train_step(Mlp* m, const std::vector<HostInstance>& hs, const int* labels, float lr, float* loss);
int mlp_gradients(Mlp* m, const std::vector<HostInstance>& hs, const int* labels, float* grads,
                  float* loss);
int mlp_apply(Mlp* m, const float* grads, float lr);
int mlp_predict(Mlp* m, const std::vector<HostInstance>& hs, float* probs);
int mlp_features(Mlp* m, const std::vector<HostInstance>& hs, float* out);
int mlp_get_params(Mlp* m, float* h);
int mlp_set_params(Mlp* m, const float* h);

// Read an instance file in the reference JSON schema.
int read_instance_json(const std::string& path, HostInstance* h);

int measure_int_peak(int device, double* lane_ops_per_s);
int measure_alu_peak(int device, double* lane_ops_per_s);

struct VfbOutcome {
  int status = SIMBA_NOT_FOUND;
  int size = 0;
  int op = -1;
  std::string postfix;
  double device_ms = 0.0;
  uint64_t candidates = 0;
  int64_t rows_total = 0;
  int64_t rows_per_size[101] = {};
  uint64_t cache_bytes = 0;
  uint64_t table_bytes = 0;
  double bytes_moved = 0.0;
  int launches = 0;
  int max_size_searched = 0;
};

// VFB bottom-up search (vfb.cu).  inverted = 1 keeps the reference's
// uniqueness test as written; cache_rows = 0 uses the reference capacity.
int vfb_run(const HostInstance& h, int max_len, const EngineOptions& o, int inverted,
            int64_t cache_rows, VfbOutcome* out);

// Format a postfix string in the SIMBA (style 0) or VFB (style 1) syntax;
// grammar 1 reads '<' '>' '/' '%' as the extended operators.
std::string format_postfix(const std::string& postfix, int style, int grammar = 0);

// Host-side exact check of an expression on every sample.
bool host_check(const std::string& postfix, const HostInstance& h);

}  // namespace simba
