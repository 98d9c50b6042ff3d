// C ABI of libsimba_b200.so (declared in include/simba_b200.h).
#include <cuda_runtime.h>

#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <mutex>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/simba_b200.h"
#include "cuda_util.h"
#include "engine.h"
#include "grammar.h"
#include "ext_grammar.h"
#include "json_lite.h"

namespace simba {

static thread_local std::string g_last_error;

std::string last_error() { return g_last_error; }
void set_last_error(const std::string& e) { g_last_error = e; }

// ---------------------------------------------------------------- device cache

namespace {
struct DeviceCache {
  std::mutex mu;
  std::multimap<size_t, std::pair<int, void*>> blocks;  // bytes -> (device, pointer)
  size_t cached = 0;
  size_t cap = 0;
};
DeviceCache& cache() {
  // created once, never destroyed: no cudaFree runs after the CUDA runtime
  // has shut down at process exit
  static DeviceCache* c = [] {
    DeviceCache* d = new DeviceCache;
    const char* e = getenv("SIMBA_DEVICE_CACHE_BYTES");
    d->cap = e ? (size_t)strtoull(e, nullptr, 10) : (size_t)32 << 30;
    return d;
  }();
  return *c;
}
// frees the cached blocks of one device (-1: all); the caller holds the lock
void drop_cached(DeviceCache& c, int dev) {
  int cur = -1;
  cudaGetDevice(&cur);
  for (auto it = c.blocks.begin(); it != c.blocks.end();) {
    if (dev >= 0 && it->second.first != dev) {
      ++it;
      continue;
    }
    cudaSetDevice(it->second.first);
    cudaFree(it->second.second);
    c.cached -= it->first;
    it = c.blocks.erase(it);
  }
  if (cur >= 0) cudaSetDevice(cur);
}
}  // namespace

cudaError_t pool_alloc(void** p, size_t n, size_t* got) {
  DeviceCache& c = cache();
  int dev = 0;
  cudaGetDevice(&dev);
  {
    std::lock_guard<std::mutex> g(c.mu);
    // best fit on this device, at most twice the request
    for (auto it = c.blocks.lower_bound(n); it != c.blocks.end() && it->first <= 2 * n + (1 << 20);
         ++it) {
      if (it->second.first != dev) continue;
      *p = it->second.second;
      *got = it->first;
      c.cached -= it->first;
      c.blocks.erase(it);
      return cudaSuccess;
    }
  }
  cudaError_t e = cudaMalloc(p, n);
  if (e == cudaErrorMemoryAllocation) {  // give the cached blocks back and retry
    cudaGetLastError();
    {
      std::lock_guard<std::mutex> g(c.mu);
      drop_cached(c, dev);
    }
    e = cudaMalloc(p, n);
  }
  if (e == cudaSuccess) *got = n;
  return e;
}

size_t pool_cached_bytes(int dev) {
  DeviceCache& c = cache();
  std::lock_guard<std::mutex> g(c.mu);
  size_t n = 0;
  for (const auto& b : c.blocks)
    if (b.second.first == dev) n += b.first;
  return n;
}

void pool_free(void* p, size_t bytes) {
  if (!p) return;
  DeviceCache& c = cache();
  int dev = 0;
  cudaGetDevice(&dev);
  std::lock_guard<std::mutex> g(c.mu);
  if (c.cached + bytes <= c.cap) {
    c.blocks.emplace(bytes, std::make_pair(dev, p));
    c.cached += bytes;
    return;
  }
  cudaFree(p);
}

int validate(const HostInstance& h, int max_size) {
  if (h.bits != 32 && h.bits != 64) {
    set_last_error("word_bits must be 32 or 64");
    return SIMBA_E_ARG;
  }
  if (h.k < 1 || h.k > kMaxTerms) {
    set_last_error("this build supports 1.." + std::to_string(kMaxTerms) + " variables");
    return SIMBA_E_ARG;
  }
  if (h.S < 1 || h.S > kMaxSamples) {
    set_last_error("this build supports 1.." + std::to_string(kMaxSamples) + " samples");
    return SIMBA_E_ARG;
  }
  if (max_size < 1 || max_size > kMaxSize) {
    set_last_error("this build supports formulas of size at most " + std::to_string(kMaxSize));
    return SIMBA_E_ARG;
  }
  if ((int)h.in.size() != h.S * h.k || (int)h.out.size() != h.S) {
    set_last_error("instance arrays do not match num_variables / num_examples");
    return SIMBA_E_ARG;
  }
  return 0;
}

static uint64_t wmask(int bits) { return bits == 64 ? ~0ULL : 0xFFFFFFFFULL; }

static uint64_t host_op(int op, uint64_t l, uint64_t r, uint64_t m) {
  switch (op) {
    case OP_NOT: return ~r & m;
    case OP_NEG: return (0 - r) & m;
    case OP_AND: return l & r;
    case OP_OR: return l | r;
    case OP_XOR: return l ^ r;
    case OP_ADD: return (l + r) & m;
    case OP_SUB: return (l - r) & m;
    default: return (l * r) & m;
  }
}

bool host_check(const std::string& p, const HostInstance& h) {
  const uint64_t m = wmask(h.bits);
  std::vector<uint64_t> st(p.size() + 1);
  for (int i = 0; i < h.S; ++i) {
    int sp = -1;
    for (char c : p) {
      int op = char_op(c);
      if (op < 0) {
        int t = c - '0';
        if (t < 0 || t >= h.k) return false;
        st[++sp] = h.in[(size_t)i * h.k + t] & m;
      } else if (is_unary(op)) {
        if (sp < 0) return false;
        st[sp] = host_op(op, 0, st[sp], m);
      } else {
        if (sp < 1) return false;
        uint64_t r = st[sp--];
        st[sp] = host_op(op, st[sp], r, m);
      }
    }
    if (sp != 0 || st[0] != (h.out[i] & m)) return false;
  }
  return true;
}

// SIMBA style: MBAToString, simba/src/nocache.cu:162-195.
// VFB style: toString, vfb/src/full-cache.cu:483-509.
// grammar 1: '<' '>' '/' '%' are the operators << >> / % (ext_grammar.h).
std::string format_postfix(const std::string& p, int style, int grammar) {
  std::vector<std::string> st;
  for (char c : p) {
    int op = grammar == 1 ? ext_char_code(c) : char_op(c);
    if (op < 0) {
      st.push_back("v" + std::to_string(c - '0'));
    } else if (is_unary(op)) {
      if (st.empty()) return "";
      std::string a = st.back();
      st.pop_back();
      const std::string sym = op == OP_NEG ? "-" : "~";
      st.push_back(style == 0 ? "(" + sym + a + ")" : sym + "(" + a + ")");
    } else {
      if (st.size() < 2) return "";
      std::string r = st.back();
      st.pop_back();
      std::string l = st.back();
      st.pop_back();
      const std::string sym = c == '<' && op == OP_SHL ? "<<" : (c == '>' && op == OP_SHR ? ">>" : std::string(1, c));
      st.push_back(style == 0 ? "(" + l + " " + sym + " " + r + ")" : "(" + l + ")" + sym + "(" + r + ")");
    }
  }
  return st.size() == 1 ? st[0] : "";
}

static int to_host(const simba_instance* inst, HostInstance* h) {
  if (!inst || !inst->inputs || !inst->outputs) {
    set_last_error("null instance or arrays");
    return SIMBA_E_ARG;
  }
  h->k = inst->num_variables;
  h->S = inst->num_examples;
  h->bits = inst->word_bits == 0 ? 32 : inst->word_bits;
  h->unit_log2 = inst->unit_log2;
  if (h->k < 1 || h->S < 1 || h->k > kMaxTerms || h->S > kMaxSamples) {
    set_last_error("instance limits exceeded");
    return SIMBA_E_ARG;
  }
  const uint64_t m = wmask(h->bits);
  h->in.assign(inst->inputs, inst->inputs + (size_t)h->S * h->k);
  h->out.assign(inst->outputs, inst->outputs + h->S);
  for (auto& x : h->in) x &= m;
  for (auto& x : h->out) x &= m;
  return 0;
}

static EngineOptions to_opts(const simba_options* o) {
  EngineOptions e;
  if (o) {
    e.device = o->device;
    e.size_range = o->size_range;
    e.verbose = o->verbose;
    e.engine = o->engine;
    e.budget_s = o->budget_seconds;
    e.table_bytes = o->table_bytes;
    e.stream = o->stream;
    e.unit_log2 = o->unit_log2;
    e.class_prior = o->class_prior;
    e.rank_order = o->rank_order;
    e.grammar = o->grammar;
    e.lanes_log2 = o->lanes_log2 < 0 ? 0 : o->lanes_log2;
    e.filter_samples = o->filter_samples;
  }
  return e;
}

static void fill_result(const SolveOutcome& oc, double secs, simba_result* r, int grammar = 0) {
  memset(r, 0, sizeof(*r));
  r->status = oc.status;
  r->size = oc.size;
  r->op = oc.op;
  r->rank = oc.rank;
  r->table_size = oc.table_size;
  snprintf(r->postfix, sizeof(r->postfix), "%s", oc.postfix.c_str());
  if (oc.status == SIMBA_OK) {
    std::string e = format_postfix(oc.postfix, 0, grammar);
    snprintf(r->expr, sizeof(r->expr), "%s", e.c_str());
  } else {
    snprintf(r->expr, sizeof(r->expr), "Not found !");
  }
  r->seconds = secs;
  r->device_ms = oc.device_ms;
  r->candidates = oc.candidates;
  r->evaluated = oc.evaluated;
  for (int s = 0; s <= kMaxSize; ++s) r->per_size[s] = oc.per_size[s];
  r->max_size_searched = oc.max_size_searched;
  r->launches = oc.launches;
  r->kernel_ms = oc.kernel_ms;
  r->alg_ops = oc.alg_ops;
  r->join_ms = oc.join_ms;
  r->nested_ms = oc.nested_ms;
  r->join_candidates = oc.join_candidates;
  r->nested_candidates = oc.nested_candidates;
  r->join_bytes_streamed = oc.join_bytes_streamed;
  r->join_table_bytes = oc.join_table_bytes;
  r->nested_live_candidates = oc.nested_live_candidates;
}

int read_instance_json(const std::string& path, HostInstance* h) {
  std::ifstream f(path, std::ios::binary);
  if (!f) {
    set_last_error("Error: Could not open file " + path);
    return SIMBA_E_IO;
  }
  std::stringstream ss;
  ss << f.rdbuf();
  const std::string text = ss.str();
  JVal root;
  JParser jp(text);
  if (!jp.parse(&root) || root.kind != JVal::OBJ) {
    set_last_error(jp.error());
    return SIMBA_E_IO;
  }
  const JVal* nv = root.get("num_variables");
  const JVal* ne = root.get("num_examples");
  const JVal* ex = root.get("examples");
  if (!nv || !ne || !ex || !nv->is_int || !ne->is_int || ex->kind != JVal::ARR) {
    set_last_error("missing num_variables / num_examples / examples");
    return SIMBA_E_IO;
  }
  h->k = (int)nv->u;
  h->S = (int)ne->u;
  h->bits = 32;
  h->in.clear();
  h->out.clear();
  // Sample-major like instance.cpp:14-24; "size": 64 anywhere selects u64.
  for (const JVal& e : ex->a) {
    const JVal* o = e.get("output");
    const JVal* in = e.get("inputs");
    if (!o || o->kind != JVal::ARR || o->a.empty() || !in || in->kind != JVal::ARR) {
      set_last_error("malformed example");
      return SIMBA_E_IO;
    }
    const JVal* ov = o->a[0].get("value");
    const JVal* os = o->a[0].get("size");
    if (!ov || !ov->is_int) {
      set_last_error("malformed output value");
      return SIMBA_E_IO;
    }
    if (os && os->is_int && os->u == 64) h->bits = 64;
    h->out.push_back(ov->u);
    for (const JVal& x : in->a) {
      const JVal* xv = x.get("value");
      const JVal* xs = x.get("size");
      if (!xv || !xv->is_int) {
        set_last_error("malformed input value");
        return SIMBA_E_IO;
      }
      if (xs && xs->is_int && xs->u == 64) h->bits = 64;
      h->in.push_back(xv->u);
    }
  }
  if ((int)h->out.size() != h->S || (int)h->in.size() != h->S * h->k) {
    set_last_error("examples do not match num_examples x num_variables");
    return SIMBA_E_IO;
  }
  const uint64_t m = wmask(h->bits);
  for (auto& x : h->in) x &= m;
  for (auto& x : h->out) x &= m;
  return 0;
}

}  // namespace simba

using namespace simba;

struct simba_mlp {
  Mlp* m = nullptr;
};

static int to_hosts(const simba_instance* insts, int n, std::vector<HostInstance>* hs) {
  if (!insts || n < 1) {
    set_last_error("empty instance list");
    return SIMBA_E_ARG;
  }
  hs->resize(n);
  for (int i = 0; i < n; ++i) {
    const int rc = to_host(insts + i, &(*hs)[i]);
    if (rc) return rc;
  }
  return 0;
}

struct simba_session {
  SearchSession* s = nullptr;
  HostInstance h;
};

// The extended grammar is an option of simba_solve and vfb_solve only.
static bool grammar_unsupported(const simba_options* opt) {
  if (!opt || opt->grammar == 0) return false;
  set_last_error("grammar 1 (extended) is supported by simba_solve and vfb_solve only");
  return true;
}

extern "C" {

int simba_solve(const simba_instance* inst, int max_size, const simba_options* opt,
                simba_result* result) {
  if (!result) return SIMBA_E_ARG;
  memset(result, 0, sizeof(*result));
  const auto t0 = std::chrono::steady_clock::now();
  HostInstance h;
  int rc = to_host(inst, &h);
  if (!rc) rc = validate(h, max_size);
  if (rc) {
    result->status = rc;
    return rc;
  }
  if (opt && (opt->rank_order < 0 || opt->rank_order > 1 ||
              (opt->rank_order == 1 && (opt->class_prior || opt->engine == 1)))) {
    set_last_error("rank_order must be 0, or 1 for the plain spine search");
    result->status = SIMBA_E_ARG;
    return SIMBA_E_ARG;
  }
  if (opt && (opt->grammar < 0 || opt->grammar > 1)) {
    set_last_error("grammar must be 0 (reference) or 1 (extended)");
    result->status = SIMBA_E_ARG;
    return SIMBA_E_ARG;
  }
  if (opt && opt->grammar == 1) {
    if (opt->rank_order != 0 || opt->class_prior) {
      set_last_error("the extended grammar runs the plain rank order only");
      result->status = SIMBA_E_ARG;
      return SIMBA_E_ARG;
    }
    SolveOutcome oc;
    rc = ext_solve(h, max_size, to_opts(opt), &oc);
    const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    if (rc < 0) {
      memset(result, 0, sizeof(*result));
      result->status = rc;
      return rc;
    }
    fill_result(oc, secs, result, 1);
    return result->status;
  }
  SearchSession* s = nullptr;
  rc = make_search_session(h, to_opts(opt), &s);
  if (rc) {
    result->status = rc;
    return rc;
  }
  SolveOutcome oc;
  rc = s->solve(max_size, &oc);
  delete s;
  const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  if (rc < 0) {
    result->status = rc;
    return rc;
  }
  fill_result(oc, secs, result);
  return result->status;
}

int simba_solve_noalloc(const simba_instance* inst, int max_size, const simba_options* opt,
                        simba_result* result) {
  if (!result) return SIMBA_E_ARG;
  memset(result, 0, sizeof(*result));
  const auto t0 = std::chrono::steady_clock::now();
  HostInstance h;
  int rc = to_host(inst, &h);
  if (!rc) rc = validate(h, max_size);
  if (rc) {
    result->status = rc;
    return rc;
  }
  if (opt && opt->rank_order != 0) {
    set_last_error("rank_order 1 (RTid) is supported by simba_solve only");
    result->status = SIMBA_E_ARG;
    return SIMBA_E_ARG;
  }
  if (opt && (opt->engine != 0 || opt->class_prior)) {
    set_last_error("simba_solve_noalloc runs the plain spine search only (engine 0, no class_prior)");
    result->status = SIMBA_E_ARG;
    return SIMBA_E_ARG;
  }
  if (grammar_unsupported(opt)) {
    result->status = SIMBA_E_ARG;
    return SIMBA_E_ARG;
  }
  SolveOutcome oc;
  rc = solve_static(h, max_size, to_opts(opt), &oc);
  const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  if (rc < 0) {
    result->status = rc;
    return rc;
  }
  fill_result(oc, secs, result);
  return result->status;
}

int simba_solve_batch(const simba_instance* insts, int n, const int max_size_arg,
                      const simba_options* opt, simba_batch_result* results, simba_batch_stats* stats) {
  if (!insts || n < 0 || !results) return SIMBA_E_ARG;
  if (grammar_unsupported(opt)) return SIMBA_E_ARG;
  if (opt && opt->rank_order != 0) {
    set_last_error("rank_order 1 (RTid) is supported by simba_solve only");
    return SIMBA_E_ARG;
  }
  const auto t0 = std::chrono::steady_clock::now();
  std::vector<HostInstance> hs(n);
  for (int i = 0; i < n; ++i) {
    const int rc = to_host(insts + i, &hs[i]);
    if (rc) return rc;
  }
  BatchOutcome oc;
  const int rc = batch_solve(hs, max_size_arg, to_opts(opt), opt ? opt->table_bytes : 0, &oc);
  if (rc < 0) return rc;
  int solved = 0;
  for (int i = 0; i < n; ++i) {
    simba_batch_result& r = results[i];
    memset(&r, 0, sizeof(r));
    const BatchItemOutcome& o = oc.items[i];
    r.status = o.status;
    r.size = o.size;
    r.op = o.op;
    r.rank = o.rank;
    snprintf(r.postfix, sizeof(r.postfix), "%s", o.postfix.c_str());
    r.seconds = o.seconds;
    r.candidates = o.candidates;
    solved += o.status == SIMBA_OK;
  }
  if (stats) {
    memset(stats, 0, sizeof(*stats));
    stats->seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    stats->device_ms = oc.device_ms;
    stats->kernel_ms = oc.kernel_ms;
    stats->alg_ops = oc.alg_ops;
    stats->candidates = oc.candidates;
    stats->evaluated = oc.evaluated;
    stats->rounds = oc.rounds;
    stats->launches = oc.launches;
    stats->solved = solved;
  }
  return 0;
}

int simba_session_create(const simba_instance* inst, const simba_options* opt,
                         simba_session** session) {
  if (!session) return SIMBA_E_ARG;
  *session = nullptr;
  if (grammar_unsupported(opt)) return SIMBA_E_ARG;
  if (opt && opt->rank_order != 0) {
    set_last_error("rank_order 1 (RTid) is supported by simba_solve only");
    return SIMBA_E_ARG;
  }
  auto* ss = new simba_session();
  int rc = to_host(inst, &ss->h);
  if (!rc) rc = make_search_session(ss->h, to_opts(opt), &ss->s);
  if (rc) {
    delete ss;
    return rc;
  }
  *session = ss;
  return 0;
}

int simba_session_solve(simba_session* session, int max_size, simba_result* result) {
  if (!session || !result) return SIMBA_E_ARG;
  int rc = validate(session->h, max_size);
  if (rc) return rc;
  const auto t0 = std::chrono::steady_clock::now();
  SolveOutcome oc;
  rc = session->s->solve(max_size, &oc);
  const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  if (rc < 0) {
    memset(result, 0, sizeof(*result));
    result->status = rc;
    return rc;
  }
  fill_result(oc, secs, result);
  return result->status;
}

int simba_session_sweep(simba_session* session, int lo, int hi, simba_result* result) {
  if (!session || !result || lo < 1 || hi < lo || hi > kMaxSize) return SIMBA_E_ARG;
  const auto t0 = std::chrono::steady_clock::now();
  SolveOutcome oc;
  int rc = session->s->sweep(lo, hi, &oc);
  const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  if (rc < 0) {
    memset(result, 0, sizeof(*result));
    result->status = rc;
    return rc;
  }
  fill_result(oc, secs, result);
  return result->status;
}

int vfb_solve(const simba_instance* inst, int max_len, const simba_options* opt, vfb_result* result) {
  if (!result) return SIMBA_E_ARG;
  memset(result, 0, sizeof(*result));
  const auto t0 = std::chrono::steady_clock::now();
  HostInstance h;
  int rc = to_host(inst, &h);
  if (rc) {
    result->status = rc;
    return rc;
  }
  if (opt && (opt->grammar < 0 || opt->grammar > 1 ||
              (opt->grammar == 1 && opt->vfb_reference_dedup))) {
    set_last_error("grammar must be 0, or 1 (extended) without vfb_reference_dedup");
    result->status = SIMBA_E_ARG;
    return SIMBA_E_ARG;
  }
  VfbOutcome oc;
  rc = vfb_run(h, max_len, to_opts(opt), opt ? opt->vfb_reference_dedup : 0,
               opt ? opt->vfb_cache_rows : 0, &oc);
  const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  if (rc < 0) {
    result->status = rc;
    return rc;
  }
  result->status = oc.status;
  result->size = oc.size;
  result->op = oc.op;
  result->max_size_searched = oc.max_size_searched;
  snprintf(result->postfix, sizeof(result->postfix), "%s", oc.postfix.c_str());
  if (oc.status == SIMBA_OK) {
    const std::string e = format_postfix(oc.postfix, 1, opt ? opt->grammar : 0);
    snprintf(result->expr, sizeof(result->expr), "%s", e.c_str());
  } else {
    snprintf(result->expr, sizeof(result->expr), "Not found !");
  }
  result->seconds = secs;
  result->device_ms = oc.device_ms;
  result->candidates = oc.candidates;
  result->rows_total = oc.rows_total;
  for (int i = 0; i <= 100; ++i) result->rows_per_size[i] = oc.rows_per_size[i];
  result->cache_bytes = oc.cache_bytes;
  result->table_bytes = oc.table_bytes;
  result->bytes_moved = oc.bytes_moved;
  result->launches = oc.launches;
  return result->status;
}

int simba_session_search_size(simba_session* session, int size, int shard, int nshards,
                              simba_size_result* result) {
  if (!session || !result) return SIMBA_E_ARG;
  memset(result, 0, sizeof(*result));
  SizeOutcome oc;
  const int rc = session->s->search_one_size(size, shard, nshards, &oc);
  if (rc < 0) {
    result->status = rc;
    return rc;
  }
  result->status = oc.status;
  result->launches = oc.launches;
  result->best_rank = oc.best;
  result->candidates = oc.candidates;
  result->evaluated = oc.evaluated;
  result->device_ms = oc.device_ms;
  result->kernel_ms = oc.kernel_ms;
  return oc.status;
}

void simba_session_destroy(simba_session* session) {
  if (!session) return;
  delete session->s;
  delete session;
}

int simba_count_table(int max_size, int n_terms, uint64_t* table) {
  if (!table || max_size < 1 || max_size > kMaxSize || n_terms < 1) return SIMBA_E_ARG;
  CountTable t;
  const bool ok = build_count_table(max_size, n_terms, &t);
  for (int s = 0; s <= max_size; ++s)
    for (int c = 0; c < kCols; ++c) table[s * kCols + c] = t.n[s][c];
  return ok ? 0 : SIMBA_E_OVERFLOW;
}

int simba_unrank(uint64_t rank, int size, int n_terms, char* postfix) {
  if (!postfix || size < 1 || size > kMaxSize || n_terms < 1 || n_terms > kMaxTerms) return SIMBA_E_ARG;
  CountTable t;
  if (!build_count_table(size, n_terms, &t)) return SIMBA_E_OVERFLOW;
  if (rank >= t.n[size][8]) return SIMBA_E_ARG;
  unrank(rank, size, t.n, postfix);
  postfix[size] = 0;
  return 0;
}

int simba_rank_of(const char* postfix, int n_terms, uint64_t* rank) {
  if (!postfix || !rank || n_terms < 1 || n_terms > kMaxTerms) return SIMBA_E_ARG;
  const int len = (int)strlen(postfix);
  if (len < 1 || len > kMaxSize) return SIMBA_E_ARG;
  CountTable t;
  if (!build_count_table(len, n_terms, &t)) return SIMBA_E_OVERFLOW;
  return rank_of(postfix, len, t.n, n_terms, rank) ? 0 : SIMBA_E_ARG;
}

int simba_format(const char* postfix, int style, char* out, int cap) {
  if (!postfix || !out || cap <= 0) return SIMBA_E_ARG;
  const std::string s = format_postfix(postfix, style & 1, (style >> 1) & 1);
  if (s.empty()) return SIMBA_E_ARG;
  if ((int)s.size() + 1 > cap) return SIMBA_E_ARG;
  memcpy(out, s.c_str(), s.size() + 1);
  return (int)s.size();
}

int simba_instance_load(const char* path, simba_instance* inst) {
  if (!path || !inst) return SIMBA_E_ARG;
  memset(inst, 0, sizeof(*inst));
  HostInstance h;
  int rc = read_instance_json(path, &h);
  if (rc) return rc;
  uint64_t* in = new uint64_t[h.in.size()];
  uint64_t* out = new uint64_t[h.out.size()];
  memcpy(in, h.in.data(), h.in.size() * sizeof(uint64_t));
  memcpy(out, h.out.data(), h.out.size() * sizeof(uint64_t));
  inst->num_variables = h.k;
  inst->num_examples = h.S;
  inst->word_bits = h.bits;
  inst->inputs = in;
  inst->outputs = out;
  return 0;
}

void simba_instance_free(simba_instance* inst) {
  if (!inst) return;
  delete[] inst->inputs;
  delete[] inst->outputs;
  inst->inputs = nullptr;
  inst->outputs = nullptr;
}

int simba_int_peak(int device, double* lane_ops_per_s) {
  if (!lane_ops_per_s) return SIMBA_E_ARG;
  return measure_int_peak(device, lane_ops_per_s);
}

int simba_shape_class(const char* postfix) {
  if (!postfix) return SIMBA_E_ARG;
  const int len = (int)strlen(postfix);
  if (len < 2) return len == 1 ? 0 : SIMBA_E_ARG;
  const int op = char_op(postfix[len - 1]);
  if (op < 0) return SIMBA_E_ARG;
  if (is_unary(op)) {
    int m = 0;
    for (int i = len - 1; i >= 0 && char_op(postfix[i]) >= 0 && is_unary(char_op(postfix[i])); --i) ++m;
    return op * 8 + (m < 7 ? m : 7);
  }
  int need = 1, f = -1;
  for (int i = len - 2; i >= 0; --i) {
    const int o = char_op(postfix[i]);
    need -= 1;
    if (o >= 0) need += is_unary(o) ? 1 : 2;
    if (need == 0) {
      f = i;
      break;
    }
  }
  if (f <= 0) return SIMBA_E_ARG;
  return op * 8 + (f < 7 ? f : 7);
}

int64_t simba_mlp_param_count(void) { return (int64_t)mlp_param_count(); }

int simba_mlp_create(int device, uint64_t seed, simba_mlp** mlp) {
  if (!mlp) return SIMBA_E_ARG;
  *mlp = nullptr;
  auto* h = new simba_mlp();
  const int rc = mlp_create(device, seed, &h->m);
  if (rc) {
    delete h;
    return rc;
  }
  *mlp = h;
  return 0;
}

void simba_mlp_destroy(simba_mlp* mlp) {
  if (!mlp) return;
  mlp_destroy(mlp->m);
  delete mlp;
}

int simba_mlp_train_step(simba_mlp* mlp, const simba_instance* insts, int n, const int32_t* labels,
                         float lr, float* loss) {
  if (!mlp || !labels) return SIMBA_E_ARG;
  std::vector<HostInstance> hs;
  int rc = to_hosts(insts, n, &hs);
  if (rc) return rc;
  for (int i = 0; i < n; ++i)
    if (labels[i] < 0 || labels[i] >= 64) return SIMBA_E_ARG;
  return mlp_train_step(mlp->m, hs, labels, lr, loss);
}

int simba_mlp_gradients(simba_mlp* mlp, const simba_instance* insts, int n, const int32_t* labels,
                        float* grads, float* loss) {
  if (!mlp || !labels || !grads) return SIMBA_E_ARG;
  std::vector<HostInstance> hs;
  int rc = to_hosts(insts, n, &hs);
  if (rc) return rc;
  return mlp_gradients(mlp->m, hs, labels, grads, loss);
}

int simba_mlp_apply(simba_mlp* mlp, const float* grads, float lr) {
  if (!mlp || !grads) return SIMBA_E_ARG;
  return mlp_apply(mlp->m, grads, lr);
}

int simba_mlp_predict(simba_mlp* mlp, const simba_instance* insts, int n, float* probs) {
  if (!mlp || !probs) return SIMBA_E_ARG;
  std::vector<HostInstance> hs;
  int rc = to_hosts(insts, n, &hs);
  if (rc) return rc;
  return mlp_predict(mlp->m, hs, probs);
}

int simba_mlp_features(simba_mlp* mlp, const simba_instance* insts, int n, float* features) {
  if (!mlp || !features) return SIMBA_E_ARG;
  std::vector<HostInstance> hs;
  int rc = to_hosts(insts, n, &hs);
  if (rc) return rc;
  return mlp_features(mlp->m, hs, features);
}

int simba_mlp_get_params(simba_mlp* mlp, float* params) {
  if (!mlp || !params) return SIMBA_E_ARG;
  return mlp_get_params(mlp->m, params);
}

int simba_mlp_set_params(simba_mlp* mlp, const float* params) {
  if (!mlp || !params) return SIMBA_E_ARG;
  return mlp_set_params(mlp->m, params);
}

int simba_alu_peak(int device, double* lane_ops_per_s) {
  if (!lane_ops_per_s) return SIMBA_E_ARG;
  return measure_alu_peak(device, lane_ops_per_s);
}

const char* simba_version(void) { return "simba_b200 0.1 (sm_100a)"; }

const char* simba_status_string(int status) {
  switch (status) {
    case SIMBA_OK: return "found";
    case SIMBA_NOT_FOUND: return "not found";
    case SIMBA_BUDGET: return "time budget exhausted";
    case SIMBA_CACHE_FULL: return "cache full";
    case SIMBA_E_ARG: return "invalid argument";
    case SIMBA_E_CUDA: return "CUDA error";
    case SIMBA_E_NOMEM: return "out of memory";
    case SIMBA_E_NODEV: return "no CUDA device";
    case SIMBA_E_OVERFLOW: return "count overflow";
    case SIMBA_E_INTERNAL: return "internal error";
    case SIMBA_E_IO: return "I/O error";
  }
  return "unknown status";
}

const char* simba_last_error(void) { return g_last_error.c_str(); }

int simba_release_device_cache(void) {
  DeviceCache& c = cache();
  std::lock_guard<std::mutex> g(c.mu);
  drop_cached(c, -1);
  return 0;
}

int simba_device_count(void) {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess) return 0;
  return n;
}

}  // extern "C"
