// Allocation-free plain search: simba_solve_noalloc.
//
// For callers that must not allocate device memory while they run -- code
// that executes inside a host application with a fixed GPU memory budget,
// a plugin whose host owns every allocation, or a process that is capturing
// other work into a CUDA graph (cudaMalloc is not allowed during capture).
// All scratch memory of the search (samples, count table, value tables,
// spine items, counters) lives in one file-scope __device__ array of
// kStaticScratchBytes (64 MiB) that every GPU loading the library holds
// until the process exits.  The same kernels as simba_solve run on it.
//
// Rules of use:
//  * The first call on a device looks up the array's device address
//    (cudaGetSymbolAddress) with that device current; make that first call
//    before any stream capture begins.
//  * All calls share the one array and it keeps the last call's contents;
//    the search clears what must start at zero.  Calls whose work overlaps
//    on the GPU (other host threads, other streams) race on it: serialise
//    them.
//  * No stream or event is created: the search runs on options.stream (0 =
//    the legacy default stream) and is timed with the host clock.  While
//    another stream is being captured, pass a non-blocking stream: work on
//    the legacy default stream synchronises with blocking streams and would
//    break that capture.
//  * The looked-up address is cached per device ordinal; it is not valid
//    after cudaDeviceReset destroys the context that holds the array.
//  * Sizes whose value tables or spine list do not fit the array are
//    rejected with SIMBA_E_ARG and a message naming the limit.
#include <cuda_runtime.h>

#include <chrono>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <vector>

// the static entry point runs sizes with small tables: the generic explicit
// level keeps this unit's compile time down (and its kernel a symbol of its own)
#define SIMBA_XOP_SPECIALIZE 0
#include "search_impl.cuh"

namespace simba {

constexpr size_t kStaticScratchBytes = 64ull << 20;
constexpr size_t kStaticFixedBytes = 1ull << 20;     // samples, counts, scalars
constexpr size_t kStaticItemBytes = 24ull << 20;     // spine items
constexpr size_t kStaticTableBytes = kStaticScratchBytes - kStaticFixedBytes - kStaticItemBytes;

static __device__ __align__(256) unsigned char g_static_scratch[kStaticScratchBytes];

namespace {
std::mutex g_addr_mu;
void* g_addr[64] = {};

// Device address of the scratch array for the current device (looked up
// once per device; the array's name in host code is only a stand-in).
int scratch_address(int device, unsigned char** out) {
  if (device < 0 || device >= 64) {
    set_last_error("device ordinal out of range");
    return SIMBA_E_ARG;
  }
  std::lock_guard<std::mutex> lk(g_addr_mu);
  if (!g_addr[device]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_static_scratch);
    if (e != cudaSuccess || !p) {
      set_last_error(std::string("cudaGetSymbolAddress(static scratch): ") + cudaGetErrorString(e));
      return SIMBA_E_CUDA;
    }
    g_addr[device] = p;
  }
  *out = static_cast<unsigned char*>(g_addr[device]);
  return 0;
}
}  // namespace

template <class W>
static int solve_static_typed(const HostInstance& h, int max_size, const EngineOptions& o,
                              SolveOutcome* out) {
  *out = SolveOutcome();
  SB_CUDA(cudaSetDevice(o.device));
  unsigned char* base = nullptr;
  int rc = scratch_address(o.device, &base);
  if (rc) return rc;
  cudaStream_t st = reinterpret_cast<cudaStream_t>(o.stream);

  CountTable ct;
  int count_ok = kMaxSize;
  while (count_ok > 1 && !build_count_table(count_ok, h.k, &ct)) --count_ok;
  build_count_table(count_ok, h.k, &ct);
  const int first = o.size_range ? 1 : 2;
  const int last = o.size_range ? max_size : max_size - 1;
  if (last > count_ok) {
    set_last_error("candidate counts exceed 64 bits at this size");
    return SIMBA_E_OVERFLOW;
  }

  // Fixed region: counts | scalars | samples (16-byte padded).
  unsigned char* p_counts = base;
  unsigned long long* p_scal = reinterpret_cast<unsigned long long*>(base + 4096);
  unsigned char* p_desc = base + 4096 + 256;  // one InstDesc (< 512 bytes)
  unsigned char* p_in = base + 8192;
  const size_t nin16 = ((size_t)h.S * h.k * sizeof(W) + 15) / 16;
  const size_t nout16 = ((size_t)h.S * sizeof(W) + 15) / 16;
  unsigned char* p_out = p_in + nin16 * 16;
  if (8192 + (nin16 + nout16) * 16 > kStaticFixedBytes) {
    set_last_error("instance too large for the static scratch");
    return SIMBA_E_ARG;
  }
  Item* p_items = reinterpret_cast<Item*>(base + kStaticFixedBytes);
  unsigned char* p_tab = base + kStaticFixedBytes + kStaticItemBytes;

  std::vector<W> win(nin16 * 16 / sizeof(W), 0), wout(nout16 * 16 / sizeof(W), 0);
  for (size_t i = 0; i < (size_t)h.S * h.k; ++i) win[i] = (W)h.in[i];
  for (int i = 0; i < h.S; ++i) wout[i] = (W)h.out[i];
  SB_CUDA(cudaMemcpyAsync(p_counts, ct.n, sizeof(ct.n), cudaMemcpyHostToDevice, st));
  SB_CUDA(cudaMemcpyAsync(p_in, win.data(), nin16 * 16, cudaMemcpyHostToDevice, st));
  SB_CUDA(cudaMemcpyAsync(p_out, wout.data(), nout16 * 16, cudaMemcpyHostToDevice, st));

  // Largest tabled size whose tables fit the table region.
  auto padded = [](uint64_t n) { return (n + 63) / 64 * 64 + 64; };
  uint64_t off[kMaxSize + 1] = {};
  uint64_t total = 0;
  int Tcap = 0;
  for (int t = 1; t <= count_ok && t <= 20; ++t) {
    const uint64_t bytes = padded(ct.n[t][8]) * sizeof(W);
    if (total + bytes > kStaticTableBytes) break;
    off[t] = total;
    total += bytes;
    Tcap = t;
  }
  auto tab = [&](int t) { return reinterpret_cast<W*>(p_tab + off[t]); };

  for (int s = first; s <= last; ++s)
    if (s > Tcap && (s - 1) / 2 > Tcap) {
      set_last_error("size " + std::to_string(s) + " needs value tables beyond the 64 MiB static scratch");
      return SIMBA_E_ARG;
    }
  int sms = 0;
  SB_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, o.device));
  const size_t smem_base = ((sizeof(Smem) + 15) & ~size_t(15)) + (nin16 + nout16) * 16;
  const size_t join_off = (smem_base + 15) & ~size_t(15);  // one launch: join tables included
  const size_t smem = join_off + sizeof(JoinSmem);
  SB_CUDA(raise_smem_limit((const void*)spine_kernel<W>, smem));
  int occ = 1;
  SB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, spine_kernel<W>, kThreads, smem));
  const int grid = sms * std::max(occ, 1);
  const uint64_t mask = h.bits == 64 ? ~0ULL : 0xFFFFFFFFULL;

  stamp_start_kernel<<<1, 1, 0, st>>>(p_scal + 3);
  out->launches = 1;
  SB_CUDA(cudaGetLastError());
  int built = 0;
  for (int s = first; s <= last; ++s) {
    const int T = std::min(Tcap, s);
    if (s > T && (s - 1) / 2 > T) {
      set_last_error("size " + std::to_string(s) + " needs value tables beyond the 64 MiB static scratch");
      return SIMBA_E_ARG;
    }
    std::vector<Item> items;
    if (s <= T) {
      Item it;
      memset(&it, 0, sizeof(it));
      it.bottom = (int8_t)s;
      it.coefv = 1;
      it.nv = ct.n[s][8];
      items.push_back(it);
    } else {
      Enumerator en;
      en.ct = &ct;
      en.T = T;
      en.mask = mask;
      en.items = &items;
      std::vector<Level> lv;
      std::vector<ChainClass> top{{1, 0, 0}};
      en.rec(s, lv, 1, 0, top);
      if (en.too_deep) {
        set_last_error("size " + std::to_string(s) + " needs spines deeper than supported with the static scratch");
        return SIMBA_E_ARG;
      }
    }
    if (items.size() * sizeof(Item) > kStaticItemBytes) {
      set_last_error("size " + std::to_string(s) + " needs " + std::to_string(items.size()) +
                     " spines; the static scratch holds " + std::to_string(kStaticItemBytes / sizeof(Item)));
      return SIMBA_E_ARG;
    }
    // build the value tables this size needs
    for (int t = built + 1; t <= std::min(T, s); ++t) {
      W* o_t = tab(t);
      if (t == 1) {
        std::vector<W> v(padded(h.k), 0);
        for (int j = 0; j < h.k; ++j) v[j] = (W)h.in[j];
        SB_CUDA(cudaMemcpyAsync(o_t, v.data(), v.size() * sizeof(W), cudaMemcpyHostToDevice, st));
        SB_CUDA(cudaStreamSynchronize(st));
      } else {
        uint64_t o2 = 0;
        const int sub = t - 1;
        for (int op = 0; op < 8; ++op) {
          if (is_unary(op)) {
            const uint64_t n = ct.n[sub][8];
            const int blocks = (int)std::min<uint64_t>((n + 255) / 256, (uint64_t)sms * 16);
            build_unary_kernel<W><<<blocks, 256, 0, st>>>(o_t + o2, tab(sub), n, op);
            ++out->launches;
            o2 += n;
            continue;
          }
          const int fmax = is_commutative(op) ? sub / 2 : sub - 1;
          for (int f = 1; f <= fmax; ++f) {
            const uint64_t na = ct.n[f][8], nb = ct.n[sub - f][8];
            const int blocks = (int)std::min<uint64_t>((na * nb + 255) / 256, (uint64_t)sms * 16);
            build_binary_kernel<W><<<blocks, 256, 0, st>>>(o_t + o2, tab(f), tab(sub - f), na, nb, op);
            ++out->launches;
            o2 += na * nb;
          }
        }
      }
      SB_CUDA(cudaGetLastError());
      built = t;
    }
    uint64_t units = 0;
    for (auto& it : items) {
      for (int l = 0; l < it.depth; ++l)
        if (it.lv[l].kind == 1) it.lv[l].c &= mask;
      finish_item(it, kThreads, mask);
      it.unit_begin = units;
      units += item_units(it);
    }
    SB_CUDA(cudaMemcpyAsync(p_items, items.data(), items.size() * sizeof(Item), cudaMemcpyHostToDevice, st));
    // counter = 0, best = ~0, evaluated = 0 (start stamp kept), flags = 0
    const unsigned long long init[3] = {0, ~0ULL, 0};
    SB_CUDA(cudaMemcpyAsync(p_scal, init, sizeof(init), cudaMemcpyHostToDevice, st));
    SB_CUDA(cudaMemsetAsync(p_scal + 4, 0, 4 * sizeof(unsigned long long), st));
    InstDesc<W> d;
    memset(&d, 0, sizeof(d));
    for (int t = 1; t <= built; ++t) d.tab[t] = tab(t);
    d.in = reinterpret_cast<const W*>(p_in);
    d.out = reinterpret_cast<const W*>(p_out);
    d.counts = reinterpret_cast<const unsigned long long*>(p_counts);
    d.best = p_scal + 1;
    d.target = (W)h.out[0];
    d.size = s;
    d.S = h.S;
    d.K = h.k;
    SB_CUDA(cudaMemcpyAsync(p_desc, &d, sizeof(d), cudaMemcpyHostToDevice, st));
    Params<W> p;
    memset(&p, 0, sizeof(p));
    p.insts = reinterpret_cast<const InstDesc<W>*>(p_desc);
    p.items = p_items;
    p.counter = p_scal + 0;
    p.evaluated = p_scal + 2;
    p.start_ns = p_scal + 3;
    p.flags = reinterpret_cast<int*>(p_scal + 4);
    p.maxS = h.S;
    p.maxK = h.k;
    p.budget_ns = o.budget_s > 0 ? (unsigned long long)(o.budget_s * 1e9) : 0;
    p.nitems = (int)items.size();
    p.total_units = units;
    p.stop_on_match = 1;
    p.join_off = (unsigned)join_off;
    spine_kernel<W><<<grid, kThreads, smem, st>>>(p);
    ++out->launches;
    SB_CUDA(cudaGetLastError());
    unsigned long long hs[8];
    SB_CUDA(cudaMemcpyAsync(hs, p_scal, sizeof(hs), cudaMemcpyDeviceToHost, st));
    SB_CUDA(cudaStreamSynchronize(st));
    const int* fl = reinterpret_cast<const int*>(hs + 4);
    out->evaluated += hs[2];
    out->max_size_searched = s;
    out->table_size = std::max(out->table_size, T);
    if (fl[1]) {
      set_last_error("inversion failed on a level marked invertible");
      return SIMBA_E_INTERNAL;
    }
    if (fl[0]) {
      out->status = SIMBA_BUDGET;
      break;
    }
    if (hs[1] != ~0ULL) {
      const uint64_t best = hs[1];
      const int op = s == 1 ? 8 : op_of_rank(ct.n, s, best);
      uint64_t c = 0;
      if (s == 1) c = best + 1;
      else
        for (int q = 0; q <= op; ++q) c += ct.n[s][q];
      out->per_size[s] = c;
      out->candidates += c;
      char buf[kMaxSize + 1];
      unrank(best, s, ct.n, buf);
      buf[s] = 0;
      out->postfix = buf;
      out->size = s;
      out->op = op;
      out->rank = best;
      if (!host_check(out->postfix, h)) {
        set_last_error("device match failed the host re-check");
        return SIMBA_E_INTERNAL;
      }
      out->status = SIMBA_OK;
      break;
    }
    out->per_size[s] = ct.n[s][8];
    out->candidates += ct.n[s][8];
  }
  if (out->status != SIMBA_OK && out->status != SIMBA_BUDGET) out->status = SIMBA_NOT_FOUND;
  out->device_ms = 0.0;
  out->kernel_ms = 0.0;
  return out->status;
}

int solve_static(const HostInstance& h, int max_size, const EngineOptions& o, SolveOutcome* out) {
  int rc = validate(h, max_size);
  if (rc) return rc;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= o.device || o.device < 0) {
    cudaGetLastError();
    set_last_error("no usable CUDA device");
    return SIMBA_E_NODEV;
  }
  if (h.bits == 64) return solve_static_typed<uint64_t>(h, max_size, o, out);
  return solve_static_typed<uint32_t>(h, max_size, o, out);
}

}  // namespace simba
