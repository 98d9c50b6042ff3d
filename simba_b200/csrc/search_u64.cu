// 64-bit word instantiation of the plain search engine, and the session
// factory that dispatches on the instance's word width.
#include "search_impl.cuh"

namespace simba {

int make_search_u32(const HostInstance& h, const EngineOptions& o, SearchSession** out);
int batch_u32(const std::vector<HostInstance>& hs, int max_size, const EngineOptions& o,
              int64_t inst_table_bytes, BatchOutcome* out);

int batch_solve(const std::vector<HostInstance>& hs, int max_size, const EngineOptions& o,
                int64_t inst_table_bytes, BatchOutcome* out) {
  if (hs.empty()) return 0;
  for (auto& h : hs) {
    const int rc = validate(h, max_size);
    if (rc) return rc;
    if (h.bits != hs[0].bits) {
      set_last_error("a batch must use one word width");
      return SIMBA_E_ARG;
    }
  }
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= o.device || o.device < 0) {
    cudaGetLastError();
    set_last_error("no usable CUDA device");
    return SIMBA_E_NODEV;
  }
  if (hs[0].bits == 64) return batch_typed<uint64_t>(hs, max_size, o, inst_table_bytes, out);
  return batch_u32(hs, max_size, o, inst_table_bytes, out);
}

int make_search_session(const HostInstance& h, const EngineOptions& o, SearchSession** out) {
  *out = nullptr;
  int rc = validate(h, 1);
  if (rc) return rc;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= o.device || o.device < 0) {
    cudaGetLastError();
    set_last_error("no usable CUDA device");
    return SIMBA_E_NODEV;
  }
  if (h.bits == 64) return make_search_typed<uint64_t>(h, o, out);
  return make_search_u32(h, o, out);
}

}  // namespace simba
