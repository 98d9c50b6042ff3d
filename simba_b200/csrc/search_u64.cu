// 64-bit word instantiation of the plain search engine, and the session
// factory that dispatches on the instance's word width.
#include "search_impl.cuh"

namespace simba {

int make_search_u32(const HostInstance& h, const EngineOptions& o, SearchSession** out);

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
