// 32-bit word instantiation of the plain search engine (the reference's
// uint32_t arithmetic, simba/src/mba.cuh:8).
#include "search_impl.cuh"

namespace simba {

int make_search_u32(const HostInstance& h, const EngineOptions& o, SearchSession** out) {
  return make_search_typed<uint32_t>(h, o, out);
}

int batch_u32(const std::vector<HostInstance>& hs, int max_size, const EngineOptions& o,
              int64_t inst_table_bytes, BatchOutcome* out) {
  return batch_typed<uint32_t>(hs, max_size, o, inst_table_bytes, out);
}

}  // namespace simba
