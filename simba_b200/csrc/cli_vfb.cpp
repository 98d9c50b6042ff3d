// `vfb <instance.json> <maxLen>`: drop-in for the reference VFB executable
// (vfb/src/full-cache.cu:776-854).  Same arguments and checks (maxLen in
// 1..100), the same stderr summary and the same stdout line
// "<file>,<expr>,<seconds>" with the VFB expression syntax.  Optional flags
// before the positional arguments:
//   --reference-dedup   keep the reference's uniqueness test as written
//   --cache-rows N      row capacity (default: the reference's rule)
//   --budget S          stop after S seconds
//   --verbose           per-size progress on stderr
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <iostream>
#include <string>
#include <vector>

#include "../../include/simba_b200.h"
#include "engine.h"

int main(int argc, char* argv[]) {
  simba_options opt;
  memset(&opt, 0, sizeof(opt));
  std::vector<char*> pos;
  pos.push_back(argv[0]);
  for (int i = 1; i < argc; ++i) {
    if (!strcmp(argv[i], "--reference-dedup")) opt.vfb_reference_dedup = 1;
    else if (!strcmp(argv[i], "--cache-rows") && i + 1 < argc) opt.vfb_cache_rows = atoll(argv[++i]);
    else if (!strcmp(argv[i], "--budget") && i + 1 < argc) opt.budget_seconds = atof(argv[++i]);
    else if (!strcmp(argv[i], "--verbose")) opt.verbose = 1;
    else pos.push_back(argv[i]);
  }
  if (pos.size() != 3) {
    fprintf(stderr, "Arguments should be in the form of\n");
    fprintf(stderr, "-----------------------------------------------------------------\n");
    fprintf(stderr, "%s <input_file_address> <maxLen>\n", argv[0]);
    fprintf(stderr, "-----------------------------------------------------------------\n");
    return 0;
  }
  if (atoi(pos[2]) < 1 || atoi(pos[2]) > 100) {
    fprintf(stderr, "Argument maxLen = %s should be between 1 and 100", pos[2]);
    return 0;
  }
  const std::string file_name = pos[1];
  const int max_len = atoi(pos[2]);
  simba::HostInstance h;
  if (simba::read_instance_json(file_name, &h) != 0) {
    fprintf(stderr, "%s\n", simba::last_error().c_str());
    return 1;
  }
  simba_instance inst;
  memset(&inst, 0, sizeof(inst));
  inst.num_variables = h.k;
  inst.num_examples = h.S;
  inst.word_bits = h.bits;
  inst.inputs = h.in.data();
  inst.outputs = h.out.data();
  const auto start = std::chrono::high_resolution_clock::now();
  vfb_result res;
  const int rc = vfb_solve(&inst, max_len, &opt, &res);
  const auto stop = std::chrono::high_resolution_clock::now();
  if (rc < 0) {
    fprintf(stderr, "error: %s: %s\n", simba_status_string(rc), simba_last_error());
    return 1;
  }
  const std::string output = rc == SIMBA_OK ? std::string(res.expr) : std::string("Not found !");
  fprintf(stderr, "Input file : %s\n", file_name.c_str());
  fprintf(stderr, "Max length : %d\n", max_len);
  if (rc != SIMBA_OK) fprintf(stderr, "Result     : no expression found within length %d\n", max_len);
  else fprintf(stderr, "Result     : expression found\n");
  const auto duration = std::chrono::duration_cast<std::chrono::microseconds>(stop - start).count();
  const double time_s = (double)duration / 1e6;
  fprintf(stderr, "\nRunning Time: %f s", (double)duration * 0.000001);
  std::cout << file_name << "," << output << "," << time_s << std::endl;
  return 0;
}
