// `simba <instance.json> <maxLen>`: drop-in for the reference SIMBA executable
// (simba/src/nocache.cu:291-342).  Same arguments, same checks and exit
// codes, same stdout line "<file>,<expr>,<seconds>" (or "<file>,Not found !,
// <seconds>"); the count table and the running time go to stderr.  The timer
// wraps the whole solve, CUDA context creation included, as in the
// reference.  Optional flags before the positional arguments:
//   --budget S     stop after S seconds (prints "Not found !")
//   --complete     also search size 1 and size maxLen
//   --naive        one thread per rank instead of the tabled engine
//   --verbose      per-size progress on stderr
//   --rtid         RTid order (the reference's simba_rtid build); the same
//                  source built with SIMBA_CLI_RTID=1 is the simba_rtid
//                  executable, for which this is the default
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
#if defined(SIMBA_CLI_RTID) && SIMBA_CLI_RTID
  opt.rank_order = 1;
#endif
  std::vector<char*> pos;
  pos.push_back(argv[0]);
  for (int i = 1; i < argc; ++i) {
    if (!strcmp(argv[i], "--budget") && i + 1 < argc) opt.budget_seconds = atof(argv[++i]);
    else if (!strcmp(argv[i], "--complete")) opt.size_range = 1;
    else if (!strcmp(argv[i], "--naive")) opt.engine = 1;
    else if (!strcmp(argv[i], "--verbose")) opt.verbose = 1;
    else if (!strcmp(argv[i], "--rtid")) opt.rank_order = 1;
    else pos.push_back(argv[i]);
  }
  if (pos.size() != 3) {
    fprintf(stderr, "Arguments should be in the form of\n");
    fprintf(stderr, "-----------------------------------------------------------------\n");
    fprintf(stderr, "%s <input_file_address> <maxLen>\n", argv[0]);
    fprintf(stderr, "-----------------------------------------------------------------\n");
    return 0;
  }
  const int max_len = atoi(pos[2]);
  if (max_len < 1 || max_len > 50) {
    fprintf(stderr, "Argument maxLen = %s should be between 1 and %d", pos[2], 32);
    return 0;
  }
  const std::string file_name = pos[1];
  simba::HostInstance h;
  if (simba::read_instance_json(file_name, &h) != 0) {
    fprintf(stderr, "%s\n", simba::last_error().c_str());
    return 1;
  }
  const auto start = std::chrono::high_resolution_clock::now();
  simba_instance inst;
  memset(&inst, 0, sizeof(inst));
  inst.num_variables = h.k;
  inst.num_examples = h.S;
  inst.word_bits = h.bits;
  inst.inputs = h.in.data();
  inst.outputs = h.out.data();
  simba_result res;
  const int rc = simba_solve(&inst, max_len, &opt, &res);
  const auto stop = std::chrono::high_resolution_clock::now();
  if (rc < 0) {
    // The reference throws (no CSV line) on limit violations and asserts on
    // CUDA errors; report and exit without a stdout line.
    fprintf(stderr, "error: %s: %s\n", simba_status_string(rc), simba_last_error());
    return 1;
  }
  if (max_len <= 32) {
    std::vector<uint64_t> t((size_t)(max_len + 1) * 9);
    if (simba_count_table(max_len, h.k, t.data()) == 0)
      for (int i = 0; i <= max_len; ++i) {
        for (int j = 0; j < 9; ++j) fprintf(stderr, "%-12llu ", (unsigned long long)t[i * 9 + j]);
        fprintf(stderr, "\n");
      }
  }
  const auto duration = std::chrono::duration_cast<std::chrono::microseconds>(stop - start).count();
  const double time_s = (double)duration / 1e6;
  fprintf(stderr, "\nRunning Time: %f s", (double)duration * 0.000001);
  const std::string output = rc == SIMBA_OK ? std::string(res.expr) : std::string("Not found !");
  std::cout << file_name << "," << output << "," << time_s << std::endl;
  return 0;
}
