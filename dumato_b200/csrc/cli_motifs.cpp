// Drop-in `motifs` executable: per-class counts of connected induced k-vertex subgraphs.
// Output lines as the reference's motif driver (outputAggregatePattern,
// src/main/DuMatoCPU.cu:364-384): one "class, count" line per non-zero class, then
// "Aggregated: total, classes patterns.". The class table is read, as the reference reads
// it (src/main/QuickMapping.cpp:14), from ../dictionaries/<k>.csv relative to the working
// directory; where that file is missing the table is generated instead of aborting.
#include <sys/stat.h>

#include <vector>

#include "cli_common.hpp"

int main(int argc, const char** argv) {
  dmcli::Timer total;
  dmcli::Args a;
  if (!dmcli::parse(argc, argv, "motifs", a)) return 1;
  dmcli::Timer io;
  dm_graph* g = nullptr;
  if (dm_graph_load_edgelist(a.graph, &g) != DM_OK) return dmcli::die("reading the graph");
  dm_dictionary* d = nullptr;
  const std::string path = "../dictionaries/" + std::to_string(a.k) + ".csv";
  struct stat sb;
  if (stat(path.c_str(), &sb) == 0) {
    if (dm_dictionary_load_csv(path.c_str(), &d) != DM_OK) return dmcli::die("reading the dictionary");
  } else {
    std::printf("[dictionary] %s not found: generating the k=%d table\n", path.c_str(), a.k);
    if (dm_dictionary_generate(a.k, &d) != DM_OK) return dmcli::die("generating the dictionary");
  }
  const double io_s = io.seconds();
  int32_t kk = 0, nc = 0;
  int64_t nq = 0;
  dm_dictionary_shape(d, &kk, &nq, &nc);
  std::vector<uint64_t> counts(nc, 0);
  dm_opts o = dmcli::make_opts(a);
  dm_stats st{};
  dmcli::Timer gpu;
  if (dm_count_motifs(g, a.k, d, &o, counts.data(), &st) != DM_OK) {
    dm_dictionary_free(d);
    dm_graph_free(g);
    return dmcli::die("motif counting");
  }
  const double gpu_s = gpu.seconds();
  unsigned long total_subgraphs = 0;
  unsigned patterns = 0;
  for (int32_t c = 0; c < nc; ++c)
    if (counts[c]) {
      ++patterns;
      std::printf("%d, %lu\n", c, (unsigned long)counts[c]);
      total_subgraphs += counts[c];
    }
  std::printf("Aggregated: %lu, %u patterns.\n", total_subgraphs, patterns);
  dmcli::print_times(gpu_s, 0.0, io_s, total.seconds());
  dm_dictionary_free(d);
  dm_graph_free(g);
  return 0;
}
