// Drop-in `near_clique` executable: the reference's pattern-aware queries q4_PA .. q13_PA
// (src/main/q4_PA.cu .. q13_PA.cu, run with k = n) in one program: the number of non-induced
// copies of K_k minus one edge, k in [4, 13], printed as the reference's drivers print their
// count (outputAggregateCounter, src/main/DuMatoCPU.cu:360-362) with the same timer lines.
#include "cli_common.hpp"

int main(int argc, const char** argv) {
  dmcli::Timer total;
  dmcli::Args a;
  if (!dmcli::parse(argc, argv, "pattern (K_k minus one edge)", a)) return 1;
  dmcli::Timer io;
  dm_graph* g = nullptr;
  if (dm_graph_load_edgelist(a.graph, &g) != DM_OK) return dmcli::die("reading the graph");
  const double io_s = io.seconds();
  dm_opts o = dmcli::make_opts(a);
  dm_stats st{};
  uint64_t count = 0;
  dmcli::Timer gpu;
  if (dm_count_near_cliques(g, a.k, &o, &count, &st) != DM_OK) {
    dm_graph_free(g);
    return dmcli::die("pattern counting");
  }
  const double gpu_s = gpu.seconds();
  std::printf("Result: %lu.\n", (unsigned long)count);
  dmcli::print_times(gpu_s, 0.0, io_s, total.seconds());
  dm_graph_free(g);
  return 0;
}
