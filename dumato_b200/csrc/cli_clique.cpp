// Drop-in `clique` executable: k-clique count of an edgelist graph on the GPU.
// Output lines as the reference's clique driver (outputAggregateCounter,
// src/main/DuMatoCPU.cu:360-362, and the timers of src/main/clique_PA.cu:118-121).
#include "cli_common.hpp"

int main(int argc, const char** argv) {
  dmcli::Timer total;
  dmcli::Args a;
  if (!dmcli::parse(argc, argv, "clique", a)) return 1;
  dmcli::Timer io;
  dm_graph* g = nullptr;
  if (dm_graph_load_edgelist(a.graph, &g) != DM_OK) return dmcli::die("reading the graph");
  const double io_s = io.seconds();
  dm_opts o = dmcli::make_opts(a);
  dm_stats st{};
  uint64_t count = 0;
  dmcli::Timer gpu;
  if (dm_count_cliques(g, a.k, &o, &count, &st) != DM_OK) {
    dm_graph_free(g);
    return dmcli::die("clique counting");
  }
  const double gpu_s = gpu.seconds();
  std::printf("Result: %lu.\n", (unsigned long)count);
  dmcli::print_times(gpu_s, 0.0, io_s, total.seconds());
  dm_graph_free(g);
  return 0;
}
