// Shared pieces of the drop-in executables `clique` and `motifs`.
//
// Both take the reference drivers' positional arguments
//     graphFile k threads blockSize donationsPerWarp threshold
// (src/main/clique_PA.cu:35-63, src/main/motifs_DM_WCLB.cu:39-63) and print the same result
// and timing lines, so scripts that parse the reference's output keep working. threads and
// blockSize size the persistent grid, donationsPerWarp bounds the donations a task makes,
// and threshold is the hungry-warp percentage that starts donations (>= 100: none), as in
// the reference where threshold >= 100 skips load balancing (clique_PA.cu:78).
#pragma once

#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <string>

#include "../../include/dumato_b200.h"

namespace dmcli {

struct Args {
  const char* graph = nullptr;
  int k = 0;
  int threads = 0;
  int block = 0;
  int donations = 0;
  int threshold = 0;
};

inline bool parse(int argc, const char** argv, const char* what, Args& a) {
  std::printf("Usage: %s graphFile k threads blockSize donationsPerWarp threshold\n", argv[0]);
  std::printf("\t graphFile: edgelist, one undirected \"src dst\" pair per line\n");
  std::printf("\t k: %s size\n", what);
  std::printf("\t threads: total GPU threads of the persistent grid (e.g. 102400; 0 = one full wave)\n");
  std::printf("\t blockSize: threads per block (e.g. 256)\n");
  std::printf("\t donationsPerWarp: donations one task may make (e.g. 16)\n");
  std::printf("\t threshold: percentage of hungry warps that starts donations (>= 100: none)\n");
  if (argc != 7) {
    std::printf("\nWrong amount of parameters!\nExiting...\n");
    return false;
  }
  a.graph = argv[1];
  a.k = std::atoi(argv[2]);
  a.threads = std::atoi(argv[3]);
  a.block = std::atoi(argv[4]);
  a.donations = std::atoi(argv[5]);
  a.threshold = std::atoi(argv[6]);
  return true;
}

inline dm_opts make_opts(const Args& a) {
  dm_opts o{};
  o.struct_size = sizeof(dm_opts);
  o.device = -1;
  o.threads = a.threads > 0 ? a.threads : 0;
  o.block_size = 0;  // the kernels use their own tuned block shape; threads sizes the grid
  o.donations_per_warp = a.donations > 0 ? a.donations : 16;
  o.threshold = a.threshold < 0 ? 0 : a.threshold;
  return o;
}

struct Timer {
  std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now();
  double seconds() const {
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  }
};

inline int die(const char* step) {
  std::fprintf(stderr, "%s failed: %s\n", step, dm_last_error());
  return 1;
}

inline void print_times(double gpu, double lb, double io, double total) {
  std::printf("Time (GPU): %f secs.\n", gpu);
  std::printf("Time (LB): %f secs.\n", lb);
  std::printf("Time (IO): %f secs\n", io);
  std::printf("Time (TOTAL): %f secs\n", total);
}

}  // namespace dmcli
