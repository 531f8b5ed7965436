// Internal host-side types shared by the library's translation units.
#pragma once

#include <cstdint>
#include <string>
#include <vector>
#include <mutex>

#include "../../include/dumato_b200.h"

namespace dmb {

// Thread-local error message behind dm_last_error().
void set_error(const std::string& msg);
int fail(int status, const std::string& msg);

// Deterministic RNG: splitmix64 seeding + xoshiro256**.
struct Rng {
  uint64_t s[4];
  explicit Rng(uint64_t seed);
  uint64_t next();
  double uniform();                  // [0, 1) with 53 random bits
  uint64_t below(uint64_t bound);    // unbiased in [0, bound)
};

// Device-resident copy of one graph (owned by the graph, one per device). Rows start on
// 16-byte boundaries (offsets are multiples of 4 ints) and are padded with INT32_MAX so a
// row can be read with 128-bit loads.
struct DeviceGraph {
  int device = -1;
  // undirected CSR (motifs), original ids
  int32_t* d_row = nullptr;      // n (padded start offsets)
  int32_t* d_deg = nullptr;      // n
  int32_t* d_adj = nullptr;      // padded adjacency
  // oriented CSR in rank space (cliques)
  int32_t* d_orow = nullptr;     // n
  int32_t* d_odeg = nullptr;     // n
  int32_t* d_oadj = nullptr;     // padded out-adjacency
  bool has_undirected = false;
  bool has_oriented = false;
  double upload_ms = 0;
};

}  // namespace dmb

// Opaque graph handle.
struct dm_graph {
  int32_t n = 0;
  int64_t m = 0;
  int64_t self_loops = 0;
  int64_t input_pairs = 0;
  int32_t max_degree = 0;
  // undirected CSR, rows sorted ascending, no self-loops, no duplicates
  std::vector<int64_t> row;      // n+1
  std::vector<int32_t> adj;      // 2m
  // degree-ordered orientation: rank[v] = position of v in (degree, id) order;
  // out-neighbours of rank r are ranks > r, sorted ascending
  bool oriented_built = false;
  std::vector<int32_t> rank;     // n
  std::vector<int64_t> orow;     // n+1 (rank space)
  std::vector<int32_t> oadj;     // m
  int32_t max_out_degree = 0;
  // k-independent predictor features per vertex (6 per vertex), for cliques and motifs
  std::vector<float> feat[2];
  // padded device layout of the CSRs (0: undirected, 1: degree-ordered DAG), built on the
  // first upload and kept, so uploading the graph again is a plain copy
  std::vector<int32_t> pad_row[2], pad_deg[2], pad_adj[2];
  // device-independent task orders and clique-index layout, computed once and kept with the
  // graph for the same reason
  std::vector<int32_t> deg_order;     // ranks by descending DAG out-degree (stable in rank)
  std::vector<int64_t> cnt_ge;        // cnt_ge[d] = ranks with out-degree >= d
  std::vector<uint32_t> idx_boff;     // clique-index block offset per rank (16-byte units)
  std::vector<int32_t> idx_desc;      // task list of deg_order on the index, 4 ints per entry
                                      // (kept until the clique image holds it)
  std::vector<uint8_t> img;           // clique image: padded oriented CSR, order, index tables
  size_t img_off[6] = {0, 0, 0, 0, 0, 0};
  size_t img_adj_ints = 0;            // ints of the padded oriented adjacency
  int32_t idx_extra = 0;              // entries beyond one per root (roots split into parts)
  uint64_t idx_units = 0;             // 16-byte units of the whole index
  int32_t idx_maxd = 0;               // largest out-degree with a block
  std::vector<int32_t> up_order;      // motif roots by descending upper degree
  std::vector<void*> pinned;          // host arrays registered with the CUDA driver
  // device copies
  std::mutex mu;
  std::vector<dmb::DeviceGraph*> dev;
};

struct dm_dictionary {
  uint64_t uid = 0;                      // unique per dictionary object (device table cache key)
  int32_t k = 0;
  int64_t n_quicks = 0;
  int32_t n_classes = 0;
  std::vector<int32_t> quick_to_class;   // n_quicks
  std::vector<uint64_t> class_code;      // n_classes
  std::vector<uint8_t> connected;        // n_classes
};

namespace dmb {
// graph construction helpers (graph.cpp)
int build_graph_from_pairs(std::vector<uint64_t>& keys, int32_t n_vertices, int64_t self_loops,
                           int64_t input_pairs, dm_graph** out);
void ensure_oriented(dm_graph* g);
// device helpers (engine.cu)
void release_device_graphs(dm_graph* g);
void unpin_host_arrays(dm_graph* g);
}  // namespace dmb
