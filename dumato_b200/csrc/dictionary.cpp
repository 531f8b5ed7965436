// Canonical-class dictionaries for motif counting: quick code -> class id.
//
// Quick-code layout (the reference's incremental induction code, src/main/DuMatoGPU.cu:846-869
// and 930-967; generator src/motifs_DM_DFS/Manager.cpp:1069-1088): vertices are numbered in
// enumeration order 0..k-1, the edge (0,1) is implicit, and vertex p >= 2 owns the bits
// [(p-2)(p+1)/2, (p-2)(p+1)/2 + p), bit j meaning an edge (j, p). A k-vertex code has
// k(k-1)/2 - 1 bits.
//
// The reference built its tables offline with nauty. Here every class is generated from
// first principles: the orbit of a labelled graph under all k! relabellings is walked, every
// quick code in the orbit gets the same class, and the class's global code is the maximum,
// over the orbit, of the adjacency code with pairs (0,1),(0,2),..,(0,k-1),(1,2),..,(k-2,k-1)
// from the most significant bit down. Class ids are the ranks of these codes (ascending),
// which is how the reference numbers cg_local against its own cg_global. For k <= 4 the
// max-code equals nauty's canonical code, so the tables are identical to the reference's;
// for k >= 5 the partition of quick codes is identical and only the id order may differ.
#include <algorithm>
#include <atomic>
#include <cstdio>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include "dm_internal.hpp"

namespace dmb {

static inline int quick_bits(int k) { return k * (k - 1) / 2 - 1; }

static std::atomic<uint64_t> g_dict_uid{1};

// adjacency as k row bitmasks
struct Small {
  uint8_t row[8];
};

static Small graph_of_quick(int k, uint64_t q) {
  Small s;
  std::memset(&s, 0, sizeof(s));
  s.row[0] |= 2;
  s.row[1] |= 1;
  for (int p = 2; p < k; ++p) {
    int off = (p - 2) * (p + 1) / 2;
    for (int j = 0; j < p; ++j)
      if ((q >> (off + j)) & 1) {
        s.row[p] |= (uint8_t)(1u << j);
        s.row[j] |= (uint8_t)(1u << p);
      }
  }
  return s;
}

static uint64_t full_code(int k, const Small& s) {
  uint64_t c = 0;
  for (int a = 0; a < k; ++a)
    for (int b = a + 1; b < k; ++b) c = (c << 1) | ((s.row[a] >> b) & 1);
  return c;
}

static bool quick_of_graph(int k, const Small& s, uint64_t& q) {
  if (!((s.row[0] >> 1) & 1)) return false;
  q = 0;
  for (int p = 2; p < k; ++p) {
    int off = (p - 2) * (p + 1) / 2;
    for (int j = 0; j < p; ++j)
      if ((s.row[p] >> j) & 1) q |= 1ull << (off + j);
  }
  return true;
}

static bool connected_small(int k, const Small& s) {
  uint32_t seen = 1, frontier = 1;
  while (frontier) {
    uint32_t next = 0;
    for (int v = 0; v < k; ++v)
      if ((frontier >> v) & 1) next |= s.row[v];
    next &= ~seen;
    seen |= next;
    frontier = next;
  }
  return seen == (1u << k) - 1;
}

static void fill_connected(dm_dictionary* d) {
  d->connected.assign(d->n_classes, 0);
  std::vector<char> done(d->n_classes, 0);
  for (int64_t q = 0; q < d->n_quicks; ++q) {
    int c = d->quick_to_class[q];
    if (c < 0 || c >= d->n_classes || done[c]) continue;
    done[c] = 1;
    d->connected[c] = connected_small(d->k, graph_of_quick(d->k, (uint64_t)q)) ? 1 : 0;
  }
}

}  // namespace dmb

using namespace dmb;

extern "C" {

int dm_dictionary_generate(int32_t k, dm_dictionary** out) {
  if (!out) return fail(DM_EINVAL, "dm_dictionary_generate: null argument");
  if (k < 3 || k > 7) return fail(DM_EINVAL, "dm_dictionary_generate: k must be in [3, 7]");
  const int B = quick_bits(k);
  const int64_t nq = 1ll << B;
  std::vector<int> perm(k);
  for (int i = 0; i < k; ++i) perm[i] = i;
  std::vector<std::vector<int>> perms;
  do perms.push_back(perm);
  while (std::next_permutation(perm.begin(), perm.end()));

  std::vector<int32_t> orbit_of(nq, -1);  // temporary class = discovery index
  std::vector<uint64_t> orbit_code;
  for (int64_t q = 0; q < nq; ++q) {
    if (orbit_of[q] >= 0) continue;
    const int32_t id = (int32_t)orbit_code.size();
    Small g = graph_of_quick(k, (uint64_t)q);
    uint64_t best = 0;
    for (const auto& p : perms) {
      Small h;
      std::memset(&h, 0, sizeof(h));
      for (int a = 0; a < k; ++a)
        for (int b = 0; b < k; ++b)
          if ((g.row[a] >> b) & 1) h.row[p[a]] |= (uint8_t)(1u << p[b]);
      best = std::max(best, full_code(k, h));
      uint64_t qq;
      if (quick_of_graph(k, h, qq)) orbit_of[qq] = id;
    }
    orbit_code.push_back(best);
  }
  // class id = rank of the canonical code
  const int32_t nc = (int32_t)orbit_code.size();
  std::vector<int32_t> order(nc);
  for (int32_t i = 0; i < nc; ++i) order[i] = i;
  std::sort(order.begin(), order.end(), [&](int32_t x, int32_t y) { return orbit_code[x] < orbit_code[y]; });
  std::vector<int32_t> rank_of(nc);
  for (int32_t r = 0; r < nc; ++r) rank_of[order[r]] = r;
  dm_dictionary* d = new (std::nothrow) dm_dictionary();
  if (!d) return fail(DM_ENOMEM, "out of host memory");
  d->uid = g_dict_uid++;
  d->k = k;
  d->n_quicks = nq;
  d->n_classes = nc;
  d->quick_to_class.resize(nq);
  for (int64_t q = 0; q < nq; ++q) d->quick_to_class[q] = rank_of[orbit_of[q]];
  d->class_code.resize(nc);
  for (int32_t r = 0; r < nc; ++r) d->class_code[r] = orbit_code[order[r]];
  fill_connected(d);
  *out = d;
  return DM_OK;
}

// Reads the reference's dictionary CSV (src/main/QuickMapping.cpp:24-40 reads the first two
// blocks; the third block, per-class quick lists, is optional here as it is there).
int dm_dictionary_load_csv(const char* path, dm_dictionary** out) {
  if (!path || !out) return fail(DM_EINVAL, "dm_dictionary_load_csv: null argument");
  FILE* fp = std::fopen(path, "r");
  if (!fp) return fail(DM_EIO, std::string("cannot open dictionary ") + path);
  char line[256];
  auto next_line = [&](std::string& s) -> bool {
    while (std::fgets(line, sizeof line, fp)) {
      s = line;
      while (!s.empty() && (s.back() == '\n' || s.back() == '\r' || s.back() == ' ')) s.pop_back();
      if (!s.empty()) return true;
    }
    return false;
  };
  std::string s;
  auto bad = [&](const char* what) {
    std::fclose(fp);
    return fail(DM_EFORMAT, std::string("malformed dictionary ") + path + ": " + what);
  };
  if (!next_line(s) || s[0] != '#') return bad("missing #quick header");
  if (!next_line(s)) return bad("missing quick count");
  long long nq = std::atoll(s.c_str());
  int k = 0;
  for (int kk = 3; kk <= 7; ++kk)
    if ((1ll << quick_bits(kk)) == nq) k = kk;
  if (!k) return bad("quick count is not 2^(k(k-1)/2-1) for k in [3,7]");
  dm_dictionary* d = new dm_dictionary();
  d->uid = g_dict_uid++;
  d->k = k;
  d->n_quicks = nq;
  d->quick_to_class.assign(nq, -1);
  for (long long i = 0; i < nq; ++i) {
    long long q, c;
    if (!next_line(s) || std::sscanf(s.c_str(), "%lld,%lld", &q, &c) != 2 || q < 0 || q >= nq || c < 0) {
      delete d;
      return bad("bad quick line");
    }
    d->quick_to_class[q] = (int32_t)c;
  }
  if (!next_line(s) || s[0] != '#') {
    delete d;
    return bad("missing #cg_local header");
  }
  if (!next_line(s)) {
    delete d;
    return bad("missing class count");
  }
  long long nc = std::atoll(s.c_str());
  if (nc <= 0 || nc > 100000) {
    delete d;
    return bad("bad class count");
  }
  d->n_classes = (int32_t)nc;
  d->class_code.assign(nc, 0);
  for (long long i = 0; i < nc; ++i) {
    long long c;
    unsigned long long g;
    if (!next_line(s) || std::sscanf(s.c_str(), "%lld,%llu", &c, &g) != 2 || c < 0 || c >= nc) {
      delete d;
      return bad("bad class line");
    }
    d->class_code[c] = g;
  }
  std::fclose(fp);
  for (long long q = 0; q < nq; ++q)
    if (d->quick_to_class[q] < 0 || d->quick_to_class[q] >= nc) {
      delete d;
      return fail(DM_EFORMAT, std::string("dictionary ") + path + " leaves a quick code unmapped");
    }
  fill_connected(d);
  *out = d;
  return DM_OK;
}

int dm_dictionary_write_csv(const dm_dictionary* d, const char* path) {
  if (!d || !path) return fail(DM_EINVAL, "dm_dictionary_write_csv: null argument");
  FILE* fp = std::fopen(path, "w");
  if (!fp) return fail(DM_EIO, std::string("cannot write ") + path);
  std::fprintf(fp, "#quick,cg_local\n%lld\n", (long long)d->n_quicks);
  for (int64_t q = 0; q < d->n_quicks; ++q) std::fprintf(fp, "%lld,%d\n", (long long)q, d->quick_to_class[q]);
  std::fprintf(fp, "#cg_local,cg_global\n%d\n", d->n_classes);
  for (int32_t c = 0; c < d->n_classes; ++c) std::fprintf(fp, "%d,%llu\n", c, (unsigned long long)d->class_code[c]);
  std::fprintf(fp, "#cg_local,amount_of_quicks,quicks\n%d\n", d->n_classes);
  std::vector<std::vector<int64_t>> members(d->n_classes);
  for (int64_t q = 0; q < d->n_quicks; ++q) members[d->quick_to_class[q]].push_back(q);
  for (int32_t c = 0; c < d->n_classes; ++c) {
    std::fprintf(fp, "%d,%zu", c, members[c].size());
    for (int64_t q : members[c]) std::fprintf(fp, ",%lld", (long long)q);
    std::fprintf(fp, "\n");
  }
  std::fclose(fp);
  return DM_OK;
}

int dm_dictionary_shape(const dm_dictionary* d, int32_t* k, int64_t* n_quicks, int32_t* n_classes) {
  if (!d) return fail(DM_EINVAL, "dm_dictionary_shape: null dictionary");
  if (k) *k = d->k;
  if (n_quicks) *n_quicks = d->n_quicks;
  if (n_classes) *n_classes = d->n_classes;
  return DM_OK;
}

int dm_dictionary_tables(const dm_dictionary* d, int32_t* quick_to_class, uint64_t* class_code) {
  if (!d) return fail(DM_EINVAL, "dm_dictionary_tables: null dictionary");
  if (quick_to_class) std::memcpy(quick_to_class, d->quick_to_class.data(), sizeof(int32_t) * d->n_quicks);
  if (class_code) std::memcpy(class_code, d->class_code.data(), sizeof(uint64_t) * d->n_classes);
  return DM_OK;
}

int dm_dictionary_connected(const dm_dictionary* d, uint8_t* connected) {
  if (!d || !connected) return fail(DM_EINVAL, "dm_dictionary_connected: null argument");
  std::memcpy(connected, d->connected.data(), d->n_classes);
  return DM_OK;
}

void dm_dictionary_free(dm_dictionary* d) { delete d; }

}  // extern "C"
