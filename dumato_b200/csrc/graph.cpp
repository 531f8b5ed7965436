// Host-side graph store: edgelist parsing, seeded generators, CSR build and the
// degree-ordered orientation used by the clique engine.
//
// Input semantics follow the reference reader (src/main/Graph.cpp:17-75): whitespace
// separated "src dst" integer pairs, undirected, duplicates and reverse duplicates merged,
// every id in [0, max id] kept as a vertex (isolated ones too). The reference stores
// self-loops in its adjacency sets; they never take part in a count there (every
// extension is filtered by "> v"), so they are dropped here and only counted.
#include <algorithm>
#include <atomic>
#include <thread>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <numeric>

#include "dm_internal.hpp"

namespace dmb {

static thread_local std::string g_last_error;

void set_error(const std::string& msg) { g_last_error = msg; }
int fail(int status, const std::string& msg) {
  g_last_error = msg;
  return status;
}

static uint64_t splitmix64(uint64_t& x) {
  uint64_t z = (x += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

Rng::Rng(uint64_t seed) {
  uint64_t x = seed;
  for (int i = 0; i < 4; ++i) s[i] = splitmix64(x);
}

static inline uint64_t rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }

uint64_t Rng::next() {
  const uint64_t result = rotl(s[1] * 5, 7) * 9;
  const uint64_t t = s[1] << 17;
  s[2] ^= s[0];
  s[3] ^= s[1];
  s[1] ^= s[2];
  s[0] ^= s[3];
  s[2] ^= t;
  s[3] = rotl(s[3], 45);
  return result;
}

double Rng::uniform() { return (double)(next() >> 11) * (1.0 / 9007199254740992.0); }

uint64_t Rng::below(uint64_t bound) {
  // Lemire's multiply-shift with rejection
  uint64_t x = next();
  __uint128_t mprod = (__uint128_t)x * bound;
  uint64_t l = (uint64_t)mprod;
  if (l < bound) {
    uint64_t t = (0 - bound) % bound;
    while (l < t) {
      x = next();
      mprod = (__uint128_t)x * bound;
      l = (uint64_t)mprod;
    }
  }
  return (uint64_t)(mprod >> 64);
}

static inline uint64_t edge_key(uint32_t u, uint32_t v) {
  return u < v ? ((uint64_t)u << 32) | v : ((uint64_t)v << 32) | u;
}

// Open-addressing set of undirected edge keys, used by the generators so that the
// stopping point ("m distinct edges") is reached in a deterministic draw order.
struct EdgeSet {
  std::vector<uint64_t> slots;
  uint64_t mask = 0;
  int64_t size = 0;
  explicit EdgeSet(int64_t expected) {
    uint64_t cap = 1024;
    while (cap < (uint64_t)expected * 2 + 16) cap <<= 1;
    slots.assign(cap, ~0ull);
    mask = cap - 1;
  }
  bool insert(uint64_t key) {
    uint64_t h = key * 0x9E3779B97F4A7C15ull;
    uint64_t i = (h ^ (h >> 29)) & mask;
    while (true) {
      if (slots[i] == ~0ull) {
        slots[i] = key;
        ++size;
        return true;
      }
      if (slots[i] == key) return false;
      i = (i + 1) & mask;
    }
  }
  std::vector<uint64_t> keys() const {
    std::vector<uint64_t> out;
    out.reserve(size);
    for (uint64_t k : slots)
      if (k != ~0ull) out.push_back(k);
    return out;
  }
};

int build_graph_from_pairs(std::vector<uint64_t>& keys, int32_t n_vertices, int64_t self_loops,
                           int64_t input_pairs, dm_graph** out) {
  std::sort(keys.begin(), keys.end());
  keys.erase(std::unique(keys.begin(), keys.end()), keys.end());
  if ((int64_t)keys.size() * 2 >= (int64_t)INT32_MAX)
    return fail(DM_EOVERFLOW, "graph has too many edges for 32-bit device offsets");
  dm_graph* g = new (std::nothrow) dm_graph();
  if (!g) return fail(DM_ENOMEM, "out of host memory");
  g->n = n_vertices;
  g->m = (int64_t)keys.size();
  g->self_loops = self_loops;
  g->input_pairs = input_pairs;
  g->row.assign((size_t)n_vertices + 1, 0);
  for (uint64_t k : keys) {
    uint32_t u = (uint32_t)(k >> 32), v = (uint32_t)k;
    g->row[u + 1]++;
    g->row[v + 1]++;
  }
  for (int32_t i = 0; i < n_vertices; ++i) g->row[i + 1] += g->row[i];
  g->adj.resize((size_t)g->m * 2);
  std::vector<int64_t> fill(g->row.begin(), g->row.end() - 1);
  // keys are sorted by (min, max): appending in this order leaves every row sorted
  for (uint64_t k : keys) {
    uint32_t u = (uint32_t)(k >> 32), v = (uint32_t)k;
    g->adj[fill[u]++] = (int32_t)v;
    g->adj[fill[v]++] = (int32_t)u;
  }
  int32_t md = 0;
  for (int32_t i = 0; i < n_vertices; ++i) md = std::max<int32_t>(md, (int32_t)(g->row[i + 1] - g->row[i]));
  g->max_degree = md;
  *out = g;
  return DM_OK;
}

// Degree-ordered orientation: rank vertices by (degree, id) ascending and keep the arc
// u -> v iff rank(u) < rank(v). Every k-clique then has exactly one lowest-ranked vertex,
// whose out-neighbourhood contains the other k-1 vertices, and out-degrees are bounded by
// O(sqrt(m)).
void ensure_oriented(dm_graph* g) {
  if (g->oriented_built) return;
  const int32_t n = g->n;
  std::vector<int32_t> order(n);
  {
    // counting sort by degree, stable in id
    std::vector<int64_t> cnt((size_t)g->max_degree + 2, 0);
    for (int32_t v = 0; v < n; ++v) cnt[g->row[v + 1] - g->row[v] + 1]++;
    for (size_t d = 1; d < cnt.size(); ++d) cnt[d] += cnt[d - 1];
    for (int32_t v = 0; v < n; ++v) order[cnt[g->row[v + 1] - g->row[v]]++] = v;
  }
  g->rank.assign(n, 0);
  for (int32_t r = 0; r < n; ++r) g->rank[order[r]] = r;
  g->orow.assign((size_t)n + 1, 0);
  for (int32_t v = 0; v < n; ++v) {
    int32_t rv = g->rank[v];
    for (int64_t e = g->row[v]; e < g->row[v + 1]; ++e)
      if (g->rank[g->adj[e]] > rv) g->orow[rv + 1]++;
  }
  for (int32_t r = 0; r < n; ++r) g->orow[r + 1] += g->orow[r];
  g->oadj.resize((size_t)g->m);
  int32_t mo = 0;
  for (int32_t r = 0; r < n; ++r) {
    int32_t v = order[r];
    int64_t pos = g->orow[r];
    for (int64_t e = g->row[v]; e < g->row[v + 1]; ++e) {
      int32_t ru = g->rank[g->adj[e]];
      if (ru > r) g->oadj[pos++] = ru;
    }
    std::sort(g->oadj.begin() + g->orow[r], g->oadj.begin() + g->orow[r + 1]);
    mo = std::max<int32_t>(mo, (int32_t)(g->orow[r + 1] - g->orow[r]));
  }
  g->max_out_degree = mo;
  g->oriented_built = true;
}

static int gen_er(const dm_gen_params& p, std::vector<uint64_t>& keys, int64_t& drawn) {
  if (p.n < 2) return fail(DM_EINVAL, "ER generator needs n >= 2");
  double maxm = (double)p.n * (p.n - 1) / 2.0;
  if ((double)p.m > maxm) return fail(DM_EINVAL, "ER generator: m exceeds n(n-1)/2");
  Rng rng(p.seed);
  EdgeSet set(p.m);
  drawn = 0;
  while (set.size < p.m) {
    uint32_t u = (uint32_t)rng.below(p.n), v = (uint32_t)rng.below(p.n);
    ++drawn;
    if (u == v) continue;
    set.insert(edge_key(u, v));
  }
  keys = set.keys();
  return DM_OK;
}

// Chung-Lu by ball dropping: both endpoints drawn independently with probability
// proportional to w_i = dmax * (1 + i/i0)^(-1/(gamma-1)); i0 is chosen so that
// sum(w) = 2m. Self-loops and repeats are redrawn until m distinct edges exist.
static int gen_chung_lu(const dm_gen_params& p, std::vector<uint64_t>& keys, int64_t& drawn) {
  if (p.n < 2 || p.gamma <= 1.0 || p.dmax < 1.0) return fail(DM_EINVAL, "Chung-Lu: need n >= 2, gamma > 1, dmax >= 1");
  const double alpha = 1.0 / (p.gamma - 1.0);
  const double target = 2.0 * (double)p.m / p.dmax;  // sum of (1 + i/i0)^-alpha wanted
  if (target > p.n) return fail(DM_EINVAL, "Chung-Lu: m too large for n and dmax");
  auto total = [&](double i0) {
    double s = 0;
    for (int32_t i = 0; i < p.n; ++i) s += std::pow(1.0 + i / i0, -alpha);
    return s;
  };
  double lo = 1e-6, hi = 1e12;
  for (int it = 0; it < 200; ++it) {
    double mid = std::sqrt(lo * hi);
    if (total(mid) < target) lo = mid; else hi = mid;
  }
  const double i0 = std::sqrt(lo * hi);
  std::vector<double> cdf(p.n);
  double acc = 0;
  for (int32_t i = 0; i < p.n; ++i) {
    acc += std::pow(1.0 + i / i0, -alpha);
    cdf[i] = acc;
  }
  const double maxpairs = (double)p.n * (p.n - 1) / 2.0;
  if ((double)p.m > 0.5 * maxpairs) return fail(DM_EINVAL, "Chung-Lu: m too dense");
  Rng rng(p.seed);
  EdgeSet set(p.m);
  drawn = 0;
  const int64_t max_draws = p.m * 200 + 1000000;
  auto pick = [&]() {
    double x = rng.uniform() * acc;
    return (uint32_t)(std::upper_bound(cdf.begin(), cdf.end(), x) - cdf.begin());
  };
  while (set.size < p.m) {
    if (drawn > max_draws) return fail(DM_EINVAL, "Chung-Lu: could not reach m distinct edges");
    uint32_t u = pick(), v = pick();
    ++drawn;
    if (u >= (uint32_t)p.n) u = p.n - 1;
    if (v >= (uint32_t)p.n) v = p.n - 1;
    if (u == v) continue;
    set.insert(edge_key(u, v));
  }
  keys = set.keys();
  return DM_OK;
}

// R-MAT: each edge descends log2 levels choosing quadrant a/b/c/d. Ids >= n are trimmed,
// self-loops and repeats dropped, until m distinct edges; then the touched ids are
// relabelled compactly to [0, V) by a seeded random permutation (so hubs do not sit at
// the lowest ids).
static int gen_rmat(const dm_gen_params& p, std::vector<uint64_t>& keys, int64_t& drawn, int32_t& n_out) {
  if (p.n < 2) return fail(DM_EINVAL, "R-MAT: need n >= 2");
  double d = 1.0 - p.a - p.b - p.c;
  if (p.a <= 0 || p.b < 0 || p.c < 0 || d < 0) return fail(DM_EINVAL, "R-MAT: bad quadrant probabilities");
  int scale = 1;
  while ((1ll << scale) < p.n) ++scale;
  Rng rng(p.seed);
  EdgeSet set(p.m);
  drawn = 0;
  const int64_t max_draws = p.m * 1000 + 1000000;
  const double ab = p.a + p.b, abc = p.a + p.b + p.c;
  while (set.size < p.m) {
    if (drawn > max_draws) return fail(DM_EINVAL, "R-MAT: could not reach m distinct edges");
    uint32_t u = 0, v = 0;
    for (int l = 0; l < scale; ++l) {
      double r = rng.uniform();
      uint32_t bu = 0, bv = 0;
      if (r < p.a) {
      } else if (r < ab) {
        bv = 1;
      } else if (r < abc) {
        bu = 1;
      } else {
        bu = 1;
        bv = 1;
      }
      u = (u << 1) | bu;
      v = (v << 1) | bv;
    }
    ++drawn;
    if (u == v || u >= (uint32_t)p.n || v >= (uint32_t)p.n) continue;
    set.insert(edge_key(u, v));
  }
  keys = set.keys();
  // compact relabel of touched ids by a random permutation
  std::vector<int32_t> touched(p.n, 0);
  for (uint64_t k : keys) {
    touched[k >> 32] = 1;
    touched[(uint32_t)k] = 1;
  }
  std::vector<int32_t> ids;
  for (int32_t i = 0; i < p.n; ++i)
    if (touched[i]) ids.push_back(i);
  const int32_t V = (int32_t)ids.size();
  std::vector<int32_t> perm(V);
  std::iota(perm.begin(), perm.end(), 0);
  for (int32_t i = V - 1; i > 0; --i) std::swap(perm[i], perm[rng.below((uint64_t)i + 1)]);
  std::vector<int32_t> newid(p.n, -1);
  for (int32_t i = 0; i < V; ++i) newid[ids[i]] = perm[i];
  for (uint64_t& k : keys) k = edge_key((uint32_t)newid[k >> 32], (uint32_t)newid[(uint32_t)k]);
  n_out = V;
  return DM_OK;
}

}  // namespace dmb

using namespace dmb;

extern "C" {

int dm_abi_version(void) { return DM_ABI_VERSION; }

const char* dm_last_error(void) { return g_last_error.c_str(); }

int dm_graph_from_edges(const int32_t* src, const int32_t* dst, int64_t n_pairs, int32_t n_vertices,
                        dm_graph** out) {
  if (!out || n_pairs < 0 || (n_pairs > 0 && (!src || !dst))) return fail(DM_EINVAL, "dm_graph_from_edges: bad arguments");
  std::vector<uint64_t> keys;
  keys.reserve((size_t)n_pairs);
  int64_t loops = 0;
  int32_t maxid = -1;
  for (int64_t i = 0; i < n_pairs; ++i) {
    int32_t u = src[i], v = dst[i];
    if (u < 0 || v < 0) return fail(DM_EFORMAT, "dm_graph_from_edges: negative vertex id");
    maxid = std::max(maxid, std::max(u, v));
    if (u == v) {
      ++loops;
      continue;
    }
    keys.push_back(edge_key((uint32_t)u, (uint32_t)v));
  }
  int32_t n = std::max(n_vertices, maxid + 1);
  return build_graph_from_pairs(keys, n, loops, n_pairs, out);
}

int dm_graph_load_edgelist(const char* path, dm_graph** out) {
  if (!path || !out) return fail(DM_EINVAL, "dm_graph_load_edgelist: null argument");
  FILE* fp = std::fopen(path, "rb");
  if (!fp) return fail(DM_EIO, std::string("cannot open edgelist ") + path);
  std::fseek(fp, 0, SEEK_END);
  long size = std::ftell(fp);
  std::fseek(fp, 0, SEEK_SET);
  std::vector<char> buf((size_t)std::max<long>(size, 0) + 1);
  size_t got = std::fread(buf.data(), 1, (size_t)size, fp);
  std::fclose(fp);
  buf[got] = 0;
  std::vector<uint64_t> keys;
  keys.reserve(got / 6 + 16);
  int64_t loops = 0, pairs = 0;
  int64_t maxid = -1;
  const char* c = buf.data();
  const char* end = c + got;
  int64_t vals[2];
  int nv = 0;
  while (c < end) {
    char ch = *c;
    if (ch == '#' || ch == '%') {  // comment line (an extension: the reference has none)
      while (c < end && *c != '\n') ++c;
      continue;
    }
    if (ch == ' ' || ch == '\t' || ch == '\r' || ch == '\n' || ch == ',') {
      ++c;
      continue;
    }
    if (ch == '-') return fail(DM_EFORMAT, std::string("negative vertex id in ") + path);
    if (ch < '0' || ch > '9') return fail(DM_EFORMAT, std::string("non-integer token in ") + path);
    int64_t x = 0;
    while (c < end && *c >= '0' && *c <= '9') {
      x = x * 10 + (*c - '0');
      if (x > INT32_MAX - 1) return fail(DM_EFORMAT, std::string("vertex id out of int32 range in ") + path);
      ++c;
    }
    vals[nv++] = x;
    if (nv == 2) {
      nv = 0;
      ++pairs;
      maxid = std::max(maxid, std::max(vals[0], vals[1]));
      if (vals[0] == vals[1]) {
        ++loops;
      } else {
        keys.push_back(edge_key((uint32_t)vals[0], (uint32_t)vals[1]));
      }
    }
  }
  if (nv != 0) return fail(DM_EFORMAT, std::string("odd number of ids in ") + path);
  return build_graph_from_pairs(keys, (int32_t)(maxid + 1), loops, pairs, out);
}

int dm_graph_generate(const dm_gen_params* p, dm_graph** out) {
  if (!p || !out || p->m < 0) return fail(DM_EINVAL, "dm_graph_generate: bad arguments");
  std::vector<uint64_t> keys;
  int64_t drawn = 0;
  int32_t n = p->n;
  int rc;
  switch (p->kind) {
    case DM_GEN_ER: rc = gen_er(*p, keys, drawn); break;
    case DM_GEN_CHUNG_LU: rc = gen_chung_lu(*p, keys, drawn); break;
    case DM_GEN_RMAT: rc = gen_rmat(*p, keys, drawn, n); break;
    default: return fail(DM_EINVAL, "dm_graph_generate: unknown generator kind");
  }
  if (rc != DM_OK) return rc;
  return build_graph_from_pairs(keys, n, 0, drawn, out);
}

int dm_graph_info_get(const dm_graph* gc, dm_graph_info* info) {
  if (!gc || !info) return fail(DM_EINVAL, "dm_graph_info_get: null argument");
  dm_graph* g = const_cast<dm_graph*>(gc);
  {
    std::lock_guard<std::mutex> lk(g->mu);
    ensure_oriented(g);
  }
  info->n_vertices = g->n;
  info->n_edges = g->m;
  info->max_degree = g->max_degree;
  info->max_out_degree = g->max_out_degree;
  info->n_self_loops = g->self_loops;
  info->n_input_pairs = g->input_pairs;
  return DM_OK;
}

int dm_graph_edges(const dm_graph* g, int32_t* u, int32_t* v) {
  if (!g || (!u && g->m) || (!v && g->m)) return fail(DM_EINVAL, "dm_graph_edges: null argument");
  int64_t pos = 0;
  for (int32_t x = 0; x < g->n; ++x)
    for (int64_t e = g->row[x]; e < g->row[x + 1]; ++e)
      if (g->adj[e] > x) {
        u[pos] = x;
        v[pos] = g->adj[e];
        ++pos;
      }
  return DM_OK;
}

int dm_graph_csr(const dm_graph* g, int64_t* offsets, int32_t* adjacency) {
  if (!g || !offsets || (!adjacency && g->m)) return fail(DM_EINVAL, "dm_graph_csr: null argument");
  std::memcpy(offsets, g->row.data(), sizeof(int64_t) * (g->n + 1));
  if (g->m) std::memcpy(adjacency, g->adj.data(), sizeof(int32_t) * g->adj.size());
  return DM_OK;
}

int dm_graph_write_edgelist(const dm_graph* g, const char* path) {
  if (!g || !path) return fail(DM_EINVAL, "dm_graph_write_edgelist: null argument");
  FILE* fp = std::fopen(path, "w");
  if (!fp) return fail(DM_EIO, std::string("cannot write ") + path);
  for (int32_t x = 0; x < g->n; ++x)
    for (int64_t e = g->row[x]; e < g->row[x + 1]; ++e)
      if (g->adj[e] > x) std::fprintf(fp, "%d %d\n", x, g->adj[e]);
  // keep isolated top ids: the reference derives V from the max id seen
  if (g->n > 0 && g->row[g->n] == g->row[g->n - 1]) std::fprintf(fp, "%d %d\n", g->n - 1, g->n - 1);
  std::fclose(fp);
  return DM_OK;
}

int dm_clique_work_model(dm_graph* g, int32_t k, uint64_t* nodes_out, uint64_t* bytes_out) {
  if (!g || !nodes_out || !bytes_out) return fail(DM_EINVAL, "dm_clique_work_model: null argument");
  if (k < 2 || k > 12) return fail(DM_EINVAL, "dm_clique_work_model: k must be in [2, 12]");
  {
    std::lock_guard<std::mutex> lk(g->mu);
    ensure_oriented(g);
  }
  const int32_t n = g->n;
  uint64_t nodes = 0, bytes = 0;
  const size_t cap = (size_t)g->max_out_degree + 1;
  std::vector<int32_t> buf(cap * k);
  std::vector<int32_t*> C(k);
  std::vector<int32_t> nC(k), pos(k);
  for (int i = 0; i < k; ++i) C[i] = buf.data() + (size_t)i * cap;
  for (int32_t r = 0; r < n; ++r) {
    const int32_t na = (int32_t)(g->orow[r + 1] - g->orow[r]);
    std::copy(g->oadj.begin() + g->orow[r], g->oadj.begin() + g->orow[r + 1], C[0]);
    nC[0] = na;
    ++nodes;
    bytes += 8ull * (uint64_t)na;
    if (k == 2) continue;
    int l = 0;
    pos[0] = 0;
    while (l >= 0) {
      if (l == k - 2 || pos[l] >= nC[l]) {
        --l;
        continue;
      }
      const int32_t v = C[l][pos[l]++];
      const int32_t* B = g->oadj.data() + g->orow[v];
      const int32_t nb = (int32_t)(g->orow[v + 1] - g->orow[v]);
      int32_t i = pos[l], j = 0, m = 0;
      while (i < nC[l] && j < nb) {
        if (C[l][i] < B[j]) ++i;
        else if (C[l][i] > B[j]) ++j;
        else {
          C[l + 1][m++] = C[l][i];
          ++i;
          ++j;
        }
      }
      ++nodes;
      bytes += 4ull * ((uint64_t)nC[l] + (uint64_t)nb) + 4ull * (uint64_t)m;
      ++l;
      nC[l] = m;
      pos[l] = 0;
    }
  }
  *nodes_out = nodes;
  *bytes_out = bytes;
  return DM_OK;
}

// Work model of the motif path (host-side accounting for the roofline; it counts nothing):
// the DFS of the reference's motif driver visits, below every root v0, the canonical
// prefixes (v_0..v_t), t <= k-2, whose extension step reads the adjacency rows of the
// prefix and writes the deduplicated union above v0 with its sources (extend(0,k),
// DuMatoGPU.cu:1702-1721): 4 sum_i deg(v_i) + 8 |union| bytes; each leaf candidate of the
// last level costs 4(k-1) + 8 (its adjacency probes and the dictionary read,
// aggregate_pattern 930-967). Only internal prefixes are walked: with U_t the union and
// E_t the valid extensions, taking w from E_t gives excl(w) = N(w) above v0 outside U_t,
// U_{t+1} = U_t + excl(w) and E_{t+1} = {e in E_t : e > w} + excl(w), and the leaves of a
// last-level prefix are |E_{k-2}|.
namespace {

struct MotifModel {
  const dm_graph* g;
  int k;
  std::vector<int32_t> mark;     // 1 + depth at which a vertex joined U (0 = not in U)
  std::vector<int32_t> ebuf;     // E_t per level
  std::vector<int32_t> xbuf;     // excl per level
  size_t cap;
  uint64_t nodes = 0, bytes = 0;

  int32_t deg(int32_t v) const { return (int32_t)(g->row[v + 1] - g->row[v]); }

  void visit(int32_t v0, int t, const int32_t* E, int32_t nE, uint64_t degsum, uint64_t usize) {
    ++nodes;
    bytes += 4 * degsum + 8 * usize;
    if (t == k - 2) {
      bytes += (uint64_t)nE * (4ull * (uint64_t)(k - 1) + 8ull);
      return;
    }
    int32_t* X = xbuf.data() + (size_t)(t + 1) * cap;
    int32_t* En = ebuf.data() + (size_t)(t + 1) * cap;
    for (int32_t i = 0; i < nE; ++i) {
      const int32_t w = E[i];
      int32_t nx = 0;
      for (int64_t e = g->row[w]; e < g->row[w + 1]; ++e) {
        const int32_t x = g->adj[e];
        if (x > v0 && mark[x] == 0) {
          mark[x] = t + 2;
          X[nx++] = x;
        }
      }
      // E_{t+1}: members of E_t above w, then excl(w), merged in id order
      std::sort(X, X + nx);
      int32_t m = 0, a = 0, b = 0;
      const int32_t* S = E + i + 1;  // E_t is id-sorted: the members above w are its suffix
      const int32_t ns = nE - i - 1;
      while (a < ns || b < nx) {
        if (b >= nx || (a < ns && S[a] < X[b])) En[m++] = S[a++];
        else En[m++] = X[b++];
      }
      visit(v0, t + 1, En, m, degsum + (uint64_t)deg(w), usize + (uint64_t)nx);
      for (int32_t j = 0; j < nx; ++j) mark[X[j]] = 0;
    }
  }
};

}  // namespace

int dm_motif_work_model(dm_graph* g, int32_t k, uint64_t* nodes_out, uint64_t* bytes_out) {
  if (!g || !nodes_out || !bytes_out) return fail(DM_EINVAL, "dm_motif_work_model: null argument");
  if (k < 3 || k > 7) return fail(DM_EINVAL, "dm_motif_work_model: k must be in [3, 7]");
  const int32_t n = g->n;
  const unsigned nt = std::max(1u, std::min(64u, std::thread::hardware_concurrency()));
  std::vector<uint64_t> tn(nt, 0), tb(nt, 0);
  std::atomic<int32_t> next{0};
  auto work = [&](unsigned id) {
    MotifModel M;
    M.g = g;
    M.k = k;
    M.mark.assign((size_t)std::max(n, 1), 0);
    M.cap = (size_t)g->max_degree * (size_t)(k - 1) + 1;
    M.ebuf.assign(M.cap * (size_t)k, 0);
    M.xbuf.assign(M.cap * (size_t)k, 0);
    while (true) {
      const int32_t v0 = next.fetch_add(1);
      if (v0 >= n) break;
      int32_t* E0 = M.ebuf.data();
      int32_t n0 = 0;
      for (int64_t e = g->row[v0]; e < g->row[v0 + 1]; ++e) {
        const int32_t x = g->adj[e];
        if (x > v0) {
          E0[n0++] = x;
          M.mark[x] = 1;
        }
      }
      M.visit(v0, 0, E0, n0, (uint64_t)M.deg(v0), (uint64_t)n0);
      for (int32_t j = 0; j < n0; ++j) M.mark[E0[j]] = 0;
    }
    tn[id] = M.nodes;
    tb[id] = M.bytes;
  };
  std::vector<std::thread> th;
  for (unsigned i = 1; i < nt; ++i) th.emplace_back(work, i);
  work(0);
  for (auto& t : th) t.join();
  uint64_t nodes = 0, bytes = 0;
  for (unsigned i = 0; i < nt; ++i) {
    nodes += tn[i];
    bytes += tb[i];
  }
  *nodes_out = nodes;
  *bytes_out = bytes;
  return DM_OK;
}

void dm_graph_free(dm_graph* g) {
  if (!g) return;
  release_device_graphs(g);
  unpin_host_arrays(g);
  delete g;
}

}  // extern "C"
