/*
 * dm_oracle.c - CPU oracle for the DuMato clique / motif counting path.
 *
 * TEST INFRASTRUCTURE ONLY. This file is the checker and the timed CPU baseline; the
 * product never links, loads or calls it. Only tests/, __graft_entry__.smoke() and the
 * cpu_baseline / reference legs of bench.py use it.
 *
 * What it restates (paths relative to the DuMato project root):
 *   - Graph reading: src/main/Graph.cpp:17-75. fscanf "%d %d" pairs, undirected, std::set
 *     adjacency (sorted, deduplicated, self-loops KEPT as the reference keeps them).
 *   - Plain DFS k-clique counting, the algorithm of src/clique_DM_DFS/clique_DM_DFS.cu:43-75
 *     with src/clique_DM_DFS/DuMato.h:141-253: one task per root (the atomic root counter
 *     becomes an OpenMP dynamic schedule), neighbours walked one by one, an extension
 *     kept when it is > the last vertex and adjacent to every earlier vertex, checked by a
 *     linear adjacency scan (dm_findNeighbourhood2), one increment per k-clique.
 *   - Warp-centric motif counting semantics of src/main/motifs_DM_WCLB.cu:9-36:
 *     extend(0,k) (src/main/DuMatoGPU.cu:1702-1721: union of the prefix adjacencies,
 *     deduplicated, > v0, tagged with the first source), canonicalFilter2 (989-1012:
 *     drop ext if some i in [1,k] has (i > src and ext <= v_i) or (i < src and ext == v_i)),
 *     forward_induce (846-869: quick bits of the new vertex at offset (k-2)(k+1)/2) and
 *     aggregate_pattern (930-967: leaf quick bits at offset (k-1)(k+2)/2, found by linear
 *     scans (findMany), then quickToCgLocal lookup and a histogram increment).
 *   - Brute-force cross-checks (all k-subsets) for tiny graphs.
 *   - The algorithmic byte counts used by the roofline: for cliques on the degree-ordered
 *     DAG, every node computing a candidate set C_child from (C_parent, N+(v)) costs
 *     4(|C_parent| + |N+(v)|) + 4|C_child| bytes (level 0: 4|N+(v0)| + 4|C_0|); for motifs,
 *     every internal node at depth d costs 4 sum_{i<=d} deg(v_i) + 8 |union| and every
 *     leaf candidate 4(d+1) + 8.
 */
#include <omp.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

typedef struct {
  int32_t n;       /* max id + 1 */
  int64_t *off;    /* n+1 */
  int32_t *adj;    /* sorted, unique, self-loops kept */
  int32_t maxdeg;
} og_graph;

static int cmp_u64(const void *a, const void *b) {
  uint64_t x = *(const uint64_t *)a, y = *(const uint64_t *)b;
  return x < y ? -1 : x > y;
}

/* Builds the set-semantics adjacency of Graph.cpp:60-75 from directed pairs. */
static og_graph *build(const int32_t *src, const int32_t *dst, int64_t np) {
  og_graph *g = (og_graph *)calloc(1, sizeof(og_graph));
  int32_t maxid = -1;
  for (int64_t i = 0; i < np; ++i) {
    if (src[i] > maxid) maxid = src[i];
    if (dst[i] > maxid) maxid = dst[i];
  }
  g->n = maxid + 1;
  uint64_t *keys = (uint64_t *)malloc(sizeof(uint64_t) * (size_t)(2 * np + 1));
  int64_t nk = 0;
  for (int64_t i = 0; i < np; ++i) {
    keys[nk++] = ((uint64_t)(uint32_t)src[i] << 32) | (uint32_t)dst[i];
    keys[nk++] = ((uint64_t)(uint32_t)dst[i] << 32) | (uint32_t)src[i];
  }
  qsort(keys, (size_t)nk, sizeof(uint64_t), cmp_u64);
  int64_t u = 0;
  for (int64_t i = 0; i < nk; ++i)
    if (i == 0 || keys[i] != keys[i - 1]) keys[u++] = keys[i];
  g->off = (int64_t *)calloc((size_t)g->n + 1, sizeof(int64_t));
  g->adj = (int32_t *)malloc(sizeof(int32_t) * (size_t)(u + 1));
  for (int64_t i = 0; i < u; ++i) {
    g->off[(keys[i] >> 32) + 1]++;
    g->adj[i] = (int32_t)(uint32_t)keys[i];
  }
  for (int32_t v = 0; v < g->n; ++v) g->off[v + 1] += g->off[v];
  g->maxdeg = 0;
  for (int32_t v = 0; v < g->n; ++v) {
    int32_t d = (int32_t)(g->off[v + 1] - g->off[v]);
    if (d > g->maxdeg) g->maxdeg = d;
  }
  free(keys);
  return g;
}

og_graph *oracle_graph_from_pairs(const int32_t *src, const int32_t *dst, int64_t np) {
  return build(src, dst, np);
}

/* Graph.cpp:17-54: fscanf("%d %d") until EOF. Returns NULL on a malformed file. */
og_graph *oracle_graph_load(const char *path) {
  FILE *fp = fopen(path, "r");
  if (!fp) return NULL;
  int64_t cap = 1 << 16, np = 0;
  int32_t *s = (int32_t *)malloc(sizeof(int32_t) * cap), *d = (int32_t *)malloc(sizeof(int32_t) * cap);
  int a, b, r;
  while ((r = fscanf(fp, "%d %d", &a, &b)) != EOF) {
    if (r != 2 || a < 0 || b < 0) {
      free(s);
      free(d);
      fclose(fp);
      return NULL;
    }
    if (np == cap) {
      cap *= 2;
      s = (int32_t *)realloc(s, sizeof(int32_t) * cap);
      d = (int32_t *)realloc(d, sizeof(int32_t) * cap);
    }
    s[np] = a;
    d[np] = b;
    ++np;
  }
  fclose(fp);
  og_graph *g = build(s, d, np);
  free(s);
  free(d);
  return g;
}

void oracle_graph_free(og_graph *g) {
  if (!g) return;
  free(g->off);
  free(g->adj);
  free(g);
}

int32_t oracle_graph_n(const og_graph *g) { return g->n; }
int32_t oracle_graph_maxdeg(const og_graph *g) { return g->maxdeg; }
/* number of undirected edges without self-loops */
int64_t oracle_graph_m(const og_graph *g) {
  int64_t m = 0;
  for (int32_t v = 0; v < g->n; ++v)
    for (int64_t e = g->off[v]; e < g->off[v + 1]; ++e)
      if (g->adj[e] > v) ++m;
  return m;
}

static inline int lin_find(const og_graph *g, int32_t v, int32_t x) {
  for (int64_t e = g->off[v]; e < g->off[v + 1]; ++e)
    if (g->adj[e] == x) return 1;
  return 0;
}

static inline int bin_find(const og_graph *g, int32_t v, int32_t x) {
  int64_t lo = g->off[v], hi = g->off[v + 1];
  while (lo < hi) {
    int64_t mid = (lo + hi) >> 1;
    if (g->adj[mid] < x) lo = mid + 1; else hi = mid;
  }
  return lo < g->off[v + 1] && g->adj[lo] == x;
}

static int resolve_threads(int threads) { return threads > 0 ? threads : omp_get_max_threads(); }

/* ---------------- plain DFS clique counting (the CPU baseline) ---------------- */

/* One root of clique_DM_DFS.cu:43-75: id[0] = root, walk neighbours of the last vertex,
   keep ext > id[k] adjacent to id[0..k-1] (linear scans), count at size K. */
static uint64_t clique_root(const og_graph *g, int32_t root, int K) {
  int32_t id[32];
  int64_t pos[32];
  uint64_t cnt = 0;
  if (K == 1) return 1;
  int k = 0;
  id[0] = root;
  pos[0] = g->off[root];
  while (k >= 0) {
    if (k >= K - 1) {
      ++cnt;
      --k;
      continue;
    }
    int32_t v = id[k];
    if (pos[k] >= g->off[v + 1]) {
      --k;
      continue;
    }
    int32_t ext = g->adj[pos[k]++];
    if (ext > v) {
      int ok = 1;
      for (int i = 0; i < k && ok; ++i) ok = lin_find(g, id[i], ext);
      if (ok) {
        ++k;
        id[k] = ext;
        pos[k] = g->off[ext];
      }
    }
  }
  return cnt;
}

/* roots in [root_begin, root_end) (clamped to n) */
uint64_t oracle_clique_dfs_range(const og_graph *g, int K, int32_t root_begin, int32_t root_end, int threads) {
  if (K < 1 || K > 31) return 0;
  if (root_end > g->n) root_end = g->n;
  uint64_t total = 0;
#pragma omp parallel for schedule(dynamic, 1) reduction(+ : total) num_threads(resolve_threads(threads))
  for (int32_t r = root_begin; r < root_end; ++r) total += clique_root(g, r, K);
  return total;
}

uint64_t oracle_clique_dfs(const og_graph *g, int K, int threads) {
  return oracle_clique_dfs_range(g, K, 0, g->n, threads);
}

/* brute force: every K-subset of vertices, all pairs adjacent (tiny graphs only) */
uint64_t oracle_clique_brute(const og_graph *g, int K) {
  int32_t n = g->n;
  if (K < 1 || K > n || K > 31) return 0;
  int32_t c[32];
  for (int i = 0; i < K; ++i) c[i] = i;
  uint64_t cnt = 0;
  while (1) {
    int ok = 1;
    for (int i = 0; i < K && ok; ++i)
      for (int j = i + 1; j < K && ok; ++j) ok = bin_find(g, c[i], c[j]);
    cnt += (uint64_t)ok;
    int i = K - 1;
    while (i >= 0 && c[i] == n - K + i) --i;
    if (i < 0) break;
    ++c[i];
    for (int j = i + 1; j < K; ++j) c[j] = c[j - 1] + 1;
  }
  return cnt;
}

/* ---------------- motif counting with the warp-centric engine's rules ---------------- */

typedef struct {
  int32_t *ext; /* extension lists, one per level */
  int32_t *src;
  int32_t cap;  /* per level */
} motif_ws;

static int motif_extend(const og_graph *g, const int32_t *id, int k, int32_t *ext, int32_t *src, int32_t cap,
                        uint64_t *bytes, int *overflow) {
  /* extend(0,k), DuMatoGPU.cu:1702-1721 */
  int n = 0;
  int32_t v0 = id[0];
  uint64_t degsum = 0;
  for (int i = 0; i <= k; ++i) {
    int32_t v = id[i];
    degsum += (uint64_t)(g->off[v + 1] - g->off[v]);
    for (int64_t e = g->off[v]; e < g->off[v + 1]; ++e) {
      int32_t x = g->adj[e];
      if (x <= v0) continue;
      int dup = 0;
      for (int j = 0; j < n && !dup; ++j) dup = ext[j] == x;
      if (dup) continue;
      if (n >= cap) {
        *overflow = 1;
        return 0;
      }
      ext[n] = x;
      src[n] = i;
      ++n;
    }
  }
  if (bytes) *bytes += 4 * degsum + 8 * (uint64_t)n;
  if (k > 0) {
    /* canonicalFilter2, DuMatoGPU.cu:989-1012 */
    int w = 0;
    for (int j = 0; j < n; ++j) {
      int bad = 0;
      for (int i = 1; i <= k && !bad; ++i) {
        int32_t t = id[i];
        if ((i > src[j] && ext[j] <= t) || (i < src[j] && ext[j] == t)) bad = 1;
      }
      if (!bad) {
        ext[w] = ext[j];
        src[w] = src[j];
        ++w;
      }
    }
    n = w;
  }
  return n;
}

static void motif_root(const og_graph *g, int32_t root, int K, const int32_t *q2c, uint64_t *hist, motif_ws *ws,
                       uint64_t *bytes, int *overflow) {
  int32_t id[8];
  uint64_t ind[8];
  int cnt[8];
  id[0] = root;
  ind[0] = ind[1] = 0;
  int k = 0;
  cnt[0] = -1;
  while (k >= 0) {
    int32_t *ext = ws->ext + (size_t)k * ws->cap;
    int32_t *src = ws->src + (size_t)k * ws->cap;
    if (cnt[k] == -1) {
      cnt[k] = motif_extend(g, id, k, ext, src, ws->cap, bytes, overflow);
      if (*overflow) return;
    }
    if (cnt[k] == 0) {
      --k;
      continue;
    }
    if (k == K - 2) {
      /* aggregate_pattern, DuMatoGPU.cu:930-967 */
      int off = ((k - 1) * (2 + k)) / 2;
      for (int j = 0; j < cnt[k]; ++j) {
        uint64_t qp = 0;
        for (int i = 0; i <= k; ++i)
          if (lin_find(g, id[i], ext[j])) qp += 1ull << (off + i);
        qp += ind[k];
        hist[q2c[qp]]++;
        if (bytes) *bytes += 4 * (uint64_t)(k + 1) + 8;
      }
      cnt[k] = 0;
      --k;
      continue;
    }
    /* forward_induce, DuMatoGPU.cu:846-869 */
    int32_t next = ext[cnt[k] - 1];
    cnt[k]--;
    ++k;
    id[k] = next;
    cnt[k] = -1;
    if (k >= 2) {
      int off = ((k - 2) * (2 + k - 1)) / 2;
      uint64_t qp = 0;
      for (int i = 0; i < k; ++i)
        if (lin_find(g, id[i], next)) qp += 1ull << (off + i);
      ind[k] = ind[k - 1] + qp;
    } else {
      ind[k] = 0;
    }
  }
}

/* hist[n_classes] += counts for roots in [root_begin, root_end). Returns 0, or -1 when an
   extension list outgrew its bound (the caller then raises the bound). */
int oracle_motifs_range(const og_graph *g, int K, const int32_t *q2c, int32_t n_classes, uint64_t *hist,
                        int32_t root_begin, int32_t root_end, int threads, uint64_t *bytes_out) {
  if (K < 3 || K > 7) return -2;
  if (root_end > g->n) root_end = g->n;
  int nt = resolve_threads(threads);
  int overflow = 0;
  uint64_t bytes_total = 0;
  int32_t cap = (int32_t)((int64_t)g->maxdeg * K + 64);
#pragma omp parallel num_threads(nt) reduction(+ : bytes_total)
  {
    uint64_t *h = (uint64_t *)calloc((size_t)n_classes, sizeof(uint64_t));
    motif_ws ws;
    ws.cap = cap;
    ws.ext = (int32_t *)malloc(sizeof(int32_t) * (size_t)cap * K);
    ws.src = (int32_t *)malloc(sizeof(int32_t) * (size_t)cap * K);
    int ov = 0;
    uint64_t b = 0;
#pragma omp for schedule(dynamic, 1)
    for (int32_t r = root_begin; r < root_end; ++r) {
      if (!ov) motif_root(g, r, K, q2c, h, &ws, bytes_out ? &b : NULL, &ov);
    }
#pragma omp critical
    {
      for (int32_t c = 0; c < n_classes; ++c) hist[c] += h[c];
      if (ov) overflow = 1;
    }
    bytes_total += b;
    free(h);
    free(ws.ext);
    free(ws.src);
  }
  if (bytes_out) *bytes_out += bytes_total;
  return overflow ? -1 : 0;
}

int oracle_motifs(const og_graph *g, int K, const int32_t *q2c, int32_t n_classes, uint64_t *hist, int threads) {
  return oracle_motifs_range(g, K, q2c, n_classes, hist, 0, g->n, threads, NULL);
}

/* quick code of an ordering of K vertices whose first two are adjacent */
static uint64_t quick_of_order(const og_graph *g, const int32_t *v, int K) {
  uint64_t q = 0;
  for (int p = 2; p < K; ++p) {
    int off = (p - 2) * (p + 1) / 2;
    for (int j = 0; j < p; ++j)
      if (bin_find(g, v[j], v[p])) q |= 1ull << (off + j);
  }
  return q;
}

/* brute force: every K-subset, keep connected induced subgraphs, classify through the
   dictionary via any ordering that starts with an edge. Independent of the canonical rule. */
int oracle_motifs_brute(const og_graph *g, int K, const int32_t *q2c, int32_t n_classes, uint64_t *hist) {
  int32_t n = g->n;
  if (K < 3 || K > 7 || K > n) return 0;
  (void)n_classes;
  int32_t c[8];
  for (int i = 0; i < K; ++i) c[i] = i;
  while (1) {
    /* connectivity by BFS over the induced subgraph */
    int seen = 1, frontier = 1;
    while (frontier) {
      int nx = 0;
      for (int a = 0; a < K; ++a)
        if ((frontier >> a) & 1)
          for (int b = 0; b < K; ++b)
            if (!((seen >> b) & 1) && bin_find(g, c[a], c[b])) nx |= 1 << b;
      seen |= nx;
      frontier = nx;
    }
    if (seen == (1 << K) - 1) {
      int32_t ord[8];
      int found = 0;
      for (int a = 0; a < K && !found; ++a)
        for (int b = 0; b < K && !found; ++b)
          if (a != b && bin_find(g, c[a], c[b])) {
            ord[0] = c[a];
            ord[1] = c[b];
            int p = 2;
            for (int x = 0; x < K; ++x)
              if (x != a && x != b) ord[p++] = c[x];
            found = 1;
          }
      hist[q2c[quick_of_order(g, ord, K)]]++;
    }
    int i = K - 1;
    while (i >= 0 && c[i] == n - K + i) --i;
    if (i < 0) break;
    ++c[i];
    for (int j = i + 1; j < K; ++j) c[j] = c[j - 1] + 1;
  }
  return 0;
}

/* ---------------- algorithmic bytes for the clique roofline ---------------- */

/* Degree-ordered DAG: rank by (degree without self-loops, id); arcs to higher rank. */
typedef struct {
  int32_t n;
  int64_t *off;
  int32_t *adj;
  int32_t *orig; /* rank -> original id */
} og_dag;

static og_dag *make_dag(const og_graph *g) {
  int32_t n = g->n;
  int32_t *deg = (int32_t *)malloc(sizeof(int32_t) * (n + 1));
  for (int32_t v = 0; v < n; ++v) {
    int32_t d = 0;
    for (int64_t e = g->off[v]; e < g->off[v + 1]; ++e) d += g->adj[e] != v;
    deg[v] = d;
  }
  /* rank by (deg, id): key = deg << 32 | id */
  uint64_t *key = (uint64_t *)malloc(sizeof(uint64_t) * (n + 1));
  for (int32_t v = 0; v < n; ++v) key[v] = ((uint64_t)deg[v] << 32) | (uint32_t)v;
  qsort(key, (size_t)n, sizeof(uint64_t), cmp_u64);
  int32_t *rank = (int32_t *)malloc(sizeof(int32_t) * (n + 1));
  for (int32_t r = 0; r < n; ++r) rank[(uint32_t)key[r]] = r;
  og_dag *d = (og_dag *)calloc(1, sizeof(og_dag));
  d->n = n;
  d->orig = (int32_t *)malloc(sizeof(int32_t) * (n + 1));
  for (int32_t r = 0; r < n; ++r) d->orig[r] = (int32_t)(uint32_t)key[r];
  d->off = (int64_t *)calloc((size_t)n + 1, sizeof(int64_t));
  for (int32_t v = 0; v < n; ++v)
    for (int64_t e = g->off[v]; e < g->off[v + 1]; ++e) {
      int32_t u = g->adj[e];
      if (u != v && rank[u] > rank[v]) d->off[rank[v] + 1]++;
    }
  for (int32_t r = 0; r < n; ++r) d->off[r + 1] += d->off[r];
  d->adj = (int32_t *)malloc(sizeof(int32_t) * (size_t)(d->off[n] + 1));
  int64_t *fill = (int64_t *)malloc(sizeof(int64_t) * (n + 1));
  memcpy(fill, d->off, sizeof(int64_t) * n);
  for (int32_t v = 0; v < n; ++v)
    for (int64_t e = g->off[v]; e < g->off[v + 1]; ++e) {
      int32_t u = g->adj[e];
      if (u != v && rank[u] > rank[v]) d->adj[fill[rank[v]]++] = rank[u];
    }
  for (int32_t r = 0; r < n; ++r) {
    /* insertion sort per row (rows are short) */
    for (int64_t i = d->off[r] + 1; i < d->off[r + 1]; ++i) {
      int32_t x = d->adj[i];
      int64_t j = i - 1;
      while (j >= d->off[r] && d->adj[j] > x) {
        d->adj[j + 1] = d->adj[j];
        --j;
      }
      d->adj[j + 1] = x;
    }
  }
  free(fill);
  free(rank);
  free(key);
  free(deg);
  return d;
}

static void free_dag(og_dag *d) {
  free(d->orig);
  free(d->off);
  free(d->adj);
  free(d);
}

static int32_t intersect_sorted(const int32_t *a, int32_t na, const int32_t *b, int32_t nb, int32_t *out) {
  int32_t i = 0, j = 0, n = 0;
  while (i < na && j < nb) {
    if (a[i] < b[j]) ++i;
    else if (a[i] > b[j]) ++j;
    else {
      out[n++] = a[i];
      ++i;
      ++j;
    }
  }
  return n;
}

/* Counts k-cliques on the DAG by candidate-set intersection and sums the algorithmic
   bytes of every node that computes a candidate set (levels 0..K-2). */
static void dag_clique_root(const og_dag *d, int32_t r, int K, int32_t *buf, int32_t cap, uint64_t *cnt,
                            uint64_t *bytes) {
  int32_t *C[32];
  int32_t nC[32], pos[32];
  int32_t na = (int32_t)(d->off[r + 1] - d->off[r]);
  C[0] = buf;
  memcpy(C[0], d->adj + d->off[r], sizeof(int32_t) * na);
  nC[0] = na;
  *bytes += 4 * (uint64_t)na + 4 * (uint64_t)na;
  if (K == 2) {
    *cnt += (uint64_t)na;
    return;
  }
  int l = 0;
  pos[0] = 0;
  for (int i = 1; i < K - 1; ++i) C[i] = buf + (size_t)i * cap;
  while (l >= 0) {
    if (l == K - 2) {
      *cnt += (uint64_t)nC[l];
      --l;
      continue;
    }
    if (pos[l] >= nC[l]) {
      --l;
      continue;
    }
    int32_t v = C[l][pos[l]++];
    int32_t nv = (int32_t)(d->off[v + 1] - d->off[v]);
    int32_t nn = intersect_sorted(C[l], nC[l], d->adj + d->off[v], nv, C[l + 1]);
    *bytes += 4 * ((uint64_t)nC[l] + (uint64_t)nv) + 4 * (uint64_t)nn;
    ++l;
    nC[l] = nn;
    pos[l] = 0;
  }
}

/* Returns the K-clique count from the DAG and writes the algorithmic bytes. */
uint64_t oracle_clique_dag_bytes(const og_graph *g, int K, uint64_t *bytes_out, int threads) {
  if (K < 2 || K > 31) return 0;
  og_dag *d = make_dag(g);
  int32_t maxo = 0;
  for (int32_t r = 0; r < d->n; ++r) {
    int32_t x = (int32_t)(d->off[r + 1] - d->off[r]);
    if (x > maxo) maxo = x;
  }
  int32_t cap = maxo + 1;
  uint64_t total = 0, bytes = 0;
#pragma omp parallel num_threads(resolve_threads(threads)) reduction(+ : total, bytes)
  {
    int32_t *buf = (int32_t *)malloc(sizeof(int32_t) * (size_t)cap * K);
    uint64_t c = 0, b = 0;
#pragma omp for schedule(dynamic, 16)
    for (int32_t r = 0; r < d->n; ++r) dag_clique_root(d, r, K, buf, cap, &c, &b);
    total += c;
    bytes += b;
    free(buf);
  }
  free_dag(d);
  if (bytes_out) *bytes_out = bytes;
  return total;
}

/* Per-root K-clique counts on the degree-ordered DAG, indexed by original vertex id (the
   root of a clique is its lowest-ranked vertex): the subtree size logged per task, used to
   check the engine's logger and the work predictor. */
void oracle_clique_dag_per_root(const og_graph *g, int K, uint64_t *per_root, int threads) {
  og_dag *d = make_dag(g);
  int32_t maxo = 0;
  for (int32_t r = 0; r < d->n; ++r) {
    int32_t x = (int32_t)(d->off[r + 1] - d->off[r]);
    if (x > maxo) maxo = x;
  }
  int32_t cap = maxo + 1;
#pragma omp parallel num_threads(resolve_threads(threads))
  {
    int32_t *buf = (int32_t *)malloc(sizeof(int32_t) * (size_t)cap * (K > 2 ? K : 2));
#pragma omp for schedule(dynamic, 16)
    for (int32_t r = 0; r < d->n; ++r) {
      uint64_t c = 0, b = 0;
      dag_clique_root(d, r, K, buf, cap, &c, &b);
      per_root[d->orig[r]] = c;
    }
    free(buf);
  }
  free_dag(d);
}

/* Plain DFS over an explicit list of roots (the bounded samples of the CPU baseline). */
uint64_t oracle_clique_dfs_roots(const og_graph *g, int K, const int32_t *roots, int64_t n_roots, int threads) {
  if (K < 1 || K > 31) return 0;
  uint64_t total = 0;
#pragma omp parallel for schedule(dynamic, 1) reduction(+ : total) num_threads(resolve_threads(threads))
  for (int64_t i = 0; i < n_roots; ++i)
    if (roots[i] >= 0 && roots[i] < g->n) total += clique_root(g, roots[i], K);
  return total;
}

/* Motif counts over an explicit list of roots (shard checks). */
int oracle_motifs_roots(const og_graph *g, int K, const int32_t *q2c, int32_t n_classes, uint64_t *hist,
                        const int32_t *roots, int64_t n_roots, int threads) {
  if (K < 3 || K > 7) return -2;
  int overflow = 0;
  int32_t cap = (int32_t)((int64_t)g->maxdeg * K + 64);
#pragma omp parallel num_threads(resolve_threads(threads))
  {
    uint64_t *h = (uint64_t *)calloc((size_t)n_classes, sizeof(uint64_t));
    motif_ws ws;
    ws.cap = cap;
    ws.ext = (int32_t *)malloc(sizeof(int32_t) * (size_t)cap * K);
    ws.src = (int32_t *)malloc(sizeof(int32_t) * (size_t)cap * K);
    int ov = 0;
#pragma omp for schedule(dynamic, 1)
    for (int64_t i = 0; i < n_roots; ++i)
      if (!ov && roots[i] >= 0 && roots[i] < g->n) motif_root(g, roots[i], K, q2c, h, &ws, NULL, &ov);
#pragma omp critical
    {
      for (int32_t c = 0; c < n_classes; ++c) hist[c] += h[c];
      if (ov) overflow = 1;
    }
    free(h);
    free(ws.ext);
    free(ws.src);
  }
  return overflow ? -1 : 0;
}

/* ---------------- closed-form 4-vertex graphlet counts (independent check) ----------------
   Connected induced 4-vertex subgraphs of the whole graph by isomorphism type, computed
   WITHOUT enumerating them, so that the motif engine's k = 4 histogram can be checked on
   graphs whose 4-subgraph count is far beyond any enumerator (the checker's own parity
   is pinned by the enumerating oracle on small graphs). Non-induced copies of each type:
     star (claw)  S = sum_v C(d_v, 3)
     path P4      P = sum_{uv in E} (d_u - 1)(d_v - 1) - 3T          (T triangles)
     paw          W = sum_v t_v (d_v - 2)                           (t_v triangles at v)
     4-cycle      C = number of 4-cycles, each counted once from its highest-ranked vertex
                      and the vertex opposite it (wedge counting in degree order)
     diamond      D = sum_{uv in E} C(t_uv, 2)                      (t_uv triangles on uv)
     K4           Q = 4-cliques
   and the induced counts follow by removing the copies each denser type holds:
     K4 = Q, diamond = D - 6Q, C4 = C - diamond - 3Q, paw = W - 4 diamond - 12Q,
     claw = S - paw - 2 diamond - 4Q, P4 = P - 2 paw - 4 C4 - 6 diamond - 12Q.
   out[6] = {P4, claw, C4, paw, diamond, K4}. Self-loops are ignored. */
int oracle_graphlet4(const og_graph *g, uint64_t *out, int threads) {
  og_dag *d = make_dag(g);
  const int32_t n = d->n;
  int64_t *deg = (int64_t *)calloc((size_t)n + 1, sizeof(int64_t)); /* rank space */
  for (int32_t r = 0; r < n; ++r) {
    const int32_t v = d->orig[r];
    int64_t x = 0;
    for (int64_t e = g->off[v]; e < g->off[v + 1]; ++e) x += g->adj[e] != v;
    deg[r] = x;
  }
  /* undirected rank-space adjacency: in-neighbours (lower rank) then out-neighbours */
  int64_t *uoff = (int64_t *)calloc((size_t)n + 1, sizeof(int64_t));
  for (int32_t r = 0; r < n; ++r) uoff[r + 1] = deg[r];
  for (int32_t r = 0; r < n; ++r) uoff[r + 1] += uoff[r];
  int32_t *uadj = (int32_t *)malloc(sizeof(int32_t) * (size_t)(uoff[n] + 1));
  int64_t *fill = (int64_t *)malloc(sizeof(int64_t) * ((size_t)n + 1));
  memcpy(fill, uoff, sizeof(int64_t) * (size_t)n);
  for (int32_t r = 0; r < n; ++r)
    for (int64_t e = d->off[r]; e < d->off[r + 1]; ++e) uadj[fill[d->adj[e]]++] = r; /* in, ascending r */
  for (int32_t r = 0; r < n; ++r)
    for (int64_t e = d->off[r]; e < d->off[r + 1]; ++e) uadj[fill[r]++] = d->adj[e]; /* out, ascending */
  free(fill);
  const int64_t m_dag = d->off[n];
  uint64_t *te = (uint64_t *)calloc((size_t)m_dag + 1, sizeof(uint64_t)); /* per DAG edge */
  uint64_t *tv = (uint64_t *)calloc((size_t)n + 1, sizeof(uint64_t));
  uint64_t T = 0;
  const int nt = resolve_threads(threads);
#pragma omp parallel for schedule(dynamic, 64) reduction(+ : T) num_threads(nt)
  for (int32_t r = 0; r < n; ++r) {
    for (int64_t p1 = d->off[r]; p1 < d->off[r + 1]; ++p1) {
      const int32_t v = d->adj[p1];
      int64_t i = p1 + 1, j = d->off[v];
      while (i < d->off[r + 1] && j < d->off[v + 1]) {
        if (d->adj[i] < d->adj[j]) ++i;
        else if (d->adj[i] > d->adj[j]) ++j;
        else {
          const int32_t w = d->adj[i];
#pragma omp atomic
          te[p1]++;
#pragma omp atomic
          te[i]++;
#pragma omp atomic
          te[j]++;
#pragma omp atomic
          tv[r]++;
#pragma omp atomic
          tv[v]++;
#pragma omp atomic
          tv[w]++;
          ++T;
          ++i;
          ++j;
        }
      }
    }
  }
  uint64_t S = 0, P = 0, W = 0, D = 0, C = 0;
  for (int32_t r = 0; r < n; ++r) {
    const uint64_t x = (uint64_t)deg[r];
    if (x >= 3) S += x * (x - 1) * (x - 2) / 6;
    if (x >= 2) W += tv[r] * (x - 2);
    for (int64_t e = d->off[r]; e < d->off[r + 1]; ++e) {
      const uint64_t y = (uint64_t)deg[d->adj[e]];
      P += (x - 1) * (y - 1);
      D += te[e] * (te[e] - (te[e] > 0)) / 2;
    }
  }
  P -= 3 * T;
#pragma omp parallel num_threads(nt) reduction(+ : C)
  {
    uint32_t *cnt = (uint32_t *)calloc((size_t)n + 1, sizeof(uint32_t));
    int32_t *touched = (int32_t *)malloc(sizeof(int32_t) * ((size_t)n + 1));
#pragma omp for schedule(dynamic, 64)
    for (int32_t u = 0; u < n; ++u) {
      int64_t nt_ = 0;
      for (int64_t e = uoff[u]; e < uoff[u + 1]; ++e) {
        const int32_t v = uadj[e];
        if (v >= u) break; /* in-neighbours come first, ascending */
        for (int64_t f = uoff[v]; f < uoff[v + 1]; ++f) {
          const int32_t w = uadj[f];
          if (w >= u) continue;
          if (cnt[w]++ == 0) touched[nt_++] = w;
        }
      }
      for (int64_t t = 0; t < nt_; ++t) {
        const uint64_t c = cnt[touched[t]];
        C += c * (c - (c > 0)) / 2;
        cnt[touched[t]] = 0;
      }
    }
    free(cnt);
    free(touched);
  }
  free(uadj);
  free(uoff);
  free(te);
  free(tv);
  free(deg);
  free_dag(d);
  const uint64_t Q = oracle_clique_dag_bytes(g, 4, NULL, threads);
  const uint64_t dia = D - 6 * Q;
  const uint64_t c4 = C - dia - 3 * Q;
  const uint64_t paw = W - 4 * dia - 12 * Q;
  const uint64_t claw = S - paw - 2 * dia - 4 * Q;
  const uint64_t p4 = P - 2 * paw - 4 * c4 - 6 * dia - 12 * Q;
  out[0] = p4;
  out[1] = claw;
  out[2] = c4;
  out[3] = paw;
  out[4] = dia;
  out[5] = Q;
  return 0;
}

/* ---------------- pattern-aware queries q4..q13 ----------------
   src/main/q{n}_PA.cu with the extension steps of src/main/DuMatoGPU.cu:1222-1445, run with
   k = n: an increasing (n-2)-clique v_0 < .. < v_{n-3} (extend_single above v_0, then
   intersect with N(v_l) above v_l), then v_{n-2} from the clique's common neighbourhood
   outside the prefix (extend_single + intersect_unique) and v_{n-1} from the same set above
   v_{n-2} (copy_extensions), counted at the last level. The count is therefore the sum over
   (n-2)-cliques of t(t-1)/2, t = |common neighbourhood| (members excluded, self-loops
   ignored). Cliques come from the degree-ordered DAG, one per vertex set. */
static uint64_t near_root(const og_graph *g, const og_dag *d, int32_t r, int c, int32_t *buf, int32_t cap,
                          int32_t *mem, int32_t *sc0, int32_t *sc1) {
  int32_t *C[16];
  int32_t nC[16], pos[16];
  uint64_t total = 0;
  mem[0] = d->orig[r];
  C[0] = buf;
  nC[0] = (int32_t)(d->off[r + 1] - d->off[r]);
  memcpy(C[0], d->adj + d->off[r], sizeof(int32_t) * nC[0]);
  for (int i = 1; i < c; ++i) C[i] = buf + (size_t)i * cap;
  int l = 0;
  pos[0] = 0;
  if (c == 1) l = -1;
  while (l >= 0) {
    if (pos[l] >= nC[l]) {
      --l;
      continue;
    }
    int32_t v = C[l][pos[l]++];
    mem[l + 1] = d->orig[v];
    if (l + 2 == c) {
      /* common neighbourhood of mem[0..c) in the undirected graph */
      int32_t n = 0;
      const int32_t u0 = mem[0];
      for (int64_t e = g->off[u0]; e < g->off[u0 + 1]; ++e) sc0[n++] = g->adj[e];
      for (int i = 1; i < c && n; ++i) {
        const int32_t u = mem[i];
        n = intersect_sorted(sc0, n, g->adj + g->off[u], (int32_t)(g->off[u + 1] - g->off[u]), sc1);
        memcpy(sc0, sc1, sizeof(int32_t) * (size_t)n);
      }
      uint64_t t = 0;
      for (int32_t j = 0; j < n; ++j) {
        int member = 0;
        for (int i = 0; i < c; ++i) member |= sc0[j] == mem[i];
        t += !member;
      }
      total += t * (t > 0 ? t - 1 : 0) / 2;
      continue;
    }
    int32_t nv = (int32_t)(d->off[v + 1] - d->off[v]);
    nC[l + 1] = intersect_sorted(C[l] + pos[l], nC[l] - pos[l], d->adj + d->off[v], nv, C[l + 1]);
    ++l;
    pos[l] = 0;
  }
  return total;
}

uint64_t oracle_near_cliques(const og_graph *g, int n, int threads) {
  if (n < 4 || n > 13) return 0;
  const int c = n - 2;
  og_dag *d = make_dag(g);
  int32_t maxo = 0;
  for (int32_t r = 0; r < d->n; ++r) {
    int32_t x = (int32_t)(d->off[r + 1] - d->off[r]);
    if (x > maxo) maxo = x;
  }
  const int32_t cap = maxo + 1, ucap = g->maxdeg + 1;
  uint64_t total = 0;
#pragma omp parallel num_threads(resolve_threads(threads)) reduction(+ : total)
  {
    int32_t *buf = (int32_t *)malloc(sizeof(int32_t) * (size_t)cap * (c + 1));
    int32_t *sc0 = (int32_t *)malloc(sizeof(int32_t) * (size_t)ucap);
    int32_t *sc1 = (int32_t *)malloc(sizeof(int32_t) * (size_t)ucap);
    int32_t mem[16];
#pragma omp for schedule(dynamic, 16)
    for (int32_t r = 0; r < d->n; ++r) total += near_root(g, d, r, c, buf, cap, mem, sc0, sc1);
    free(buf);
    free(sc0);
    free(sc1);
  }
  free_dag(d);
  return total;
}

/* The same count by brute force over all n-subsets and all choices of the missing pair (tiny
   graphs only): non-induced copies of K_n minus one edge. */
uint64_t oracle_near_cliques_brute(const og_graph *g, int n) {
  if (n < 4 || n > 8 || g->n > 40) return 0;
  int32_t s[8];
  uint64_t total = 0;
  for (int i = 0; i < n; ++i) s[i] = i;
  while (1) {
    if (s[n - 1] < g->n) {
      /* each unordered pair (a, b) may be the missing edge; all other pairs must be edges */
      for (int a = 0; a < n; ++a)
        for (int b = a + 1; b < n; ++b) {
          int ok = 1;
          for (int x = 0; x < n && ok; ++x)
            for (int y = x + 1; y < n && ok; ++y) {
              if (x == a && y == b) continue;
              if (!bin_find(g, s[x], s[y]) || s[x] == s[y]) ok = 0;
            }
          total += ok;
        }
    }
    int i = n - 1;
    while (i >= 0 && s[i] == g->n - n + i) --i;
    if (i < 0) break;
    ++s[i];
    for (int j = i + 1; j < n; ++j) s[j] = s[j - 1] + 1;
  }
  return total;
}
