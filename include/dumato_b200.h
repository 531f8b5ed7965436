/*
 * dumato_b200.h - C ABI of the B200-native warp-centric subgraph enumeration engine.
 *
 * This is the drop-in boundary for DuMato's clique and motif counting path.
 * Every entry point takes plain pointers and sizes; no C++ or framework types cross it.
 * All functions return DM_OK (0) on success and a negative DM_E* status on failure;
 * dm_last_error() then gives a one-line message for the calling thread.
 * The library never calls exit() (unlike the reference's gpuErrorCheck,
 * src/main/Structs.cu:7-16) and never falls back to a CPU path: counting entry points
 * return DM_ENODEVICE when no CUDA device can be used.
 *
 * Reference interfaces replaced (paths are relative to the DuMato project root):
 *   Graph::Graph(const char*)            src/main/Graph.cpp:17-54      -> dm_graph_load_edgelist
 *   DuMatoCPU CSR build                  src/main/DuMatoCPU.cu:94-108  -> dm_graph_* (internal CSR)
 *   DuMatoCPU::DuMatoCPU(...)            src/main/DuMatoCPU.h:46       -> dm_opts (threads, blockSize,
 *                                                                          donationsPerWarp, threshold)
 *   DuMatoCPU::runKernel/waitKernel      src/main/DuMatoCPU.cu:316-326 -> dm_count_cliques / dm_count_motifs
 *   clique kernel + outputAggregateCounter  src/main/clique_PA.cu:9-32,
 *                                        src/main/DuMatoCPU.cu:360-362 -> dm_count_cliques
 *   motifs kernel + outputAggregatePattern  src/main/motifs_DM_WCLB.cu:9-36,
 *                                        src/main/DuMatoCPU.cu:364-384 -> dm_count_motifs
 *   QuickMapping::QuickMapping(int k)    src/main/QuickMapping.cpp:5-45 -> dm_dictionary_load_csv
 *   nauty-based dictionary generation    src/motifs_DM_DFS/Manager.cpp:1067-1118
 *                                                                       -> dm_dictionary_generate
 */
#ifndef DUMATO_B200_H
#define DUMATO_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define DM_ABI_VERSION 2

#if defined(__GNUC__)
#define DM_API __attribute__((visibility("default")))
#else
#define DM_API
#endif

/* status codes */
#define DM_OK 0
#define DM_EINVAL (-1)     /* bad argument (k out of range, null pointer, bad options) */
#define DM_EIO (-2)        /* file missing or unreadable */
#define DM_EFORMAT (-3)    /* malformed edgelist or dictionary */
#define DM_ENOMEM (-4)     /* host or device allocation failed */
#define DM_ENODEVICE (-5)  /* no usable CUDA device */
#define DM_ECUDA (-6)      /* a CUDA call failed */
#define DM_ETIMEOUT (-7)   /* a bounded device-side wait gave up (error word set by a kernel) */
#define DM_EOVERFLOW (-8)  /* a device-side capacity bound was exceeded */
#define DM_EINTERNAL (-9)  /* a kernel found its own state inconsistent (a library fault, not the input) */

typedef struct dm_graph dm_graph;
typedef struct dm_dictionary dm_dictionary;
typedef struct dm_predictor dm_predictor;

/* Graph generators (seeded, deterministic on every platform). */
#define DM_GEN_ER 0        /* G(n, m): m distinct undirected pairs, no self-loops */
#define DM_GEN_CHUNG_LU 1  /* power-law weights w_i ~ (1 + i/i0)^(-1/(gamma-1)) capped at dmax */
#define DM_GEN_RMAT 2      /* R-MAT (a, b, c, 1-a-b-c), trimmed to ids < n, touched ids relabelled */

typedef struct dm_gen_params {
  int32_t kind;       /* DM_GEN_* */
  int32_t n;          /* vertices (R-MAT: id bound before compaction) */
  int64_t m;          /* distinct undirected edges wanted */
  double gamma;       /* Chung-Lu degree exponent */
  double dmax;        /* Chung-Lu weight cap */
  double a, b, c;     /* R-MAT quadrant probabilities */
  uint64_t seed;
} dm_gen_params;

typedef struct dm_graph_info {
  int32_t n_vertices;      /* max id + 1 (isolated ids kept, as Graph.cpp:34-38) */
  int64_t n_edges;         /* distinct undirected edges, self-loops dropped */
  int32_t max_degree;
  int32_t max_out_degree;  /* in the degree-ordered orientation used for cliques */
  int64_t n_self_loops;    /* self-loops seen in the input and dropped */
  int64_t n_input_pairs;   /* pairs read or generated before dedup */
} dm_graph_info;

/* Engine options. Zero-initialise and set struct_size = sizeof(dm_opts). */
#define DM_MODE_AUTO 0
#define DM_MODE_LIST 1     /* sorted-list intersection with warp ballot compaction */
#define DM_MODE_BITMAP 2   /* per-root local adjacency bitmaps, from the graph's clique index when it fits */
#define DM_MODE_REBUILD 3  /* per-root local adjacency bitmaps rebuilt from the CSR in every launch */

/* How a counting launch moves a root's bitmap block from the clique index into shared memory. */
#define DM_STAGE_AUTO 0    /* the library's default (bulk asynchronous copies) */
#define DM_STAGE_LOADS 1   /* 16-byte loads by every lane */
#define DM_STAGE_TMA 2     /* one bulk asynchronous copy (cp.async.bulk) per block */

#define DM_SCHED_PLAIN 0   /* roots in descending degree order + device donation */
#define DM_SCHED_LEARNED 1 /* roots ordered by the work predictor (needs a trained predictor) */
#define DM_SCHED_ID 2      /* roots in id order (the reference's striping order) */

/* A live sample of a running count (the reference's Report thread, src/main/Report.cpp:24-89,
   which prints the share of active warps every interval). */
typedef struct dm_report {
  double elapsed_ms;           /* host time since the counting kernel was launched */
  int32_t warps;               /* warps of the launch */
  int32_t hungry_warps;        /* warps waiting for work when sampled */
  int64_t roots_claimed;       /* root tasks dealt to warps so far */
  int64_t roots_total;
  int64_t pending;             /* root and donated tasks not settled */
  uint64_t donations;          /* tasks donated between warps so far */
  uint64_t progress;           /* work finished (advances while long items run) */
} dm_report;
typedef void (*dm_report_fn)(const dm_report* sample, void* user);

typedef struct dm_opts {
  int32_t struct_size;
  int32_t device;              /* CUDA ordinal; -1 = current device */
  uint64_t stream;             /* cudaStream_t to launch on; 0 = the library's own stream */
  int32_t threads;             /* reference argv[3]: total GPU threads (0 = persistent default) */
  int32_t block_size;          /* reference argv[4]: threads per block (0 = 256) */
  int32_t donations_per_warp;  /* reference argv[5]: donations one task may make (0 = 64) */
  int32_t threshold;           /* reference argv[6]: idle-warp percentage that triggers donation;
                                  >= 100 disables donation (clique_PA.cu:78) */
  int32_t vwarp;               /* virtual-warp width 0 (auto), 8, 16 or 32: motifs, the lanes sharing
                                  a task's second vertices per group; cliques, the lanes running one
                                  first-level candidate's DFS on the list path (the bitmap paths run
                                  one DFS per lane) */
  int32_t mode;                /* DM_MODE_* */
  int32_t scheduler;           /* DM_SCHED_* */
  int32_t rank;                /* root shard: this process counts roots r with r % world == rank */
  int32_t world_size;          /* 0 or 1 = unsharded */
  int32_t timeout_ms;          /* bound on every device-side wait without progress (0 = 30000 ms) */
  const void* predictor;       /* dm_predictor* for DM_SCHED_LEARNED, else NULL */
  uint64_t* subtree_counts;    /* optional, n_vertices entries (original ids), overwritten: the
                                  subgraphs counted under each root task (the subtree-size log) */
  int32_t test_flags;          /* DM_TEST_* (tests of the failure paths only), else 0 */
  int32_t staging;             /* DM_STAGE_* (cliques on the index) */
  int32_t flags;               /* DM_FLAG_* */
  int32_t report_ms;           /* > 0 with report set: sampling interval of live reports */
  dm_report_fn report;         /* called on a library thread every report_ms while a counting
                                  kernel runs (optional) */
  void* report_user;           /* passed to report */
} dm_opts;

/* flags: for the duration of the call, mark the graph's device CSR (and the clique index) as
   persisting in L2 through an access-policy window on the call's stream, with the context's
   persisting set-aside raised to cover it; the window, the set-aside and the persisting lines
   are reset before the call returns. */
#define DM_FLAG_L2_PERSIST 1

/* test_flags: every warp that finishes waits on a device word nothing sets, so the bounded
   wait expires and the call returns DM_ETIMEOUT (exercises the timeout path without a
   fault or a hang; use a short timeout_ms). */
#define DM_TEST_STALL_AT_EXIT 1
/* donations need no minimum task age, so small inputs exercise the donation paths */
#define DM_TEST_EAGER_DONATION 2

typedef struct dm_stats {
  double kernel_ms;            /* device time of the counting kernels (CUDA events) */
  double prep_ms;              /* device time of graph upload/orientation/task ordering */
  uint64_t tasks;              /* root (or donated-prefix) tasks executed */
  uint64_t donations;          /* prefixes donated between warps */
  uint64_t idle_polls;         /* polls by warps that found no work */
  uint64_t nodes;              /* DFS nodes expanded (extend calls) */
  int32_t mode_used;           /* DM_MODE_* actually run */
  int32_t vwarp_used;
  int32_t grid;                /* CTAs launched */
  int32_t block;               /* threads per CTA */
  int32_t kernel_launches;     /* kernels of this library launched for the call */
  int32_t reserved;
  double idle_warp_fraction;   /* time warps waited for work / (warps x kernel time) */
  double max_task_ms;          /* longest single task (root or donated range) */
  int32_t max_task_root;       /* its root (cliques: rank space; motifs: vertex id) */
  int32_t prefix_donations;    /* of the donations, DFS prefixes below the first level (motifs) */
} dm_stats;

/* ---- version / errors ---- */
DM_API int dm_abi_version(void);
DM_API const char* dm_last_error(void);
DM_API int dm_device_count(void);

/* ---- graphs ---- */
DM_API int dm_graph_load_edgelist(const char* path, dm_graph** out);
/* The same reader on the GPU (replaces Graph::Graph + the CSR build, src/main/Graph.cpp:17-75,
   src/main/DuMatoCPU.cu:94-108): the file's bytes are parsed, deduplicated, symmetrised
   and degree-oriented on the device of opts (may be NULL), and the graph is identical to
   dm_graph_load_edgelist's (same CSR, orientation, counts and format errors). Files below
   2 GiB. *device_ms (may be NULL) receives the device time from the byte upload to the
   read-back of the CSRs. */
DM_API int dm_graph_load_edgelist_device(const char* path, const dm_opts* opts, dm_graph** out, double* device_ms);
DM_API int dm_graph_from_edges(const int32_t* src, const int32_t* dst, int64_t n_pairs,
                        int32_t n_vertices, dm_graph** out);
DM_API int dm_graph_generate(const dm_gen_params* params, dm_graph** out);
DM_API int dm_graph_info_get(const dm_graph* g, dm_graph_info* info);
/* Distinct undirected edges as (u < v) pairs, sorted; arrays of length info.n_edges. */
DM_API int dm_graph_edges(const dm_graph* g, int32_t* u, int32_t* v);
/* Undirected CSR: offsets[n+1] (int64), adjacency[2m] sorted ascending per row. */
DM_API int dm_graph_csr(const dm_graph* g, int64_t* offsets, int32_t* adjacency);
DM_API int dm_graph_write_edgelist(const dm_graph* g, const char* path);
DM_API void dm_graph_free(dm_graph* g);

/* ---- canonical-class dictionaries (quick code -> class) ---- */
DM_API int dm_dictionary_generate(int32_t k, dm_dictionary** out);
DM_API int dm_dictionary_load_csv(const char* path, dm_dictionary** out);
DM_API int dm_dictionary_write_csv(const dm_dictionary* d, const char* path);
/* k, number of quick codes (2^(k(k-1)/2-1)), number of classes */
DM_API int dm_dictionary_shape(const dm_dictionary* d, int32_t* k, int64_t* n_quicks, int32_t* n_classes);
/* quick_to_class[n_quicks] and class_code[n_classes] (the class's global code) */
DM_API int dm_dictionary_tables(const dm_dictionary* d, int32_t* quick_to_class, uint64_t* class_code);
/* 1 if the class is a connected graph, else 0; connected[n_classes] */
DM_API int dm_dictionary_connected(const dm_dictionary* d, uint8_t* connected);
DM_API void dm_dictionary_free(dm_dictionary* d);

/* ---- counting (GPU only) ---- */
/* Number of k-cliques, k in [2, 12]. */
DM_API int dm_count_cliques(dm_graph* g, int32_t k, const dm_opts* opts, uint64_t* count, dm_stats* stats);
/* Clique counts of every size 3..kmax (kmax in [4, 8]): counts[j] = number of (j + 3)-cliques
   (no counterpart in the reference, whose driver counts one k per run). One launch walks the
   clique index to depth kmax and counts every size on the way down, since a DFS to depth
   kmax meets every smaller clique as a prefix. A graph whose index is not available, with
   roots above 256 out-neighbours, or a call with mode DM_MODE_LIST / DM_MODE_REBUILD or a
   subtree log, is counted with one launch per size instead (the same counts; the subtree log
   then holds the kmax log). */
DM_API int dm_count_cliques_upto(dm_graph* g, int32_t kmax, const dm_opts* opts, uint64_t* counts,
                                 dm_stats* stats);
/* The reference's pattern-aware queries q4..q13 (src/main/q4_PA.cu .. q13_PA.cu, extension
   steps src/main/DuMatoGPU.cu:1222-1445, run with k = n): the number of non-induced copies of
   K_n minus one edge, n in [4, 13] - an (n-2)-clique with two vertices adjacent to all of it,
   sum over (n-2)-cliques C of t(t-1)/2 with t the size of C's common neighbourhood. */
DM_API int dm_count_near_cliques(dm_graph* g, int32_t n, const dm_opts* opts, uint64_t* count, dm_stats* stats);
/* Connected induced k-vertex subgraphs per class of dict (k in [3, 7]).
   class_counts has n_classes entries (dm_dictionary_shape). */
DM_API int dm_count_motifs(dm_graph* g, int32_t k, const dm_dictionary* dict, const dm_opts* opts,
                    uint64_t* class_counts, dm_stats* stats);

/* ---- batched mining (no counterpart in the reference, whose drivers run one graph and one
   query per process) ----
   Many (graph, query) pairs run in ONE persistent kernel launch over the disjoint union of
   their graphs, captured once in a CUDA graph and replayed by dm_batch_run. Every task
   carries its query; a per-query descriptor selects the path (clique bitmap/list, motif
   with virtual-warp width 8/16/32) and the donation trigger. */
#define DM_QUERY_CLIQUE 0
#define DM_QUERY_MOTIF 1
#define DM_AUTOTUNE_MODEL 0    /* choose per query from a cost model of the graph */
#define DM_AUTOTUNE_MEASURE 1  /* time each candidate on the query alone, keep the fastest */

typedef struct dm_query {
  int32_t kind;                /* DM_QUERY_* */
  int32_t k;                   /* cliques: [2, 6]; motifs: [3, 5] */
  dm_graph* graph;
  const dm_dictionary* dict;   /* motifs: the k-vertex dictionary; cliques: NULL */
  int32_t vwarp;               /* 0 = autotune, else 8, 16 or 32 (motifs) */
  int32_t threshold;           /* -1 = autotune, else the dm_opts.threshold meaning */
  int32_t mode;                /* DM_MODE_AUTO = autotune, DM_MODE_LIST, DM_MODE_BITMAP (cliques) */
  int32_t reserved;
} dm_query;

typedef struct dm_query_tuning {
  int32_t vwarp;               /* chosen virtual-warp width (cliques: 32) */
  int32_t threshold;           /* chosen donation threshold (100 = no donation) */
  int32_t mode;                /* DM_MODE_LIST / DM_MODE_BITMAP (motifs: DM_MODE_LIST) */
  int32_t n_results;           /* 1 (cliques) or the dictionary's class count (motifs) */
  int64_t result_offset;       /* first result of this query in dm_batch_run's output */
  double tune_ms;              /* measured time of the chosen setting (DM_AUTOTUNE_MEASURE), else 0 */
  double est_cost;             /* cost-model estimate of the query's work (arbitrary units) */
} dm_query_tuning;

typedef struct dm_batch dm_batch;

/* Builds the union graph and descriptor table on the device, tunes every query and
   captures the launch. opts: device, threads, donations_per_warp, timeout_ms as in
   dm_count_cliques (may be NULL). The graphs must stay alive until dm_batch_free. */
DM_API int dm_batch_create(const dm_query* queries, int32_t n_queries, const dm_opts* opts, int32_t autotune,
                           dm_batch** out);
/* Total result words (sum of n_results over the queries). */
DM_API int64_t dm_batch_num_results(const dm_batch* b);
DM_API int dm_batch_tuning(const dm_batch* b, int32_t query, dm_query_tuning* out);
/* Replays the captured launch: results[result_offset(q) ..] receives query q's count(s). */
DM_API int dm_batch_run(dm_batch* b, uint64_t* results, int64_t n_results, dm_stats* stats);
DM_API void dm_batch_free(dm_batch* b);

/* Work model of the clique path (host-side, for roofline accounting only; it is not a
   counting path): on the degree-ordered DAG, every DFS node at levels 0..k-2 that computes
   a candidate set C_child = C_parent cap N+(v) costs 4(|C_parent| + |N+(v)|) + 4|C_child|
   bytes (level 0: 4|N+(v0)| + 4|C_0|). Writes the node count and the byte total. */
DM_API int dm_clique_work_model(dm_graph* g, int32_t k, uint64_t* nodes, uint64_t* bytes);

/* Work model of the motif path (host-side, for roofline accounting only; it counts nothing):
   every canonical prefix (v_0..v_t), t <= k-2, of the reference's motif DFS costs
   4 sum_i deg(v_i) + 8 |union of their neighbourhoods above v_0| bytes (extend(0,k)), and
   every leaf candidate 4(k-1) + 8 (adjacency probes and the dictionary read). Writes the
   number of prefixes and the byte total; walks the prefixes only (not the leaves). */
DM_API int dm_motif_work_model(dm_graph* g, int32_t k, uint64_t* nodes, uint64_t* bytes);

/* k-cliques of a DAG already in device memory, with no GPU allocation (no counterpart in
   the reference). For callers that cannot call cudaMalloc: code that runs inside another
   framework's memory pool or an allocator-free runtime, or that must not change the
   device's allocation state. Inputs (device pointers, current device): d_row[v] start of
   v's out-neighbours in d_adj, d_deg[v] their number; every row sorted ascending and
   holding only ids greater than v (for example, an undirected graph keeping u -> v for
   u < v); d_roots[0..n_roots) the vertices to start from (each clique is counted from its
   lowest vertex, so pass every vertex whose out-degree is at least k-1). max_out_degree
   must be at most 256: larger roots need per-warp scratch this entry point does not hold
   (use dm_count_cliques). Output: *count (host). Runs on `stream` and waits for it.
   Scratch: one fixed device array of about 260 KB (counters + donation queue) that every
   GPU loading the library keeps until exit. Every call looks up the array's device address
   in the current context and starts with a small set-up kernel that zeroes the counters
   and, when a tag word in the array says the queue is not in its empty state (the first
   call in a context, or the call after one that failed), rebuilds the queue; the first
   call in a context also loads the array, so make that first call before any stream
   capture. Calls share the array and each leaves its contents behind: calls that overlap
   on the GPU (other streams, threads or processes sharing the context) race and must be
   serialised by the caller. A root whose out-degree exceeds max_out_degree makes the call
   return DM_EOVERFLOW; the next call starts clean. */
DM_API int dm_count_cliques_noalloc(const int32_t* d_row, const int32_t* d_deg, const int32_t* d_adj,
                                    int32_t n_vertices, const int32_t* d_roots, int32_t n_roots,
                                    int32_t max_out_degree, int32_t k, uint64_t stream, uint64_t* count);

/* Host-only planning: the ordered root tasks this shard (o->rank of o->world_size) would run
   for a k query (clique != 0: cliques, else motifs), as original vertex ids with their part
   words (p | P << 16, 0 = whole root). Writes at most cap entries and the total to *n. The
   plain and id schedules need no device. */
DM_API int dm_plan_roots(dm_graph* g, int32_t k, int32_t clique, const dm_opts* o, int32_t* roots, int32_t* parts,
                         int64_t cap, int64_t* n);

/* ---- learned work predictor (no counterpart in the reference) ----
   An 8 -> 32 -> 32 -> 1 FP32 MLP predicting log(1 + subtree size) of a root task, trained
   and evaluated by this library's CUDA kernels. Pass it as dm_opts.predictor with
   scheduler = DM_SCHED_LEARNED to order root tasks by predicted cost and pre-split the
   predicted-heavy ones. */
DM_API int dm_predictor_create(uint64_t seed, dm_predictor** out);
DM_API void dm_predictor_free(dm_predictor* p);
DM_API int dm_predictor_num_params(void);
DM_API int dm_predictor_get_params(const dm_predictor* p, float* params);
DM_API int dm_predictor_set_params(dm_predictor* p, const float* params);
/* features[n_vertices * 8] of every vertex as a root of a k query (clique != 0: clique
   tasks, else motif tasks) */
DM_API int dm_predictor_features(dm_graph* g, int32_t k, int32_t clique, float* features);
DM_API int dm_predictor_predict(const dm_predictor* p, const float* X, int64_t n, float* y);
/* gradient of the mean squared error over (X, T) (one full batch), and the loss */
DM_API int dm_predictor_gradients(const dm_predictor* p, const float* X, const float* T, int64_t n, float* grad,
                                  float* loss);
/* Adam over shuffled minibatches for `epochs` passes; writes the last epoch's mean loss */
DM_API int dm_predictor_train(dm_predictor* p, const float* X, const float* T, int64_t n, int32_t epochs,
                              int32_t batch, float lr, float* final_loss);

/* Release this library's device copies of g on its device (host CSR stays). */
DM_API int dm_graph_release_device(dm_graph* g);

#ifdef __cplusplus
}
#endif
#endif /* DUMATO_B200_H */
