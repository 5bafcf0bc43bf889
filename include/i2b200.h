/*
 * i2b200 — B200 (sm_100a) engine for the edge-relaxation hot path of the
 * Indigo2 suite: BFS levels, SSSP distances and connected-component labels on
 * ECLgraph CSR graphs. Plain C ABI: host pointers, sizes and status codes.
 *
 * Reference interfaces replaced (paths inside the Indigo2Suite project):
 *   struct ECLgraph, readECLgraph, writeECLgraph, freeECLgraph  include/ECLgraph.h:44-106
 *   static double GPUbfs_vertex(int src, const ECLgraph&, int* dist)    include/bfs_vertex_cuda.h:61
 *   static double GPUbfs_edge(int src, const ECLgraph&, int* dist, const int* sp)  include/bfs_edge_cuda.h:61
 *   static double GPUsssp_vertex(...)  include/sssp_vertex_cuda.h:60
 *   static double GPUsssp_edge(...)    include/sssp_edge_cuda.h:60
 *   static double GPUcc_vertex(const ECLgraph&, int* label)              include/cc_vertex_cuda.h:57
 *   static double GPUcc_edge(const ECLgraph&, int* label, const int* sp) include/cc_edge_cuda.h:57
 *   synthetic SSSP weights 1 + (i*nei) % nodes                          include/sssp_vertex_cuda.h:127-137
 *   starting-point array sp[]                                           include/bfs_edge_cuda.h:140-146
 * Unlike the reference, no function here calls exit(): every failure is a
 * status code (the reference exits in CheckCuda(), include/bfs_vertex_cuda.h:101-109).
 */
#ifndef I2B200_H
#define I2B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  I2_OK = 0,
  I2_ERR_ARG = 1,         /* null pointer, source out of range, bad size or option */
  I2_ERR_IO = 2,          /* file could not be opened, read or written */
  I2_ERR_FORMAT = 3,      /* malformed or truncated ECLgraph file or CSR */
  I2_ERR_NOMEM = 4,       /* host or device allocation failed */
  I2_ERR_CUDA = 5,        /* CUDA runtime error */
  I2_ERR_NO_DEVICE = 6,   /* no CUDA device */
  I2_ERR_UNSUPPORTED = 7, /* variant not applicable to this graph (pull on a directed graph) */
  I2_ERR_ITER_CAP = 8,    /* iteration cap reached before the fixed point */
  I2_ERR_OVERFLOW = 9,    /* int32 limit or capacity exceeded */
  I2_ERR_CAPACITY = 10,   /* graph larger than i2_run_noalloc's fixed scratch */
  I2_ERR_STALL = 11       /* a resident traversal's barrier wait ran out of time
                             (I2_STALL_MS, default 10 s); the result is incomplete */
} i2_status;

/* Host CSR graph. Layout-identical to struct ECLgraph (include/ECLgraph.h:44-50). */
typedef struct {
  int nodes;
  int edges;
  int* nindex;  /* nodes + 1 */
  int* nlist;   /* edges */
  int* eweight; /* edges, or NULL */
} i2_eclgraph;

/* Algorithms. */
enum { I2_BFS = 0, I2_SSSP = 1, I2_CC = 2, I2_MIS = 3 };

/* Relaxation variants (styles). Every variant reaches the same fixed point. */
enum {
  I2_AUTO_HEURISTIC = -1, /* per-iteration choice by a fixed frontier-size rule; CC on
                             symmetric graphs takes union-find, and single-source SSSP on
                             graphs of skewed degrees with 2^26 CSR entries or more takes
                             I2_VP_CTA in the budgeted near/far ordering (sssp_budget, the
                             engine's default when 0), both chosen before the first launch */
  I2_AUTO_LEARNED = -2,   /* per-iteration choice by the on-device MLP selector, with the
                             same two choices made before the first launch; on graphs with
                             more vertices than any it was trained on (2^21) it defers to
                             the frequency rule */
  I2_VP_THREAD = 0,       /* vertex push, data-driven, thread per frontier vertex */
  I2_VP_WARP = 1,         /* vertex push, data-driven, warp per frontier vertex */
  I2_VP_CTA = 2,          /* edge-balanced push: thread per frontier edge */
  I2_VP_BLOCK = 3,        /* vertex push, data-driven, block per frontier vertex */
  I2_PULL_FRONTIER = 4,   /* pull from frontier neighbours (bottom-up); symmetric graphs */
  I2_PULL_TOPO = 5,       /* topology-driven pull from all neighbours; symmetric graphs */
  I2_EDGE_TOPO = 6,       /* edge-centric sweep over all CSR entries */
  I2_PUSH_TOPO = 7,       /* topology sweep of the frontier bitmap, thread per vertex */
  I2_UNION_FIND = 8,      /* CC on symmetric graphs only: union-find over all edges, linking the
                             larger root below the smaller, then every label set to its root
                             (two launches; same minimum-ID labels as label propagation) */
  I2_NUM_VARIANTS = 9
};

/* Loop modes. */
enum {
  I2_LOOP_GRAPH = 0,   /* whole traversal is one CUDA graph; its relax kernel is one
                          cooperative launch that runs every iteration, the grid
                          meeting at a barrier between iterations */
  I2_LOOP_HOST = 1,    /* host launches each iteration and reads the frontier size back */
  I2_LOOP_RELAUNCH = 2 /* one CUDA graph with a device-side while loop that launches
                          the relax kernel once per iteration */
};

typedef struct {
  int variant;      /* I2_VP_* ... or I2_AUTO_* */
  int loop_mode;    /* I2_LOOP_GRAPH (default 0) or I2_LOOP_HOST */
  int iter_cap;     /* 0: default cap of nodes + 2 launches (enough for every algorithm) */
  int record_iters; /* 1: keep per-iteration records (i2_get_records) */
  void* stream;     /* cudaStream_t to run on; NULL: the graph's own stream */
  int sssp_delta;   /* SSSP with I2_VP_CTA only: threshold step of the near/far
                       ordering (pushes at or above the threshold wait on a far
                       pile until the near frontier is empty). <= 0: off
                       (plain frontier-driven relaxation), > 0: this step.
                       The distances do not depend on it. */
  int then_at;      /* > 0: run `variant` for iterations 0..then_at-1 and then_variant
                       from iteration then_at on (a fixed switch of style; results do
                       not change). 0: no switch. */
  int then_variant;
  int sssp_budget;  /* SSSP with I2_VP_CTA only, when sssp_delta <= 0: budgeted
                       near/far ordering. Each iteration relaxes only the frontier
                       vertices below a distance threshold that the engine sets on
                       the device so that about `sssp_budget` edges lie below it
                       (from distance histograms of the frontier, and of the far
                       pile when the frontier runs dry); the rest wait on the far
                       pile. 0: off; > 0: this many edges;
                       I2_SSSP_BUDGET_AUTO: the engine's default (28672 per SM,
                       twice that on graphs of 2^30 CSR entries or more).
                       The distances do not depend on it. */
} i2_opts;

#define I2_SSSP_BUDGET_AUTO (-1)

typedef struct {
  double seconds;          /* device time of init + all iterations (CUDA events) */
  double relax_seconds;    /* sum of the relax launches' device durations */
  int iterations;          /* relax launches */
  int variant_hist[16];    /* launches per variant */
  long long reached_vertices;
  long long reached_edges; /* sum of degrees of reached vertices */
} i2_report;

/* Per-iteration record (one per relax launch). */
typedef struct {
  int iter;
  int variant;
  int size;                /* light frontier entries consumed */
  int hsize;               /* heavy frontier entries consumed */
  unsigned long long edges;/* frontier edges consumed */
  int maxdeg;
  int mindist;
  long long visited;       /* vertices reached before this launch */
  unsigned long long t_ns; /* launch duration (device timer) */
  float feat[16];          /* selector features of the consumed frontier */
  int kind;                /* SSSP near/far ordering: 0 relaxation, 1 move from the far pile,
                              3 frontier trim (nothing is relaxed in 1 and 3) */
  int threshold;           /* near/far threshold the launch used (INT_MAX: none) */
  unsigned pile;           /* far-pile entries after the launch (live or superseded) */
  int pad;
} i2_iter_record;

typedef struct {
  int nodes;
  int edges;
  int maxdeg;
  int nheavy;
  int wmin;
  int symmetric;
  int has_weights;
  float avgdeg;
  float degcv;
} i2_graph_info;

typedef struct i2_graph i2_graph;

/* ---- library ---- */
const char* i2_status_string(int status);
const char* i2_variant_name(int variant);
int i2_version(void);
int i2_device_count(void);

/* ---- ECLgraph files (include/ECLgraph.h:52-106; errors are status codes) ---- */
int i2_read_eclgraph(const char* path, i2_eclgraph* out);
int i2_write_eclgraph(const i2_eclgraph* g, const char* path);
void i2_free_eclgraph(i2_eclgraph* g);
/* Allocate an empty graph of the given size (nindex zeroed; eweight if weighted). */
int i2_alloc_eclgraph(int nodes, int edges, int weighted, i2_eclgraph* out);
/* Fill eweight with the reference's synthetic weights (include/sssp_vertex_cuda.h:127-137). */
int i2_synth_weights(i2_eclgraph* g);
/* Host starting-point array sp[e] = source vertex of CSR entry e (include/bfs_edge_cuda.h:140-146). */
int i2_build_sp(const i2_eclgraph* g, int* sp);

/* ---- seeded synthetic graphs (host, OpenMP). Symmetrised, deduplicated, no
   self-loops, sorted adjacency; weights uniform in [1,255], one per undirected edge. ---- */
int i2_gen_er(int n, long long m, uint64_t seed, int weighted, i2_eclgraph* out);
int i2_gen_rmat(int scale, int edge_factor, double a, double b, double c, uint64_t seed,
                int weighted, i2_eclgraph* out);
/* RMAT on n vertices (n need not be a power of two): scale ceil(log2 n),
   edge_factor * 2^scale samples, endpoints >= n rejected after relabelling. */
int i2_gen_rmat_n(int n, int edge_factor, double a, double b, double c, uint64_t seed, int weighted,
                  i2_eclgraph* out);
int i2_gen_grid(int side, double remove_frac, double add_frac, uint64_t seed, int weighted,
                i2_eclgraph* out);

/* ---- device graphs ---- */
/* Copy a host CSR to the device and compute its statistics. */
int i2_graph_upload(const i2_eclgraph* host, i2_graph** out);
/* Wrap CSR arrays already on the device (the reference harness's d_g, include/bfs_vertex_cuda.h:140-144).
   The arrays stay owned by the caller and must outlive the handle. */
int i2_graph_wrap_device(const i2_eclgraph* dev, i2_graph** out);
/* Generate an RMAT graph directly on the device (identical CSR to i2_gen_rmat). */
int i2_graph_generate_rmat(int scale, int edge_factor, double a, double b, double c, uint64_t seed,
                           int weighted, i2_graph** out);
/* RMAT on n vertices directly on the device (identical CSR to i2_gen_rmat_n). */
int i2_graph_generate_rmat_n(int n, int edge_factor, double a, double b, double c, uint64_t seed, int weighted,
                             i2_graph** out);
/* Generate G(n, m) directly on the device (identical CSR to i2_gen_er). */
int i2_graph_generate_er(int n, long long m, uint64_t seed, int weighted, i2_graph** out);
/* Generate the grid graph directly on the device (identical CSR to i2_gen_grid). */
int i2_graph_generate_grid(int side, double remove_frac, double add_frac, uint64_t seed, int weighted,
                           i2_graph** out);
/* Build a CSR graph on the device from m directed pairs (src[k], dst[k]) and,
   if w is not NULL, their int32 weights, all in device memory of the current
   GPU (no counterpart in the reference, whose graphs come from .egr files;
   the host analogue of its sp[] loop is include/bfs_edge_cuda.h:140-146).
   symmetrize != 0 adds the reverse of every pair. Self-loops are dropped,
   duplicate pairs merged (keeping the smallest weight), adjacency sorted.
   Pairs outside [0, nodes) give I2_ERR_FORMAT. */
int i2_graph_from_coo_device(int nodes, long long m, const int* src, const int* dst, const int* w,
                             int symmetrize, i2_graph** out);
/* The highest-degree vertex (lowest ID on ties), the benchmark configurations' source. */
int i2_graph_hub(i2_graph* g, int* v);
/* The starting-point array sp[e] = source vertex of CSR entry e (the
   reference's host loop, include/bfs_edge_cuda.h:140-146), built on the device
   on first need: *sp_dev receives its device address (valid while g lives),
   and sp_host (edges ints, may be NULL) a copy. */
int i2_graph_sp(i2_graph* g, const int** sp_dev, int* sp_host);
int i2_graph_size(const i2_graph* g, int* nodes, int* edges);
int i2_graph_degree(const i2_graph* g, int v, int* deg);
/* Statistics of the graph; the first call also checks symmetry (one pass over the CSR). */
int i2_graph_info_get(const i2_graph* g, i2_graph_info* out);
/* Copy the device CSR back to a host graph allocated by the callee. */
int i2_graph_download(const i2_graph* g, i2_eclgraph* out);
/* Launch tuning of a graph: degree threshold from which a frontier vertex is
   split across the whole grid (heavy path; 0 keeps it), cap on resident blocks
   per SM of the relax kernels (0 keeps it), and the preferred shared-memory
   carveout in percent (-1: driver default; applies process-wide). Results do
   not depend on any of them. */
int i2_graph_tune(i2_graph* g, int heavy_threshold, int blocks_per_sm, int smem_carveout);
/* Vertex numbering the traversals run under. No counterpart in the reference,
   which always traverses the CSR as read. I2_ORDER_DEGREE builds on the device
   a copy of the graph with its vertices renumbered by descending degree (ties
   by ascending ID), kept beside the original: BFS and SSSP then run on the
   copy from the mapped source, and one gather puts their levels or distances
   back in original IDs, identical to the original CSR's (they do not depend on
   the numbering). CC on a graph with symmetric edges runs on the copy too,
   its labels mapped to each component's smallest original ID (the same
   labels); CC on other graphs and MIS keep running on the original CSR (their
   values are IDs). The copy puts the few vertices that most adjacency lists
   name side by side, so their values stay in L2 on graphs whose value arrays
   do not fit there (RMAT scale 26: SSSP 1.5x, BFS 1.4-1.9x, CC 1.7x faster).
   Costs a second CSR in device memory (and, while building, scratch of
   24 bytes per CSR entry) and g.nodes ints on the host; a graph without
   edges keeps no copy. I2_ORDER_NONE drops the copy. Waits for the graph's
   work and the device. */
enum { I2_ORDER_NONE = 0, I2_ORDER_DEGREE = 1 };
int i2_graph_reorder(i2_graph* g, int order);
/* Give the graph the reference's synthetic weights when it has none (on the device). */
int i2_graph_synth_weights(i2_graph* g);
int i2_graph_free(i2_graph* g);
/* Device memory of freed graphs stays reserved in the engine's pool on its
   device, so the next upload or workspace reuses it without a cudaMalloc;
   this hands the unused part of the current device's pool back to the driver
   (for another allocator in the same process). Waits for the device. */
int i2_trim_device_memory(void);

/* ---- traversals (replace GPU<alg>_<vertex|edge>) ----
   dist/label are HOST arrays of g.nodes ints, filled before return. */
int i2_bfs(i2_graph* g, int src, int* dist, const i2_opts* opts, i2_report* rep);
int i2_sssp(i2_graph* g, int src, int* dist, const i2_opts* opts, i2_report* rep);
int i2_cc(i2_graph* g, int* label, const i2_opts* opts, i2_report* rep);
/* Maximal independent set (replaces GPUmis_vertex, include/mis_vertex_cuda.h:52,
   and GPUmis_edge, include/mis_edge_cuda.h:54): status[v] = 1 in the set, 2 not,
   the set the reference's deterministic CUDA MIS variants converge to (priority
   hash(v + 712313887) as int, ties to the larger ID). Symmetric graphs only
   (I2_ERR_UNSUPPORTED otherwise); opts->variant is ignored (one style: a warp
   per frontier vertex). */
int i2_mis(i2_graph* g, int* status, const i2_opts* opts, i2_report* rep);
/* Same, with the result left in (or copied to) DEVICE memory; out_dev may be NULL
   to keep the result only inside the engine. src is ignored for I2_CC and I2_MIS. */
int i2_run_device(i2_graph* g, int algo, int src, int* out_dev, const i2_opts* opts, i2_report* rep);
/* Records of the last traversal run with record_iters = 1. */
int i2_get_records(const i2_graph* g, i2_iter_record* out, int cap, int* n);

/* Per-iteration sweep for selector training: follows the trajectory of `follow`
   (a variant, I2_AUTO_HEURISTIC or I2_AUTO_LEARNED) and times every allowed
   variant from each iteration's state (state saved and restored on the device,
   each launch bracketed by CUDA events, best of `reps`).
   times[it * I2_NUM_VARIANTS + v] in ns (-1: not allowed). */
int i2_sweep(i2_graph* g, int algo, int src, int follow, int reps, i2_iter_record* recs,
             float* times, int cap, int* n);

/* ---- learned selector ---- */
/* Number of floats in the MLP parameter blob (normaliser + 16-64-64-8 weights). */
int i2_mlp_param_count(void);
/* Install the selector's parameters on the current device. */
int i2_mlp_set_params(const float* params, int count);
/* One forward + backward pass of the masked-MSE loss on the device (hand-written
   kernels). X: n x 16 features, T: n x 8 targets, M: n x 8 mask. Outputs the loss
   and the gradient w.r.t. every parameter (same layout as the blob). */
int i2_mlp_loss_grad(const float* params, const float* X, const float* T, const float* M, int n,
                     float* loss, float* grad);
/* Train on the device with Adam for `epochs` passes of minibatches of `batch` rows;
   params is read as the initial point and overwritten with the result. */
int i2_mlp_train(float* params, const float* X, const float* T, const float* M, int n, int epochs,
                 int batch, float lr, uint64_t seed, float* final_loss);
/* Device inference on n feature rows; writes the chosen variant per row (mask of allowed variants). */
int i2_mlp_predict(const float* params, const float* X, int n, int allowed_mask, int* choice);

/* ---- traversal that allocates nothing ----
   No counterpart in the reference. For callers that cannot allocate device
   memory when they query (device memory held by another allocator, query loops
   that cannot afford cudaMalloc's device synchronisation, or no tolerance for
   out-of-memory at query time). The caller passes the CSR and the output
   `dist_dev` (nodes ints), all in device memory; the scratch is a fixed device
   array inside the library (about 3 MB, held on every GPU that loads the
   library until exit), so graphs above 131072 vertices return I2_ERR_CAPACITY.
   Style: edge-balanced push, host-driven loop on `stream` (NULL: legacy
   stream); the call is synchronous: it waits for `stream` after every
   iteration to read the frontier size, and returns when the result is in
   dist_dev. The first call on each device looks up the scratch's device
   address and keeps it for the life of the process; make that first call
   before any stream capture, and make no call after a cudaDeviceReset of that
   device. All calls share the one scratch: calls that overlap on the GPU
   (other streams, other host threads) race and must be serialised by the
   caller. Arrays on another GPU than the current one are refused
   (I2_ERR_ARG), as are negative SSSP weights (I2_ERR_UNSUPPORTED, like
   i2_sssp). src is ignored for I2_CC. `iterations` may be NULL. */
int i2_run_noalloc(int algo, const i2_eclgraph* dev, int src, int* dist_dev, void* stream, int* iterations);

/* ---- batches of graphs traversed together ---- */
typedef struct i2_batch i2_batch;
int i2_batch_upload(const i2_eclgraph* graphs, int n, i2_batch** out);
/* The same batch from graphs already on the device (copied device to device;
   the graphs stay owned by the caller). */
int i2_batch_from_device(i2_graph* const* graphs, int n, i2_batch** out);
/* dist: host array of sum(nodes) ints, graph k's vertices at offset voff[k]. */
int i2_batch_run(i2_batch* b, int algo, const int* srcs, int* dist, const i2_opts* opts, i2_report* rep);
int i2_batch_offsets(const i2_batch* b, long long* voff);
/* Same traversal with the result left on the device (asynchronous on
   opts->stream when rep is NULL); i2_batch_result copies it to the host. */
int i2_batch_run_device(i2_batch* b, int algo, const int* srcs, const i2_opts* opts, i2_report* rep);
int i2_batch_result(i2_batch* b, int* dist, const i2_opts* opts);
/* Tuning of the batch's traversals, as i2_graph_tune (no counterpart in the
   reference; the values come from indigo2suite_b200/tuning_table.json, written
   by the project's autotuner). */
int i2_batch_tune(i2_batch* b, int heavy_threshold, int blocks_per_sm, int smem_carveout);
int i2_batch_free(i2_batch* b);

#ifdef __cplusplus
}
#endif

#endif /* I2B200_H */
