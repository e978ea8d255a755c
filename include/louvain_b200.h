/*
 * louvain_b200.h -- C ABI of the B200 Louvain engine.
 *
 * The reference (FedeFonto/louvain-fast-move-cuda) has no library boundary: its API is the
 * header-compiled static method ModularityAlgorithms::Louvain(GraphHost&, MODE)
 * (modularityAlgorithms.h:8-10) plus the phase classes it calls. Every entry point below
 * replaces one of those reference interfaces; the reference file:line is given beside it.
 * All functions are `extern "C"`, take plain pointers and sizes, never throw, and return
 * an lv_status. include/louvain_b200.hpp rebuilds the reference's C++ surface on top.
 *
 * Conventions
 *  - Graphs are symmetric CSR: row_ptr int64[n+1], col int32[E] (E = row_ptr[n]), optional
 *    weights float32[E] (NULL = every weight 1, the reference's only input kind,
 *    graph.cu:32,68-79). Each undirected edge is stored in both directions with the same
 *    weight. Every vertex needs at least one entry (the reference drops such vertices,
 *    graph.cuh:79-85); self-loop entries are allowed.
 *  - LV_MEM_HOST / LV_MEM_DEVICE say where the caller's buffers live. Host buffers are
 *    copied in and out inside the call.
 *  - Errors never abort the process: a non-zero lv_status is returned and
 *    lv_last_error() gives the message (the reference exits or throws, graph.cu:52-55,
 *    main.cu:26-42).
 */
#ifndef LOUVAIN_B200_H
#define LOUVAIN_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  LV_OK = 0,
  LV_ERR_ARGUMENT = 1,      /* bad pointer, size or configuration */
  LV_ERR_INPUT = 2,         /* graph violates the input contract (range, empty row) */
  LV_ERR_RANGE = 3,         /* total weight or edge count beyond the supported limit */
  LV_ERR_CUDA = 4,          /* a CUDA runtime call failed */
  LV_ERR_NOMEM = 5,         /* device or host allocation failed (reference: bad_alloc) */
  LV_ERR_DEVICE_CHECK = 6,  /* a bounded device loop gave up (probe limit, table full) */
  LV_ERR_BUDGET = 7,        /* serving: request does not fit the memory budget */
  LV_ERR_STATE = 8          /* call not valid in the object's current state */
} lv_status;

/* constants.h:13 enum MODE { HASH, SORT, ADAPTIVE_SPEED, ADAPTIVE_MEMORY } */
typedef enum {
  LV_MODE_HASH = 0,            /* iteration >= 1: highest community wins equal gains */
  LV_MODE_SORT = 1,            /* iteration >= 1: lowest community wins equal gains */
  LV_MODE_ADAPTIVE_SPEED = 2,  /* SORT rule for iterations <= 4, HASH rule after
                                  (phaseOptimization.cuh:125,135) */
  LV_MODE_ADAPTIVE_MEMORY = 3  /* HASH rule for optimisation, SORT-style aggregation
                                  (phaseOptimization.cuh:125,135; phaseAggregation.cuh:51) */
} lv_mode;

typedef enum { LV_MEM_HOST = 0, LV_MEM_DEVICE = 1 } lv_mem;

typedef enum {
  LV_WEIGHTS_AUTO = 0,     /* integer semantics when every weight is a non-negative integer */
  LV_WEIGHTS_INTEGER = 1,  /* reference semantics: u32 weights, exact sums */
  LV_WEIGHTS_FLOAT = 2     /* fp32 weights, double accumulation (no reference counterpart) */
} lv_weight_mode;

/* Runtime replacement for constants.h:6-20 (compile-time macros in the reference). */
typedef struct {
  int32_t mode;             /* lv_mode; default LV_MODE_SORT */
  int32_t fast_first;       /* iteration 0 of each level is the per-edge "fast" pass with the
                               v <= c gate (phaseOptimizationSort.cu:28-158,
                               phaseOptimizationUpdate.cu:99); default 1 */
  int32_t max_iterations;   /* EARLY_STOP_LIMIT (constants.h:16); default 1e9 */
  int32_t max_levels;       /* 0 = no limit (the reference has none) */
  double threshold;         /* MODULARITY_CONVERGED_THRESHOLD (constants.h:15); default 1e-3 */
  int64_t chunk_edges;      /* STEP_ROUND (constants.h:18); the reference ends a pass at the
                               first edge chunk with no selected edge
                               (phaseOptimizationSort.cu:81-86,235-240). 0 turns that
                               emulation off; default 50,000,000 */
  int32_t weight_mode;      /* lv_weight_mode; default LV_WEIGHTS_AUTO */
  int32_t validate;         /* 1 = check row_ptr monotone / col in range / no empty row on
                               the device before running (default 1) */
  int32_t use_graphs;       /* 1 = run the level loop (passes, aggregation, next level) as one
                               captured CUDA graph with device-side loop control, captured once
                               per context (or serving slot) and replayed (default);
                               0 = host-driven, one stream launch sequence per pass */
  int32_t refine;           /* 1 = refine each level's partition before aggregating it (a
                               Leiden-style refinement behind the reference's empty
                               RefinePhase hook, phaseRefine.cuh:1-3; no reference
                               counterpart). Host-driven runs only (use_graphs is ignored);
                               not available to the server or lv_community_resume. Default 0 */
  int32_t refine_passes;    /* refinement passes per level at most; 0 = until a pass raises the
                               refined partition's modularity by no more than `threshold` */
  int32_t reserved_i[5];
  /* degree-bin tiling; 0 = use the autotuned or built-in table */
  int32_t bin_max_degree[8];
  double refine_tolerance;  /* a refined level also continues while its aggregate graph has
                               fewer than refine_tolerance x n vertices (default 0.95) */
  double reserved_d[3];
} lv_config;

/* Per-run statistics (modularityAlgorithms.h:18-20,73-79 "Metrics" line and more). */
typedef struct {
  double modularity;        /* final Q, as Community::modularity (community.h:104) */
  int64_t n;                /* vertices of the input */
  int64_t m;                /* undirected edges of the input (graph.cu:48 n_links) */
  int32_t levels;           /* optimisation levels run */
  int32_t iterations;       /* optimisation passes over all levels */
  int32_t n_communities;    /* n_of_best_communities (community.h:23) */
  int32_t reserved0;
  float ms_total;           /* upload -> result, host-observed device time */
  float ms_window;          /* the reference's window: after the device graph build to the
                               end of the final aggregation (modularityAlgorithms.h:26,69-75) */
  float ms_optimization;    /* all optimisation passes */
  float ms_aggregation;     /* all aggregations */
  float ms_first_optimization;  /* opt0 of the Metrics line */
  float ms_first_aggregation;   /* agg0 of the Metrics line */
  double bytes_optimization;    /* algorithmic bytes of the optimisation kernels, summed over
                                   passes: 12 per active entry + 24 per active vertex */
  float ms_optimization_kernels;  /* device time of the optimisation kernels only (binning and
                                     gain evaluation, without apply / modularity) */
  int32_t reserved1;
  int64_t kernel_launches;      /* engine kernels launched by the call */
  int64_t active_entries;       /* sum over passes of the active vertices' entries */
  int64_t active_vertices;      /* sum over passes of the active vertices */
  int64_t graph_launches;       /* launches of the captured level loop (0: host-driven run;
                                   more than 1 when the run stopped to grow its hash arena) */
  int64_t refine_passes;        /* refinement passes over all levels (refine = 1) */
  int64_t reserved[1];
} lv_stats;

typedef struct lv_context lv_context;
typedef struct lv_community lv_community;

/* ---- context --------------------------------------------------------------------------
 * A context owns one device, its streams and a reusable device arena (the reference
 * re-allocates 6 x STEP_ROUND scratch vectors on every level, phaseOptimization.cuh:50-68).
 * Communities, ingested graphs and servers created on a context use it until they are
 * destroyed: destroy them before the context. */
void lv_config_default(lv_config* cfg);
lv_status lv_create(int32_t device, const lv_config* cfg, lv_context** out);
lv_status lv_destroy(lv_context* ctx);
const char* lv_last_error(const lv_context* ctx);
const char* lv_status_string(lv_status s);
int32_t lv_abi_version(void);

/* ---- one-shot runs ----------------------------------------------------------------------
 * lv_run_csr replaces ModularityAlgorithms::Louvain(GraphHost&, MODE)
 * (modularityAlgorithms.h:8-10,14-81): builds the device graph, runs every level, returns
 * best_communities (community.h:21, values 0..K-1 per input vertex), modularity and K.
 * out_comm is int32[n] in `out_mem` memory; out_modularity / stats may be NULL. */
lv_status lv_run_csr(lv_context* ctx, int64_t n, const int64_t* row_ptr, const int32_t* col,
                     const float* w, int32_t in_mem, int32_t* out_comm, int32_t out_mem,
                     double* out_modularity, lv_stats* stats);

/* Batched: n_graphs independent graphs packed into one CSR (vertex ranges
 * vtx_offsets[g]..vtx_offsets[g+1], col holds packed/global vertex IDs) run together in one
 * device-driven launch sequence. No reference counterpart (the reference runs one graph per
 * call, main.cu:19-39). out_comm int32[total n] holds per-graph community IDs 0..K_g-1;
 * out_modularity double[n_graphs] and out_ncomm int32[n_graphs] may be NULL. */
lv_status lv_run_batch(lv_context* ctx, int32_t n_graphs, const int64_t* vtx_offsets,
                       const int64_t* row_ptr, const int32_t* col, const float* w,
                       int32_t in_mem, int32_t* out_comm, int32_t out_mem,
                       double* out_modularity, int32_t* out_ncomm, lv_stats* stats);

/* Autotuner (no reference counterpart): times full runs of a sample -- one graph
 * (n_graphs = 1, vtx_offsets = {0, n}) or a packed batch -- under a fixed set of candidate
 * degree-bin tables (the boundaries that pick 4 / 8 / 16 / 32 lanes, a block or many blocks
 * per row, and with them each row's hash-table capacity): per candidate one untimed run
 * (which captures its level loop), then `trials` timed runs of the level loop alone; the
 * fastest candidate is kept if it beats the first (built-in) table by more than 3 %, else the
 * built-in table is kept. The chosen table becomes the context's cfg.bin_max_degree for later
 * runs and is returned in *out_cfg; *out_ms = its best run time. Results do not depend on the
 * table for integer weights (every table computes the same sums). */
lv_status lv_autotune(lv_context* ctx, int32_t n_graphs, const int64_t* vtx_offsets,
                      const int64_t* row_ptr, const int32_t* col, const float* w, int32_t in_mem,
                      int32_t trials, lv_config* out_cfg, double* out_ms);

/* ---- phase-level interface ----------------------------------------------------------------
 * The reference's own phase boundaries, so callers (and parity tests) can step a run pass
 * by pass the way modularity_routine does. */

/* Community(GraphHost&) (community.h:31-46): upload, build k, identity partition, Q. */
lv_status lv_community_create(lv_context* ctx, int64_t n, const int64_t* row_ptr,
                              const int32_t* col, const float* w, int32_t in_mem,
                              lv_community** out);
lv_status lv_community_destroy(lv_community* c);
/* Resume a run checkpointed at the start of a level (no reference counterpart; the reference
 * keeps nothing between levels but Community::best_communities and the contracted GraphDevice,
 * community.h:16-26). A checkpoint is what the getters below return at a level start:
 * lv_community_info (n0, level, weights_integer, and `iterations` = passes so far from
 * lv_stats or the trace), lv_community_get_graph (the level's CSR, weights as doubles) and
 * lv_community_get_best (each input vertex's vertex at this level). Host memory. The resumed
 * run continues exactly as the interrupted one would (integer weights: bit-identical). */
lv_status lv_community_resume(lv_context* ctx, int64_t n0, const int32_t* best, int32_t level,
                              int32_t iterations, int64_t n, const int64_t* row_ptr,
                              const int32_t* col, const double* w, int32_t weights_integer,
                              lv_community** out);
/* One OptimizationPhase::optimize() + Community::compute_modularity()
 * (phaseOptimization.cuh:116-155,171): returns Q_after - Q_before and the number of moves. */
lv_status lv_optimization_step(lv_community* c, double* delta_q, int64_t* n_moved);
/* OptimizationPhase::run (phaseOptimization.cuh:184-206): passes until dQ <= threshold. */
lv_status lv_optimization_run(lv_community* c, int32_t* iterations);
/* AggregationPhase::run(community, aggregate, mode) (phaseAggregation.cuh:19-190). */
lv_status lv_aggregation_run(lv_community* c, int32_t aggregate);
/* modularity_routine's level loop (modularityAlgorithms.h:31-67) on an existing community. */
lv_status lv_louvain(lv_community* c, lv_stats* stats);

typedef struct {
  int64_t n;            /* vertices of the current level */
  int64_t E;            /* directed entries of the current level */
  int64_t n0;           /* vertices of the input */
  int32_t level;
  int32_t iteration;    /* passes run in the current level */
  double modularity;    /* Community::modularity */
  double internal;      /* sum of w over entries with comm[src] == comm[dst] (community.h:87-100) */
  double sum_a2;        /* sum of squared community totals (community.h:71-83) */
  double total_weight;  /* m, fixed at level 0 (graph.cu:81) */
  int64_t n_best;       /* n_of_best_communities */
  int32_t weights_integer;
  int32_t reserved;
} lv_community_info;

lv_status lv_community_info_get(lv_community* c, lv_community_info* info);
/* communities (community.h:17) and communities_weight (community.h:18) of the current level,
 * copied to host buffers int32[n] / double[n]; either may be NULL. */
lv_status lv_community_get_partition(lv_community* c, int32_t* comm, double* totals);
/* best_communities (community.h:21): int32[n0] host buffer. */
lv_status lv_community_get_best(lv_community* c, int32_t* best);
/* The current level's graph (GraphDevice, graph.cuh:14-33) as host CSR: int64[n+1],
 * int32[E], double[E] weights and double[n] k (tot_weight_per_nodes); any may be NULL.
 * Rows come out sorted by destination, as the reference's sort_by_key leaves them. */
lv_status lv_community_get_graph(lv_community* c, int64_t* row_ptr, int32_t* col, double* w,
                                 double* k);

/* Per-pass record of a single-graph run: the (I, S, Q) triple compute_modularity prints
 * after every pass (community.h:102, phaseOptimization.cuh:174-177) plus the move count. */
typedef struct {
  int32_t level, iteration, n_moved, reserved;
  double internal, sum_a2, modularity, delta;
} lv_trace_record;

/* Copies up to `cap` records (oldest first) and sets *len to the number recorded. */
lv_status lv_community_get_trace(lv_community* c, lv_trace_record* out, int32_t cap, int32_t* len);

/* ---- allocation-free modularity ----------------------------------------------------------
 * No counterpart in the reference. For callers that may not allocate device memory when they
 * call (a framework that owns all of HBM through its own pool, a serving loop that must not
 * stall on cudaMalloc): Q = I/(2m) - S/(4 m m) of partition `comm` (int32[n], labels in
 * [0, n)) on the CSR graph, with every buffer in device memory. Uses only the caller's buffers
 * and one scratch array compiled into the library (LV_NOALLOC_MAX_VERTICES + 64 words of 8
 * bytes, held on each GPU that loads the library until the process exits); n above
 * LV_NOALLOC_MAX_VERTICES returns LV_ERR_RANGE before anything runs. Writes out[0..3] =
 * {Q, I, S, m} (device memory) asynchronously on `stream` (a cudaStream_t, NULL = default
 * stream). Checked on the device: a label or column outside [0, n), or with integer weights a
 * total weight 2m >= 2^32, makes Q and m NaN; weights summing to zero give m = 0 and Q NaN.
 * The first call on a device loads this entry point's module (CUDA loads modules lazily),
 * which reserves the scratch array and the kernels' code in device memory at that moment,
 * and looks up the array's address: make it before the caller's own pool claims the rest of
 * HBM and before any stream capture on that device. Calls that overlap on the GPU share the
 * scratch array and race. weights_integer != 0 (or w == NULL) sums exactly in u64 like
 * LV_WEIGHTS_INTEGER; otherwise in double. */
#define LV_NOALLOC_MAX_VERTICES 1048576
lv_status lv_modularity_noalloc(int64_t n, const int64_t* row_ptr, const int32_t* col, const float* w,
                                const int32_t* comm, int32_t weights_integer, double* out, void* stream);

/* ---- edge-list ingest --------------------------------------------------------------------
 * GraphHost(name, weighted = false, skip_line) (graph.cu:17-87, graph.cuh:60-91) on the GPU:
 * `text` is the file's bytes (host or device memory). The first `skip_line` lines are skipped;
 * the rest is read as whitespace-separated integers taken in pairs, ending at the first token
 * that is not an integer (an unpaired last token is dropped); distinct unordered pairs become
 * edges (a self-loop pair included), ids are renumbered as id - min_id and must be contiguous.
 * The result is the symmetric CSR the reference's GraphDevice holds (both directions, a
 * self-loop stored twice, rows sorted), kept on the device. Errors: LV_ERR_INPUT (no pair,
 * ids not contiguous), LV_ERR_RANGE (too large). */
typedef struct lv_ingest lv_ingest;
lv_status lv_ingest_edge_list(lv_context* ctx, const char* text, int64_t len, int32_t skip_line,
                              int32_t in_mem, lv_ingest** out);
/* n_nodes, n_links (graphHost.cuh:8-9), CSR entries (2 n_links), min_id (graphHost.cuh:11). */
lv_status lv_ingest_info(const lv_ingest* g, int64_t* n_nodes, int64_t* n_links, int64_t* entries,
                         int64_t* min_id);
/* row_ptr int64[n_nodes + 1], col int32[entries], into host or device memory. */
lv_status lv_ingest_copy_csr(const lv_ingest* g, int64_t* row_ptr, int32_t* col, int32_t out_mem);
/* lv_run_csr on the ingested graph without leaving the device. */
lv_status lv_ingest_run(lv_ingest* g, int32_t* out_comm, int32_t out_mem, double* out_modularity,
                        lv_stats* stats);
lv_status lv_ingest_destroy(lv_ingest* g);

/* ---- serving ---------------------------------------------------------------------------
 * Continuous batching with graph state resident in HBM. No reference counterpart.
 * Requests are admitted while the device memory they need fits `budget_bytes` and a slot is
 * free (1 <= max_slots <= 64); a free slot takes the request at the head of the queue and the
 * other queued small requests (up to 4M entries each) as one batch, and slots run concurrently
 * on their own streams. With cfg.use_graphs each slot replays one captured level loop. */
typedef struct lv_server lv_server;
lv_status lv_server_create(lv_context* ctx, int64_t budget_bytes, int32_t max_slots,
                           lv_server** out);
lv_status lv_server_destroy(lv_server* s);
/* Copies the request's host CSR (the caller may reuse its buffers at once) and queues it;
 * returns its id. */
lv_status lv_server_submit(lv_server* s, int64_t n, const int64_t* row_ptr, const int32_t* col,
                           const float* w, int64_t* request_id);
/* The same without the copy: the buffers are borrowed and must stay valid and unchanged until
 * lv_server_poll reports the request done (pinned host memory gives full-speed uploads). */
lv_status lv_server_submit_borrowed(lv_server* s, int64_t n, const int64_t* row_ptr,
                                    const int32_t* col, const float* w, int64_t* request_id);
/* Moves finished work forward; returns immediately. *n_done = finished requests so far. */
lv_status lv_server_progress(lv_server* s, int64_t* n_done, int64_t* n_inflight,
                             int64_t* n_queued);
/* If `request_id` has finished: copies its communities (int32[n]) and modularity, returns
 * LV_OK and sets *done = 1; otherwise *done = 0. latency_ms: submit -> completion. */
lv_status lv_server_poll(lv_server* s, int64_t request_id, int32_t* out_comm,
                         double* out_modularity, double* latency_ms, int32_t* done);
/* Blocks until every submitted request has finished. */
lv_status lv_server_drain(lv_server* s);

#ifdef __cplusplus
}
#endif

#endif /* LOUVAIN_B200_H */
