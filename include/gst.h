/*
 * gst.h — C ABI of the B200 group Steiner tree (GST) engine.
 *
 * One engine is bound to one CUDA device.  A graph is uploaded once and stays
 * resident in HBM; vertex groups are registered against it; queries name k
 * groups (and optionally a hop / diameter bound D) and return the optimal tree
 * cost and the tree's edge set.  Every entry point returns a gst_status; no entry
 * point exits the process or falls back to a CPU solver.
 *
 * What each entry point replaces in the reference (rucdatascience/GPU4GST-sigmod-fullEXP),
 * whose only interface is a per-experiment executable:
 *   gst_graph_create      graph<> ctor + gpu_graph upload: code/TrimCDP-WB/include/graph.hpp:12-126,
 *                         code/TrimCDP-WB/include/gpu_graph.cuh:35-90 (int64 files narrowed to int32)
 *   gst_graph_create_i64  the same, taking the int64 _beg_pos/_csr/_weight.bin arrays as read
 *                         (code/TrimCDP-WB/include/graph.hpp:25-112)
 *   gst_groups_create     read_Group: code/TrimCDP-WB/include/read_group.hpp:9-54
 *                         (group id in a query = .g id - 1)
 *   gst_solve (D < 0)     per-query body of code/TrimCDP-WB/src/GSTnonHop.cu:247-497
 *                         (set_max_ID init, one-label SSSP, lb tables, balanced_push, min over V)
 *   gst_solve (D >= 0)    per-query body of code/D-TrimCDP-WB/src/GPUHop.cu:172-266 with the
 *                         answer semantics of code/D-PrunedDP++/include/CPUHOP.h:146-225
 *                         (minimum over every d <= D)
 *   gst_solve_batch       the q_start..q_end loop of the same drivers (GSTnonHop.cu:247,
 *                         GPUHop.cu:172), run as one batched device loop
 *   result edge set       code/PrunedDP++/include/CPUNONHOP.h:387-429 (build_tree) and
 *                         code/D-PrunedDP++/include/CPUHOP.h:231-257 — the reference GPU
 *                         engines return the cost only
 *   gst_status codes      exit()/assert paths of code/TrimCDP-WB/include/util.h:5-16 and
 *                         read_group.hpp:47-52; INFEASIBLE replaces the 100000 sentinel
 *                         (code/TrimCDP-WB/include/header.h:13)
 */
#ifndef GST_H
#define GST_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum gst_status {
  GST_OK = 0,
  GST_INFEASIBLE = 1,     /* the queried groups cannot be connected (reference: cost 100000) */
  GST_OOM_ADMISSION = 2,  /* the query's state table does not fit the device memory budget */
  GST_BAD_INPUT = 3,      /* malformed graph, groups or query */
  GST_TIMEOUT = 4,        /* the query exceeded its level budget */
  GST_DEVICE_ERROR = 5,   /* a CUDA call failed or a kernel reported an error */
  GST_CAPACITY = 6,       /* a device worklist overflowed its capacity */
  GST_NOT_READY = 7       /* serving: the polled query has not finished */
} gst_status;

typedef struct gst_engine gst_engine;
typedef struct gst_graph gst_graph;
typedef struct gst_groups gst_groups;
typedef struct gst_server gst_server;

/* Engine tunables; zero fields take defaults (gst_config_default). */
typedef struct gst_config {
  int64_t mem_budget_bytes;   /* HBM the engine may use for query state; 0 = 85% of free */
  int32_t split_degree;       /* edges per grow work item: hubs split into chunks of this size */
  int32_t bucket_delta;       /* cost-bucket width of the frontier ordering; 0 = one bucket
                                 (no ordering; the distance search of unbounded queries then
                                 runs one item per vertex and group mask) */
  int32_t max_levels;         /* per-query level budget (GST_TIMEOUT beyond) */
  int32_t threads_per_block;  /* CTA size of the rows (merge) kernel, 64..256 */
  int32_t blocks_per_sm;      /* resident CTAs per SM for the level kernels */
  int32_t max_batch;          /* queries resident at once in gst_solve_batch / serving */
  int32_t use_graphs;         /* 1 (default): run the level loop as a CUDA graph whose
                                 conditional WHILE node repeats the level body on the device
                                 until a query finishes; ignored while profile_kernels != 0 */
  int32_t profile_kernels;    /* bit0 grow, bit1 rows, bit2 sssp, bit3 the shared search's relax
                                 steps: bracket those launches with CUDA events and report
                                 their summed device time */
  int32_t verbose;
  int32_t hop_cut_mult;       /* hop-bounded queries: the distance search stops at this
                                 multiple of the star bound (0 = 1); larger prunes more
                                 DP states and costs a longer search */
  int32_t search_cut_permille; /* unbounded queries: the distance search stops at this
                                 many thousandths of the star bound (0 = 1000); less
                                 searches fewer vertices and leaves weaker, still exact
                                 bounds to the DP (the autotuner chooses it) */
  int32_t hop_cut_permille;   /* hop-bounded queries: the same in thousandths (0: use
                                 hop_cut_mult x 1000) */
  int32_t batch_search;       /* 1 (default): gst_solve, gst_solve_batch and the server
                                 search the distances of their waiting queries' groups
                                 together, one search per kind (unbounded, or one hop bound
                                 <= 8), up to 256 groups and 64 queries at a time (one
                                 relaxation of an edge serves every group that improved at
                                 its source; a lone query runs the same kernels); 0: every
                                 query runs its own group-mask search */
} gst_config;

typedef struct gst_query {
  int32_t k;                /* number of groups, 1..8 */
  const int32_t* group_ids; /* k distinct group ids (0-based, as in <name><k>.csv) */
  int32_t hop_bound;        /* D >= 0: diameter-bounded query; < 0: no bound */
  uint64_t user_tag;        /* returned unchanged in the result */
} gst_query;

typedef struct gst_stats {
  int64_t levels;           /* DP levels (grow+merge rounds), all phases */
  int64_t states_expanded;  /* grow work items processed (state x edge chunk) */
  int64_t edge_relaxations; /* grow relaxations attempted */
  int64_t merge_pairs;      /* merge pairs evaluated */
  int64_t rows_merged;      /* vertex rows run through the merge closure */
  int64_t sssp_relaxations; /* one-label distance relaxations */
  int64_t kernel_launches;  /* engine kernels launched (batch: for the whole batch) */
  int64_t h2d_bytes;        /* host->device bytes moved for the call (batch: whole batch) */
  int64_t d2h_bytes;        /* device->host bytes moved for the call (batch: whole batch) */
  double device_ms;         /* device time of the query (batch: of the whole batch) */
  double latency_ms;        /* host time from the call's start to this result being ready */
  double grow_ms;           /* profiled device time of the grow / rows / sssp launches */
  double rows_ms;           /*   (batch totals; 0 unless cfg.profile_kernels selects them) */
  double sssp_ms;
  int64_t queue_max;        /* largest worklist fill of the query (items) */
  int64_t grow_launches;    /* profiled launches behind grow_ms / rows_ms / sssp_ms */
  int64_t rows_launches;
  int64_t sssp_launches;
  int64_t shared_sectors;   /* batch-shared distance search of the call: target-row sectors
                               read (edges x active 8-group sectors), */
  double shared_ms;         /*   its device time, */
  int64_t shared_launches;  /*   and its kernel launches, */
  int64_t shared_relax_launches; /* of which relax steps (k_bs_relax), */
  double shared_relax_ms;   /*   their device time (0 unless profile_kernels bit3) */
} gst_stats;

typedef struct gst_result {
  int32_t status;     /* gst_status of this query */
  int32_t cost;       /* optimal cost (valid when status == GST_OK) */
  int32_t root;       /* root vertex of the DP state holding the optimum */
  int32_t root_hop;   /* hop index of that state (0 for unbounded queries) */
  int64_t n_edges;    /* tree edges (duplicates removed) */
  int32_t* edge_u;    /* engine-allocated, released by gst_result_free */
  int32_t* edge_v;
  int32_t* edge_w;
  uint64_t user_tag;
  gst_stats stats;
} gst_result;

void gst_config_default(gst_config* cfg);
/* Change cfg.profile_kernels of a live engine (bit0 grow, bit1 rows, bit2 sssp, bit3 the
 * shared search's relax steps); the next solve brackets those launches with CUDA events
 * (and runs the level loop without the CUDA graph while any bit is set). */
gst_status gst_engine_set_profiling(gst_engine* eng, int32_t bits);

gst_status gst_engine_create(int32_t device, const gst_config* cfg, gst_engine** out);
/* Refuses (GST_BAD_INPUT) while graphs of the engine are alive: destroy them first. */
gst_status gst_engine_destroy(gst_engine* eng);
/* Message of the last failure on this engine (thread-local copy; never NULL). */
const char* gst_last_error_string(gst_engine* eng);

/* Graph in CSR with both directions stored (beg_pos[V+1], csr[E], weight[E]);
 * weights must be >= 1.  The caller keeps ownership of its arrays; the engine
 * copies them to the device (adjacency sorted per vertex, vertices renumbered by
 * degree so that high-degree vertices share cache lines; group members and every
 * result are translated, so callers only ever see their own vertex ids). */
gst_status gst_graph_create(gst_engine* eng, int64_t V, int64_t E, const int64_t* beg_pos,
                            const int32_t* csr, const int32_t* weight, gst_graph** out);
gst_status gst_graph_create_i64(gst_engine* eng, int64_t V, int64_t E, const int64_t* beg_pos,
                                const int64_t* csr, const int64_t* weight, gst_graph** out);
gst_status gst_graph_destroy(gst_graph* g);

/* Groups: members of group g are members[grp_ptr[g] .. grp_ptr[g+1]). */
gst_status gst_groups_create(gst_graph* g, int32_t n_groups, const int64_t* grp_ptr,
                             const int32_t* members, gst_groups** out);
gst_status gst_groups_destroy(gst_groups* grp);

/* One-label distance cache for serving hot groups (no counterpart in the reference,
 * which recomputes a group's distances for every query: mapper_enactor.cuh:249-366).
 * A group's distances to every vertex depend on the group only.  This computes them,
 * without cutoff, for each listed group not yet cached and keeps them on the device,
 * up to max_bytes (4 x V bytes per group; when the list holds more groups than fit,
 * the first ones are kept; groups of earlier calls that this call does not list are
 * replaced least recently used first).  Unbounded queries whose groups are all cached
 * then skip the distance search; with some of their groups cached, the search runs for
 * the others only.  A different max_bytes drops the cache first;
 * max_bytes = 0 frees it.  *n_cached (optional) = listed groups now cached. */
gst_status gst_groups_cache_warm(gst_groups* grp, int32_t n, const int32_t* group_ids,
                                 int64_t max_bytes, int32_t* n_cached);
/* The same for queries with hop bound hop_bound (1..30): per group, the cheapest paths
 * of at most h edges to every vertex for every hop budget the engine bounds with
 * (4 x V x (min(hop_bound-1, 7) + 1) bytes per group).  A hop-bounded query with that
 * bound whose groups are all cached skips the distance search; with some cached, the
 * search runs for the others only.  One hop bound at a time: warming with another (or
 * another max_bytes) drops the hop cache first. */
gst_status gst_groups_cache_warm_hop(gst_groups* grp, int32_t n, const int32_t* group_ids,
                                     int32_t hop_bound, int64_t max_bytes, int32_t* n_cached);

/* One query, synchronous.  Fills *res (call gst_result_free afterwards). */
gst_status gst_solve(gst_graph* g, gst_groups* grp, const gst_query* q, gst_result* res);

/* n queries, run as one batched device loop with up to cfg.max_batch resident at
 * once; results[i] belongs to queries[i].  Returns GST_OK when every query got a
 * status (per-query statuses are in the results). */
gst_status gst_solve_batch(gst_graph* g, gst_groups* grp, int32_t n, const gst_query* queries,
                           gst_result* results);

void gst_result_free(gst_result* res);

/* Autotuner (no counterpart in the reference, whose launch shapes are compile-time
 * constants: BLKS_NUM / THDS_NUM in code/TrimCDP-WB/include/header.h and the 1024/512
 * virtual-split degrees of graph.hpp:128-378).  Times the engine on the sample
 * queries under candidate CTA sizes, hub-split (work chunk) sizes, cost-bucket
 * widths, CTAs per SM and numbers of resident queries (at most cfg.max_batch), one
 * parameter at a time, keeps the fastest setting in
 * the engine, and appends it to the text file cache_path (NULL: no cache) under a
 * key of the graph's shape (V, E, max degree, max weight, batch size, SM count).  A
 * later call with a cached shape applies the cached setting without timing
 * anything.  Every candidate must reproduce the sample's optimal costs, else
 * GST_DEVICE_ERROR.  *chosen (may be NULL) receives the engine's new configuration. */
gst_status gst_autotune(gst_graph* g, gst_groups* grp, int32_t n, const gst_query* sample,
                        const char* cache_path, gst_config* chosen);

/* Serving (no counterpart in the reference, whose drivers run a fixed query list;
 * this replaces the q_start..q_end loop of GSTnonHop.cu:247 / GPUHop.cu:172 for
 * queries that arrive over time).  A server owns a host thread and a set of query
 * slots on the engine's device.  Submitted queries wait in arrival order until a
 * slot and the HBM of their state table (2^k x (D+1) x V x 8 bytes plus worklists,
 * within cfg.mem_budget_bytes) are free, and are folded into the running batch at
 * the next DP-level boundary, alongside queries already on the GPU.  Each result is
 * the same as gst_solve's for that query. */
gst_status gst_server_create(gst_graph* g, gst_groups* grp, gst_server** out);
/* Queue one query (copied); *ticket names it in gst_poll / gst_wait.  A malformed
 * query is accepted and completes at once with GST_BAD_INPUT. */
gst_status gst_submit(gst_server* s, const gst_query* q, uint64_t* ticket);
/* GST_NOT_READY while the query runs; otherwise fills *res (release it with
 * gst_result_free), forgets the ticket and returns the query's status. */
gst_status gst_poll(gst_server* s, uint64_t ticket, gst_result* res);
/* Like gst_poll, but blocks until the query has finished. */
gst_status gst_wait(gst_server* s, uint64_t ticket, gst_result* res);
/* Finishes every submitted query, then stops the server's thread and frees its
 * slots.  Results not taken are released. */
gst_status gst_server_destroy(gst_server* s);

/* Diagnostics (no counterpart in the reference): copy the first n_cells packed
 * state cells (cost<<32 | pending<<31 | parent) of a query slot's row pool (rows of
 * 2^k x (D+1) cells in the order the query's vertices took them) and the packed
 * best full-set state (cost<<32 | hop<<27 | vertex) of the query last run in it; vertices
 * here are in the engine's device numbering (by degree, highest first, ties by id). */
gst_status gst_debug_slot_state(gst_graph* g, int32_t slot, uint64_t* cells, int64_t n_cells,
                                uint64_t* best_out);

/* No-allocation solve (no counterpart in the reference; added for callers that
 * may not allocate device memory).  Some hosts own all device memory through their
 * own pool (a database's GPU memory manager, a framework's caching allocator, a
 * serving process that carves HBM up front) and forbid a library from calling
 * cudaMalloc/cudaFree, which would also synchronise the device under their other
 * work.  This entry point runs one query with the same kernels and pruning as
 * gst_solve but allocates nothing: the graph (d_beg_pos[V+1]; d_edges[2E] =
 * neighbour, weight interleaved, sorted by neighbour per vertex, weights >= 1) and
 * the groups (d_grp_ptr[n_groups+1], d_members) are the caller's, already in device
 * memory; the tree is written into the caller's host arrays res->edge_u/edge_v/edge_w
 * of edge_cap entries each (do not call gst_result_free on this result; a tree of
 * more distinct edges than edge_cap returns GST_CAPACITY).  All scratch lives in a
 * static device array of GST_NOALLOC_SCRATCH_BYTES that the library holds on every
 * GPU that loads it until the process exits; a query whose state table and worklists
 * do not fit is rejected with GST_OOM_ADMISSION (about V <= 150k vertices at k = 3,
 * fewer for larger k and hop bounds).  Without the caller's light-edge index every
 * relaxation reads a vertex's whole edge list, so large graphs run slower than with
 * gst_solve.  The first call on a device looks the array's address up and creates two
 * timing events (issue it before any stream capture).  Calls share the array, which
 * keeps the previous call's contents (each call clears what must start empty): work
 * of two calls that overlapped on one GPU would race, so the library serialises its
 * calls with a process-wide lock and each call returns only after its GPU work is
 * done.  `stream` is a cudaStream_t (NULL = legacy default stream).  Every failure
 * is also stored in res->status; the caller's current device is left as it was. */
#define GST_NOALLOC_SCRATCH_BYTES (64ll << 20)
gst_status gst_solve_noalloc(int32_t device, void* stream, int64_t V, int64_t E,
                             const int64_t* d_beg_pos, const int32_t* d_edges, int32_t n_groups,
                             const int64_t* d_grp_ptr, const int32_t* d_members,
                             const gst_query* q, int64_t edge_cap, gst_result* res);

/* Memory-system probe (no counterpart in the reference): the random-access rates that
 * bound the engine's kernels, measured on `device` with an array of `bytes` (>= 256 MB;
 * allocated and freed by the call).  *gather_dram: uniformly random 32-byte row reads per
 * second from the whole array; *gather_l2: the same within 32 MB (an L2-resident set);
 * *red_dram: random 4-byte atomicMin reductions per second over the whole array.  Every
 * relaxation of the engine reads a random target's distance row or state cell, so these,
 * not the streaming copy bandwidth, are the ceilings of its level kernels. */
gst_status gst_probe_random_access(int32_t device, int64_t bytes, double* gather_dram,
                                   double* gather_l2, double* red_dram);

#ifdef __cplusplus
}
#endif
#endif /* GST_H */
