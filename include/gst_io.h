/*
 * gst_io.h — host-side graph / group / query data for the GST engine:
 * reference file formats, seeded synthetic inputs, and the tree verifier.
 *
 * Everything here runs on the host and allocates with malloc; arrays returned
 * in the structs below are released with the matching *_free call.
 *
 * Reference formats (rucdatascience/GPU4GST-sigmod-fullEXP, README.md:58-74):
 *   <name>.in            text: "V E" then one "u v w" line per undirected edge;
 *                        read by code/PrunedDP++/include/graph_hash_of_mixed_weighted_read_for_GSTP.h:15-66
 *                        (both directions added, adjacency sorted by neighbour id)
 *   <name>_beg_pos.bin   int64[V+1]   CSR offsets, both directions
 *   <name>_csr.bin       int64[E]     neighbour ids
 *   <name>_weight.bin    int64[E]     edge weights
 *                        read by code/TrimCDP-WB/include/graph.hpp:12-112 (narrowed to int32)
 *   <name>.g             "g<id>:v v v" lines, 1-based group ids in file order;
 *                        read by code/TrimCDP-WB/include/read_group.hpp:9-54 (index = id-1)
 *   <name><k>.csv        one query per line: k 0-based group ids separated by spaces;
 *                        read by code/TrimCDP-WB/include/read_group.hpp:55-90
 */
#ifndef GST_IO_H
#define GST_IO_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* CSR graph with both directions stored; adjacency of each vertex sorted by id. */
typedef struct gst_host_graph {
  int64_t V;
  int64_t E;        /* directed entries = 2 x undirected edges */
  int64_t* beg_pos; /* V+1 */
  int32_t* adj;     /* E   */
  int32_t* weight;  /* E   */
} gst_host_graph;

/* Vertex groups: members of group g are members[grp_ptr[g] .. grp_ptr[g+1]), sorted. */
typedef struct gst_host_groups {
  int32_t n_groups;
  int64_t* grp_ptr; /* n_groups+1 */
  int32_t* members;
} gst_host_groups;

void gst_host_graph_free(gst_host_graph* g);
void gst_host_groups_free(gst_host_groups* g);

/* ---- synthetic inputs (no counterpart in the reference; they stand in for its
 *      datasets, which are not distributed with it) ------------------------ */

/* Barabasi-Albert: a (m+1)-clique, then each new vertex attaches to m distinct
 * existing vertices chosen proportionally to degree.  Weights uniform in
 * [wmin,wmax] per undirected edge (mirrored).  Returns 0 on success. */
int gst_synth_ba(int64_t V, int32_t m, uint64_t seed, int32_t wmin, int32_t wmax,
                 gst_host_graph* out);

/* R-MAT (a,b,c, d=1-a-b-c) on scale = ceil(log2 V) with ids >= V rejected, self
 * loops rejected, duplicate undirected edges removed, until n_undirected distinct
 * edges; if keep_lcc, only the largest connected component is kept and its
 * vertices relabelled in increasing original id.  Deterministic for a seed,
 * independent of the number of host threads. */
int gst_synth_rmat(int64_t V, int64_t n_undirected, double a, double b, double c,
                   uint64_t seed, int32_t wmin, int32_t wmax, int32_t keep_lcc,
                   gst_host_graph* out);

/* Groups with sizes uniform in [smin,smax]; members uniform without replacement. */
int gst_synth_groups_uniform(int64_t V, int32_t n_groups, int32_t smin, int32_t smax,
                             uint64_t seed, gst_host_groups* out);

/* Groups with sizes drawn from Zipf(s) on {1,2,...} then clamped to [smin,smax]. */
int gst_synth_groups_zipf(int64_t V, int32_t n_groups, double s, int32_t smin,
                          int32_t smax, uint64_t seed, gst_host_groups* out);

/* n_queries queries of k distinct group ids uniform in [0,n_groups); writes
 * n_queries*k ids row-major into out. */
int gst_synth_queries(int32_t n_groups, int32_t n_queries, int32_t k, uint64_t seed,
                      int32_t* out);

/* ---- reference formats -------------------------------------------------- */

/* Write <dir>/<name>.in, _beg_pos.bin, _csr.bin, _weight.bin, .g and, when
 * n_queries > 0, <name><k>.csv.  Returns 0 on success. */
int gst_write_reference_files(const char* dir, const char* name, const gst_host_graph* g,
                              const gst_host_groups* groups, int32_t n_queries, int32_t k,
                              const int32_t* queries);

/* Read the int64 CSR triple <dir>/<name>_beg_pos.bin/_csr.bin/_weight.bin. */
int gst_read_reference_bin(const char* dir, const char* name, gst_host_graph* out);

/* Read <dir>/<name>.in (adds both directions, sorts adjacency, like the reference). */
int gst_read_reference_in(const char* path, gst_host_graph* out);

/* Read a .g group file. */
int gst_read_reference_groups(const char* path, gst_host_groups* out);

/* Read a <name><k>.csv query file: returns the number of queries, writes at most
 * max_queries*k ids into out; k_out receives the ids per line.  -1 on error. */
int32_t gst_read_reference_queries(const char* path, int32_t max_queries, int32_t* k_out,
                                   int32_t* out);

/* ---- tree verifier ------------------------------------------------------- */

/* Checks that the edge list (u[i],v[i],w[i]) is a connected subgraph of g whose
 * vertex set covers every queried group, that each edge exists in g with that
 * weight, that the sum of weights equals `cost`, that the edge set has no
 * cycle, and, if hop_bound >= 0, that its diameter in hops is <= hop_bound.
 * A single-vertex tree is passed as n_edges = 0 with root_vertex set.
 * Returns 0 if all hold, otherwise a positive code naming the first failure:
 *   1 edge not in graph / wrong weight, 2 disconnected, 3 group not covered,
 *   4 weight sum != cost, 5 diameter > hop_bound, 6 cycle, 7 bad argument.
 * Mirrors the feasibility test of code/PrunedDP++/include/exp_CPU_nonHop.h:17-49
 * and adds the cost, acyclicity and hop checks. */
int32_t gst_verify_tree(const gst_host_graph* g, const gst_host_groups* groups,
                        int32_t k, const int32_t* group_ids, int32_t hop_bound,
                        int64_t cost, int64_t n_edges, const int32_t* u, const int32_t* v,
                        const int32_t* w, int32_t root_vertex);

#ifdef __cplusplus
}
#endif
#endif /* GST_IO_H */
