// Command-line drivers with the reference's argv and result-file layout, running
// every query through the engine's C ABI.
//
//   gst_cli <type> <path> <name> <k> <q_start> <q_end>          (type 1: no hop bound)
//   gst_cli <type> <path> <name> <k> <D> <q_start> <q_end>      (type 2: hop bound D)
//
// type 1 replaces code/TrimCDP-WB/src/GSTnonHop.cu:160-510 (argv :162-163, result
// file :241-243, row :493); type 2 replaces code/D-TrimCDP-WB/src/GPUHop.cu:96-273
// (argv :98-99, result file :157-159, row :262).  Inputs are the reference formats
// read by the reference drivers: <path><name>_beg_pos.bin / _csr.bin / _weight.bin,
// <path><name>.g and <path><name><k>.csv.  Output goes to
// <path>result/{TrimCDP-WB,D-TrimCDP-WB}_<name>_T<k>[_D<D>]_<start>-<end>.csv with the
// reference's columns; the cost column holds 100000 when a query has no solution,
// like the reference.  The time column is the engine's device time per query in
// seconds; the memory column is the number of tree edges.
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "gst.h"
#include "gst_io.h"

int main(int argc, char** argv) {
  if (argc < 7) {
    fprintf(stderr,
            "usage: %s 1 <path> <name> <k> <q_start> <q_end>\n"
            "       %s 2 <path> <name> <k> <D> <q_start> <q_end>\n",
            argv[0], argv[0]);
    return 2;
  }
  const int type = atoi(argv[1]);
  const std::string path = argv[2], name = argv[3];
  const int k = atoi(argv[4]);
  int D = -1, a = 5;
  if (type == 2) {
    if (argc < 8) return 2;
    D = atoi(argv[5]);
    a = 6;
  }
  const int q0 = atoi(argv[a]), q1 = atoi(argv[a + 1]);

  gst_host_graph hg{};
  if (gst_read_reference_bin(path.c_str(), name.c_str(), &hg)) {
    fprintf(stderr, "cannot read %s%s_{beg_pos,csr,weight}.bin\n", path.c_str(), name.c_str());
    return 1;
  }
  gst_host_groups hgr{};
  if (gst_read_reference_groups((path + name + ".g").c_str(), &hgr)) {
    fprintf(stderr, "cannot read %s%s.g\n", path.c_str(), name.c_str());
    return 1;
  }
  const std::string qfile = path + name + std::to_string(k) + ".csv";
  int32_t kk = 0;
  const int32_t nq = gst_read_reference_queries(qfile.c_str(), 0, &kk, nullptr);
  if (nq <= 0 || kk != k) {
    fprintf(stderr, "cannot read %d-group queries from %s\n", k, qfile.c_str());
    return 1;
  }
  std::vector<int32_t> qs((size_t)nq * k);
  gst_read_reference_queries(qfile.c_str(), nq, &kk, qs.data());

  gst_engine* eng = nullptr;
  gst_status st = gst_engine_create(0, nullptr, &eng);
  if (st != GST_OK) {
    fprintf(stderr, "engine: %s\n", gst_last_error_string(nullptr));
    return 1;
  }
  gst_graph* g = nullptr;
  gst_groups* grp = nullptr;
  if (gst_graph_create(eng, hg.V, hg.E, hg.beg_pos, hg.adj, hg.weight, &g) != GST_OK ||
      gst_groups_create(g, hgr.n_groups, hgr.grp_ptr, hgr.members, &grp) != GST_OK) {
    fprintf(stderr, "upload: %s\n", gst_last_error_string(eng));
    return 1;
  }
  const std::string prefix = type == 2 ? "D-TrimCDP-WB_" : "TrimCDP-WB_";
  std::string out = path + "result/" + prefix + name + "_T" + std::to_string(k) + "_";
  if (type == 2) out += "D" + std::to_string(D) + "_";
  out += std::to_string(q0) + "-" + std::to_string(q1) + ".csv";
  FILE* f = fopen(out.c_str(), "w");
  if (!f) {
    fprintf(stderr, "cannot write %s\n", out.c_str());
    return 1;
  }
  fprintf(f, "task_ID,task,%s_time,%s_cost,%s_memory,counts,process_num\n",
          type == 2 ? "GPU2_Hop" : "GPU2_nonHop", type == 2 ? "GPU2_Hop" : "GPU2_nonHop",
          type == 2 ? "GPU2_Hop" : "GPU2_nonHop");
  int rc = 0;
  for (int i = q0; i <= q1 && i < nq; i++) {
    gst_query q{k, &qs[(size_t)i * k], D, (uint64_t)i};
    gst_result r{};
    gst_status s = gst_solve(g, grp, &q, &r);
    std::string task;
    for (int j = 0; j < k; j++) task += std::to_string(qs[(size_t)i * k + j]) + " ";
    const int cost = s == GST_OK ? r.cost : 100000;
    if (s != GST_OK && s != GST_INFEASIBLE) {
      fprintf(stderr, "query %d: status %d: %s\n", i, (int)s, gst_last_error_string(eng));
      rc = 1;
    }
    fprintf(f, "%d,%s,%.8f,%d,%lld,%lld,%lld\n", i, task.c_str(), r.stats.device_ms / 1e3, cost,
            (long long)r.n_edges, (long long)r.stats.states_expanded,
            (long long)r.stats.levels);
    printf("query %d cost %d\n", i, cost);
    gst_result_free(&r);
  }
  fprintf(f, "\n");
  fclose(f);
  gst_groups_destroy(grp);
  gst_graph_destroy(g);
  gst_engine_destroy(eng);
  gst_host_graph_free(&hg);
  gst_host_groups_free(&hgr);
  return rc;
}
