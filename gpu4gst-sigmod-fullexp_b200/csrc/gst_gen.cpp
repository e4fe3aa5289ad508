// gst_gen: write a seeded synthetic workload in the reference's file formats.
//
//   gst_gen <dir> <name> rmat <V> <E> <seed> | ba <V> <m> <seed>
//           zipf <n> <s> <smin> <smax> <seed> | uniform <n> <smin> <smax> <seed>
//           [pool <k> <n> <seed>]...
//
// Writes <dir>/<name>.in, <name>_beg_pos.bin, _csr.bin, _weight.bin and <name>.g
// (README.md:58-74 of the reference), and for every `pool` the query pool of that
// k as <dir>/<name>_pool<k>.txt, one query of k group ids per line.  The graph,
// groups and queries are those of gst_synth_rmat / gst_synth_ba,
// gst_synth_groups_zipf / _uniform and gst_synth_queries with the same arguments
// (largest component kept for R-MAT), so a workload generated here is the one the
// engine solves.  This is a standalone program built from the generator and IO
// sources only: timing the reference's CPU solvers on a workload needs none of the
// engine's code in the process.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "gst_io.h"

static int usage() {
  fprintf(stderr,
          "usage: gst_gen <dir> <name> rmat <V> <E> <seed> | ba <V> <m> <seed>\n"
          "               zipf <n> <s> <smin> <smax> <seed> | uniform <n> <smin> <smax> <seed>\n"
          "               [pool <k> <n> <seed>]...\n");
  return 2;
}

int main(int argc, char** argv) {
  if (argc < 4) return usage();
  const std::string dir = argv[1], name = argv[2];
  int i = 3;
  gst_host_graph g{};
  auto need = [&](int n) { return i + n <= argc; };
  if (!strcmp(argv[i], "rmat") && need(4)) {
    if (gst_synth_rmat(atoll(argv[i + 1]), atoll(argv[i + 2]), 0.57, 0.19, 0.19,
                       strtoull(argv[i + 3], nullptr, 10), 1, 100, 1, &g))
      return fprintf(stderr, "gst_gen: bad R-MAT arguments\n"), 1;
    i += 4;
  } else if (!strcmp(argv[i], "ba") && need(4)) {
    if (gst_synth_ba(atoll(argv[i + 1]), atoi(argv[i + 2]), strtoull(argv[i + 3], nullptr, 10), 1,
                     100, &g))
      return fprintf(stderr, "gst_gen: bad BA arguments\n"), 1;
    i += 4;
  } else {
    return usage();
  }
  gst_host_groups grp{};
  if (i < argc && !strcmp(argv[i], "zipf") && need(6)) {
    if (gst_synth_groups_zipf(g.V, atoi(argv[i + 1]), atof(argv[i + 2]), atoi(argv[i + 3]),
                              atoi(argv[i + 4]), strtoull(argv[i + 5], nullptr, 10), &grp))
      return fprintf(stderr, "gst_gen: bad Zipf group arguments\n"), 1;
    i += 6;
  } else if (i < argc && !strcmp(argv[i], "uniform") && need(5)) {
    if (gst_synth_groups_uniform(g.V, atoi(argv[i + 1]), atoi(argv[i + 2]), atoi(argv[i + 3]),
                                 strtoull(argv[i + 4], nullptr, 10), &grp))
      return fprintf(stderr, "gst_gen: bad uniform group arguments\n"), 1;
    i += 5;
  } else {
    return usage();
  }
  if (int rc = gst_write_reference_files(dir.c_str(), name.c_str(), &g, &grp, 0, 0, nullptr)) {
    fprintf(stderr, "gst_gen: writing the reference files failed (%d)\n", rc);
    return 1;
  }
  while (i < argc) {
    if (strcmp(argv[i], "pool") || !need(4)) return usage();
    const int k = atoi(argv[i + 1]), n = atoi(argv[i + 2]);
    const uint64_t seed = strtoull(argv[i + 3], nullptr, 10);
    std::vector<int32_t> q((size_t)n * (size_t)k);
    if (gst_synth_queries(grp.n_groups, n, k, seed, q.data()))
      return fprintf(stderr, "gst_gen: bad query pool arguments\n"), 1;
    const std::string path = dir + "/" + name + "_pool" + std::to_string(k) + ".txt";
    FILE* f = fopen(path.c_str(), "w");
    if (!f) return fprintf(stderr, "gst_gen: cannot write %s\n", path.c_str()), 1;
    for (int r = 0; r < n; r++) {
      for (int j = 0; j < k; j++) fprintf(f, "%s%d", j ? " " : "", q[(size_t)r * k + j]);
      fprintf(f, "\n");
    }
    fclose(f);
    i += 4;
  }
  printf("V %lld E %lld groups %d\n", (long long)g.V, (long long)g.E, grp.n_groups);
  gst_host_graph_free(&g);
  gst_host_groups_free(&grp);
  return 0;
}
