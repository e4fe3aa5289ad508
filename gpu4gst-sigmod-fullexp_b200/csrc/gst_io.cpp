// Reference file formats (readers and writers) and the host-side tree verifier.
// Formats follow the reference README.md:58-74; the readers accept what the
// reference's own readers accept (trailing space on a line, "g<id>:" prefix).
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <queue>
#include <sstream>
#include <string>
#include <sys/stat.h>
#include <unordered_map>
#include <unordered_set>
#include <utility>
#include <vector>

#include "gst_io.h"

namespace {

template <class T>
T* dup_array(const std::vector<T>& v) {
  T* p = (T*)malloc(sizeof(T) * (v.size() ? v.size() : 1));
  if (p && !v.empty()) memcpy(p, v.data(), sizeof(T) * v.size());
  return p;
}

int64_t file_size(const std::string& f) {
  struct stat st;
  if (stat(f.c_str(), &st) != 0) return -1;
  return (int64_t)st.st_size;
}

bool write_i64(const std::string& path, const std::vector<int64_t>& v) {
  FILE* f = fopen(path.c_str(), "wb");
  if (!f) return false;
  size_t n = v.empty() ? 0 : fwrite(v.data(), sizeof(int64_t), v.size(), f);
  fclose(f);
  return n == v.size();
}

bool read_i64(const std::string& path, std::vector<int64_t>& v) {
  int64_t sz = file_size(path);
  if (sz < 0 || sz % 8) return false;
  v.resize((size_t)(sz / 8));
  FILE* f = fopen(path.c_str(), "rb");
  if (!f) return false;
  size_t n = v.empty() ? 0 : fread(v.data(), sizeof(int64_t), v.size(), f);
  fclose(f);
  return n == v.size();
}

}  // namespace

extern "C" {

int gst_write_reference_files(const char* dir, const char* name, const gst_host_graph* g,
                              const gst_host_groups* groups, int32_t n_queries, int32_t k,
                              const int32_t* queries) {
  if (!dir || !name || !g) return 1;
  const std::string base = std::string(dir) + "/" + name;
  {
    // .in lists each undirected edge once (u < v); the reference reader mirrors it
    FILE* f = fopen((base + ".in").c_str(), "w");
    if (!f) return 2;
    fprintf(f, "%lld %lld\n", (long long)g->V, (long long)(g->E / 2));
    for (int64_t u = 0; u < g->V; u++)
      for (int64_t i = g->beg_pos[u]; i < g->beg_pos[u + 1]; i++)
        if (u < g->adj[i]) fprintf(f, "%lld %d %d\n", (long long)u, g->adj[i], g->weight[i]);
    fclose(f);
  }
  std::vector<int64_t> beg(g->beg_pos, g->beg_pos + g->V + 1);
  std::vector<int64_t> adj(g->adj, g->adj + g->E), wt(g->weight, g->weight + g->E);
  if (!write_i64(base + "_beg_pos.bin", beg) || !write_i64(base + "_csr.bin", adj) ||
      !write_i64(base + "_weight.bin", wt))
    return 3;
  if (groups) {
    FILE* f = fopen((base + ".g").c_str(), "w");
    if (!f) return 4;
    for (int32_t gi = 0; gi < groups->n_groups; gi++) {
      fprintf(f, "g%d:", gi + 1);
      for (int64_t j = groups->grp_ptr[gi]; j < groups->grp_ptr[gi + 1]; j++)
        fprintf(f, "%s%d", j == groups->grp_ptr[gi] ? "" : " ", groups->members[j]);
      fprintf(f, "\n");
    }
    fclose(f);
  }
  if (n_queries > 0 && queries) {
    FILE* f = fopen((base + std::to_string(k) + ".csv").c_str(), "w");
    if (!f) return 5;
    for (int32_t q = 0; q < n_queries; q++) {
      for (int32_t j = 0; j < k; j++) fprintf(f, "%s%d", j ? " " : "", queries[(int64_t)q * k + j]);
      fprintf(f, "\n");
    }
    fclose(f);
  }
  return 0;
}

int gst_read_reference_bin(const char* dir, const char* name, gst_host_graph* out) {
  if (!dir || !name || !out) return 1;
  const std::string base = std::string(dir) + "/" + name;
  std::vector<int64_t> beg, adj, wt;
  if (!read_i64(base + "_beg_pos.bin", beg) || beg.size() < 2) return 2;
  if (!read_i64(base + "_csr.bin", adj)) return 3;
  if (!read_i64(base + "_weight.bin", wt)) return 4;
  const int64_t V = (int64_t)beg.size() - 1, E = beg[V];
  if ((int64_t)adj.size() < E || (int64_t)wt.size() < E || E < 0) return 5;
  std::vector<int32_t> a32((size_t)E), w32((size_t)E);
  for (int64_t i = 0; i < E; i++) {
    if (adj[i] < 0 || adj[i] >= V) return 6;
    a32[i] = (int32_t)adj[i];
    w32[i] = (int32_t)wt[i];
  }
  out->V = V;
  out->E = E;
  out->beg_pos = dup_array(beg);
  out->adj = dup_array(a32);
  out->weight = dup_array(w32);
  return 0;
}

int gst_read_reference_in(const char* path, gst_host_graph* out) {
  if (!path || !out) return 1;
  std::ifstream f(path);
  if (!f.is_open()) return 2;
  std::string line;
  if (!std::getline(f, line)) return 3;
  long long V = 0;
  {
    std::istringstream ss(line);
    double vd = 0;
    if (!(ss >> vd)) return 3;
    V = (long long)vd;
  }
  if (V < 1 || V > INT32_MAX) return 3;
  std::vector<std::vector<std::pair<int32_t, int32_t>>> al((size_t)V);
  while (std::getline(f, line)) {
    std::istringstream ss(line);
    long long a, b, w;
    if (!(ss >> a >> b >> w)) continue;
    if (a < 0 || b < 0 || a >= V || b >= V) return 4;
    al[a].push_back({(int32_t)b, (int32_t)w});
    al[b].push_back({(int32_t)a, (int32_t)w});
  }
  std::vector<int64_t> beg((size_t)V + 1, 0);
  for (long long v = 0; v < V; v++) {
    std::sort(al[v].begin(), al[v].end());
    beg[v + 1] = beg[v] + (int64_t)al[v].size();
  }
  std::vector<int32_t> adj((size_t)beg[V]), wt((size_t)beg[V]);
  for (long long v = 0; v < V; v++)
    for (size_t j = 0; j < al[v].size(); j++) {
      adj[beg[v] + j] = al[v][j].first;
      wt[beg[v] + j] = al[v][j].second;
    }
  out->V = V;
  out->E = beg[V];
  out->beg_pos = dup_array(beg);
  out->adj = dup_array(adj);
  out->weight = dup_array(wt);
  return 0;
}

int gst_read_reference_groups(const char* path, gst_host_groups* out) {
  if (!path || !out) return 1;
  std::ifstream f(path);
  if (!f.is_open()) return 2;
  std::string line;
  std::vector<std::vector<int32_t>> groups;
  while (std::getline(f, line)) {
    while (!line.empty() && (line.back() == ' ' || line.back() == '\r')) line.pop_back();
    if (line.empty()) continue;
    size_t colon = line.find(':');
    if (colon == std::string::npos || line[0] != 'g') return 3;
    long gid = std::strtol(line.substr(1, colon - 1).c_str(), nullptr, 10) - 1;
    if (gid < 0) return 3;
    if ((size_t)gid >= groups.size()) groups.resize((size_t)gid + 1);
    std::istringstream ss(line.substr(colon + 1));
    long v;
    std::vector<int32_t> mem;
    while (ss >> v) mem.push_back((int32_t)v);
    std::sort(mem.begin(), mem.end());
    groups[gid] = mem;
  }
  std::vector<int64_t> ptr(groups.size() + 1, 0);
  std::vector<int32_t> mem;
  for (size_t g = 0; g < groups.size(); g++) {
    ptr[g + 1] = ptr[g] + (int64_t)groups[g].size();
    mem.insert(mem.end(), groups[g].begin(), groups[g].end());
  }
  out->n_groups = (int32_t)groups.size();
  out->grp_ptr = dup_array(ptr);
  out->members = dup_array(mem);
  return 0;
}

int32_t gst_read_reference_queries(const char* path, int32_t max_queries, int32_t* k_out,
                                   int32_t* out) {
  if (!path || !k_out) return -1;
  std::ifstream f(path);
  if (!f.is_open()) return -1;
  std::string line;
  int32_t n = 0, k = -1;
  while (std::getline(f, line)) {
    std::istringstream ss(line);
    std::vector<int32_t> ids;
    long v;
    while (ss >> v) ids.push_back((int32_t)v);
    if (ids.empty()) continue;
    if (k < 0) k = (int32_t)ids.size();
    if ((int32_t)ids.size() != k) return -1;
    if (out && n < max_queries)
      for (int32_t j = 0; j < k; j++) out[(int64_t)n * k + j] = ids[j];
    n++;
  }
  *k_out = k < 0 ? 0 : k;
  return n;
}

int32_t gst_verify_tree(const gst_host_graph* g, const gst_host_groups* groups, int32_t k,
                        const int32_t* group_ids, int32_t hop_bound, int64_t cost,
                        int64_t n_edges, const int32_t* u, const int32_t* v, const int32_t* w,
                        int32_t root_vertex) {
  if (!g || !groups || !group_ids || k < 1 || n_edges < 0) return 7;
  if (n_edges > 0 && (!u || !v || !w)) return 7;
  // 1: edges exist with their weight
  int64_t sum = 0;
  std::unordered_map<int32_t, std::vector<int32_t>> nb;
  std::unordered_set<uint64_t> seen;
  for (int64_t i = 0; i < n_edges; i++) {
    int32_t a = u[i], b = v[i];
    if (a < 0 || b < 0 || a >= g->V || b >= g->V || a == b) return 1;
    bool ok = false;
    for (int64_t j = g->beg_pos[a]; j < g->beg_pos[a + 1]; j++)
      if (g->adj[j] == b && g->weight[j] == w[i]) {
        ok = true;
        break;
      }
    if (!ok) return 1;
    uint64_t key = ((uint64_t)(uint32_t)std::min(a, b) << 32) | (uint32_t)std::max(a, b);
    if (!seen.insert(key).second) return 6;  // an edge listed twice counts as a cycle
    sum += w[i];
    nb[a].push_back(b);
    nb[b].push_back(a);
  }
  if (n_edges == 0) {
    if (root_vertex < 0 || root_vertex >= g->V) return 7;
    nb[root_vertex];
  }
  // 2: connected, 6: acyclic (a connected graph with |E| = |V|-1)
  const int32_t start = nb.begin()->first;
  std::unordered_map<int32_t, int32_t> depth;
  std::queue<int32_t> q;
  depth[start] = 0;
  q.push(start);
  while (!q.empty()) {
    int32_t x = q.front();
    q.pop();
    for (int32_t y : nb[x])
      if (!depth.count(y)) {
        depth[y] = depth[x] + 1;
        q.push(y);
      }
  }
  if (depth.size() != nb.size()) return 2;
  if ((int64_t)nb.size() != n_edges + 1) return 6;
  // 3: every queried group has a member in the tree
  for (int32_t j = 0; j < k; j++) {
    int32_t gid = group_ids[j];
    if (gid < 0 || gid >= groups->n_groups) return 7;
    bool covered = false;
    for (int64_t t = groups->grp_ptr[gid]; t < groups->grp_ptr[gid + 1] && !covered; t++)
      covered = nb.count(groups->members[t]) > 0;
    if (!covered) return 3;
  }
  // 4: weight sum
  if (sum != cost) return 4;
  // 5: diameter (two BFS passes on a tree)
  if (hop_bound >= 0) {
    int32_t far = start, best = 0;
    for (auto& kv : depth)
      if (kv.second > best) {
        best = kv.second;
        far = kv.first;
      }
    std::unordered_map<int32_t, int32_t> d2;
    d2[far] = 0;
    q.push(far);
    int32_t diam = 0;
    while (!q.empty()) {
      int32_t x = q.front();
      q.pop();
      diam = std::max(diam, d2[x]);
      for (int32_t y : nb[x])
        if (!d2.count(y)) {
          d2[y] = d2[x] + 1;
          q.push(y);
        }
    }
    if (diam > hop_bound) return 5;
  }
  return 0;
}

}  // extern "C"
