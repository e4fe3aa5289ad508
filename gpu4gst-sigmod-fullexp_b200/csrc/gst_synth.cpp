// Seeded synthetic inputs in the shapes of the reference's experiments: power-law
// graphs (Barabasi-Albert, R-MAT), vertex groups (uniform or Zipf sizes) and
// k-group queries.  The reference distributes no datasets that run here (its
// Twitch fixture lacks the .in / _csr.bin / _weight.bin blobs), so these stand in
// for them.  All randomness comes from counter-based splitmix64 streams, so a
// seed gives the same graph on any machine and any number of host threads.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <numeric>
#include <unordered_set>
#include <utility>
#include <vector>

#include <parallel/algorithm>

#include "gst_io.h"

namespace {

inline uint64_t splitmix64(uint64_t x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}

struct Rng {
  uint64_t s;
  explicit Rng(uint64_t seed) : s(splitmix64(seed ^ 0x6A09E667F3BCC909ull)) {}
  uint64_t next() {
    s += 0x9E3779B97F4A7C15ull;
    uint64_t z = s;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
  }
  // uniform in [0, n) by 128-bit multiply (Lemire), bias < 2^-32 for n < 2^32
  uint64_t below(uint64_t n) { return (uint64_t)(((__uint128_t)next() * n) >> 64); }
  double unit() { return (double)(next() >> 11) * (1.0 / 9007199254740992.0); }
};

template <class T>
T* dup_array(const std::vector<T>& v) {
  T* p = (T*)malloc(sizeof(T) * (v.size() ? v.size() : 1));
  if (p && !v.empty()) memcpy(p, v.data(), sizeof(T) * v.size());
  return p;
}

// Build a CSR with both directions from undirected edges (u != v, no duplicates).
void build_csr(int64_t V, const std::vector<std::pair<int32_t, int32_t>>& edges,
               const std::vector<int32_t>& w, gst_host_graph* out) {
  std::vector<int64_t> deg(V + 1, 0);
  for (auto& e : edges) {
    deg[e.first]++;
    deg[e.second]++;
  }
  std::vector<int64_t> beg(V + 1, 0);
  for (int64_t i = 0; i < V; i++) beg[i + 1] = beg[i] + deg[i];
  const int64_t E = beg[V];
  std::vector<int64_t> pos(beg.begin(), beg.end() - 1);
  std::vector<int32_t> adj(E), wt(E);
  for (size_t i = 0; i < edges.size(); i++) {
    int32_t a = edges[i].first, b = edges[i].second;
    adj[pos[a]] = b;
    wt[pos[a]++] = w[i];
    adj[pos[b]] = a;
    wt[pos[b]++] = w[i];
  }
#pragma omp parallel for schedule(dynamic, 1024)
  for (int64_t v = 0; v < V; v++) {
    int64_t b = beg[v], e = beg[v + 1];
    std::vector<std::pair<int32_t, int32_t>> tmp;
    tmp.reserve(e - b);
    for (int64_t i = b; i < e; i++) tmp.push_back({adj[i], wt[i]});
    std::sort(tmp.begin(), tmp.end());
    for (int64_t i = b; i < e; i++) {
      adj[i] = tmp[i - b].first;
      wt[i] = tmp[i - b].second;
    }
  }
  out->V = V;
  out->E = E;
  out->beg_pos = dup_array(beg);
  out->adj = dup_array(adj);
  out->weight = dup_array(wt);
}

std::vector<int32_t> draw_weights(size_t n, uint64_t seed, int32_t wmin, int32_t wmax) {
  std::vector<int32_t> w(n);
  const uint64_t span = (uint64_t)(wmax - wmin + 1);
  const uint64_t base = splitmix64(seed ^ 0xB7E151628AED2A6Bull);
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < (int64_t)n; i++) {
    uint64_t r = splitmix64(base + (uint64_t)i);
    w[i] = wmin + (int32_t)(((__uint128_t)r * span) >> 64);
  }
  return w;
}

int find_root(std::vector<int32_t>& p, int32_t x) {
  while (p[x] != x) {
    p[x] = p[p[x]];
    x = p[x];
  }
  return x;
}

}  // namespace

extern "C" {

void gst_host_graph_free(gst_host_graph* g) {
  if (!g) return;
  free(g->beg_pos);
  free(g->adj);
  free(g->weight);
  g->beg_pos = nullptr;
  g->adj = nullptr;
  g->weight = nullptr;
}

void gst_host_groups_free(gst_host_groups* g) {
  if (!g) return;
  free(g->grp_ptr);
  free(g->members);
  g->grp_ptr = nullptr;
  g->members = nullptr;
}

int gst_synth_ba(int64_t V, int32_t m, uint64_t seed, int32_t wmin, int32_t wmax,
                 gst_host_graph* out) {
  if (!out || m < 1 || V < m + 1 || V > INT32_MAX || wmin < 1 || wmax < wmin) return 1;
  Rng rng(seed);
  std::vector<std::pair<int32_t, int32_t>> edges;
  std::vector<int32_t> repeated;  // each endpoint once per incident edge
  for (int32_t a = 0; a <= m; a++)
    for (int32_t b = a + 1; b <= m; b++) {
      edges.push_back({a, b});
      repeated.push_back(a);
      repeated.push_back(b);
    }
  std::vector<int32_t> targets;
  for (int64_t v = m + 1; v < V; v++) {
    targets.clear();
    while ((int32_t)targets.size() < m) {
      int32_t t = repeated[rng.below(repeated.size())];
      if (std::find(targets.begin(), targets.end(), t) == targets.end()) targets.push_back(t);
    }
    for (int32_t t : targets) {
      edges.push_back({t, (int32_t)v});
      repeated.push_back(t);
      repeated.push_back((int32_t)v);
    }
  }
  std::vector<int32_t> w = draw_weights(edges.size(), seed, wmin, wmax);
  build_csr(V, edges, w, out);
  return 0;
}

int gst_synth_rmat(int64_t V, int64_t n_undirected, double a, double b, double c,
                   uint64_t seed, int32_t wmin, int32_t wmax, int32_t keep_lcc,
                   gst_host_graph* out) {
  if (!out || V < 2 || V > INT32_MAX || n_undirected < 1 || wmin < 1 || wmax < wmin) return 1;
  if (a < 0 || b < 0 || c < 0 || a + b + c > 1.0) return 1;
  if ((double)n_undirected > 0.45 * (double)V * (double)(V - 1)) return 1;
  int scale = 1;
  while (((int64_t)1 << scale) < V) scale++;
  const double ab = a + b, abc = a + b + c;
  const int64_t BLOCK = 1 << 20;
  // candidate = (key, generation index); the accepted edge set is the first
  // n_undirected distinct keys in generation order.
  std::vector<std::pair<uint64_t, int64_t>> uniq;  // sorted by key, min index per key
  int64_t next_block = 0;
  while ((int64_t)uniq.size() < n_undirected) {
    int64_t need = n_undirected - (int64_t)uniq.size();
    int64_t nblocks = (int64_t)((double)need * 1.08 / BLOCK) + 1;
    std::vector<std::pair<uint64_t, int64_t>> cand((size_t)(nblocks * BLOCK));
#pragma omp parallel for schedule(dynamic, 1)
    for (int64_t bi = 0; bi < nblocks; bi++) {
      const int64_t blk = next_block + bi;
      Rng r(seed * 0x100000001B3ull + (uint64_t)blk);
      for (int64_t j = 0; j < BLOCK; j++) {
        const int64_t gi = blk * BLOCK + j;
        uint64_t key = ~0ull;
        // one attempt per candidate slot; rejected draws leave key = ~0 (dropped)
        int64_t u = 0, v = 0;
        for (int lv = 0; lv < scale; lv++) {
          double x = r.unit();
          int bu, bv;
          if (x < a) { bu = 0; bv = 0; }
          else if (x < ab) { bu = 0; bv = 1; }
          else if (x < abc) { bu = 1; bv = 0; }
          else { bu = 1; bv = 1; }
          u = (u << 1) | bu;
          v = (v << 1) | bv;
        }
        if (u < V && v < V && u != v) {
          int64_t lo = std::min(u, v), hi = std::max(u, v);
          key = ((uint64_t)lo << 32) | (uint64_t)hi;
        }
        cand[(size_t)(bi * BLOCK + j)] = {key, gi};
      }
    }
    next_block += nblocks;
    cand.insert(cand.end(), uniq.begin(), uniq.end());
    __gnu_parallel::sort(cand.begin(), cand.end());
    std::vector<std::pair<uint64_t, int64_t>> merged;
    merged.reserve(cand.size());
    for (size_t i = 0; i < cand.size(); i++) {
      if (cand[i].first == ~0ull) break;
      if (!merged.empty() && merged.back().first == cand[i].first) continue;  // keep min index
      merged.push_back(cand[i]);
    }
    uniq.swap(merged);
  }
  // first n_undirected distinct edges in generation order
  std::vector<std::pair<int64_t, uint64_t>> byidx(uniq.size());
  for (size_t i = 0; i < uniq.size(); i++) byidx[i] = {uniq[i].second, uniq[i].first};
  std::vector<std::pair<uint64_t, int64_t>>().swap(uniq);
  __gnu_parallel::sort(byidx.begin(), byidx.end());
  byidx.resize((size_t)n_undirected);
  std::vector<std::pair<int32_t, int32_t>> edges(byidx.size());
  for (size_t i = 0; i < byidx.size(); i++)
    edges[i] = {(int32_t)(byidx[i].second >> 32), (int32_t)(byidx[i].second & 0xffffffffu)};
  std::vector<std::pair<int64_t, uint64_t>>().swap(byidx);

  int64_t Vout = V;
  if (keep_lcc) {
    std::vector<int32_t> p(V);
    std::iota(p.begin(), p.end(), 0);
    for (auto& e : edges) {
      int32_t ra = find_root(p, e.first), rb = find_root(p, e.second);
      if (ra != rb) p[std::max(ra, rb)] = std::min(ra, rb);
    }
    std::vector<int64_t> csize(V, 0);
    std::vector<char> has_edge(V, 0);
    for (auto& e : edges) has_edge[e.first] = has_edge[e.second] = 1;
    for (int64_t v = 0; v < V; v++)
      if (has_edge[v]) csize[find_root(p, (int32_t)v)]++;
    int32_t best = (int32_t)(std::max_element(csize.begin(), csize.end()) - csize.begin());
    std::vector<int32_t> relabel(V, -1);
    int32_t nv = 0;
    for (int64_t v = 0; v < V; v++)
      if (has_edge[v] && find_root(p, (int32_t)v) == best) relabel[v] = nv++;
    std::vector<std::pair<int32_t, int32_t>> kept;
    kept.reserve(edges.size());
    for (auto& e : edges)
      if (relabel[e.first] >= 0) kept.push_back({relabel[e.first], relabel[e.second]});
    edges.swap(kept);
    Vout = nv;
  }
  std::vector<int32_t> w = draw_weights(edges.size(), seed, wmin, wmax);
  build_csr(Vout, edges, w, out);
  return 0;
}

static int fill_groups(int64_t V, const std::vector<int32_t>& sizes, Rng& rng,
                       gst_host_groups* out) {
  const int32_t n = (int32_t)sizes.size();
  std::vector<int64_t> ptr(n + 1, 0);
  for (int32_t g = 0; g < n; g++) ptr[g + 1] = ptr[g] + sizes[g];
  std::vector<int32_t> mem((size_t)ptr[n]);
  std::unordered_set<int64_t> chosen;
  for (int32_t g = 0; g < n; g++) {
    // Floyd's sampling without replacement
    chosen.clear();
    const int64_t s = sizes[g];
    for (int64_t j = V - s; j < V; j++) {
      int64_t t = (int64_t)rng.below((uint64_t)(j + 1));
      if (!chosen.insert(t).second) chosen.insert(j);
    }
    std::vector<int32_t> tmp(chosen.begin(), chosen.end());
    std::sort(tmp.begin(), tmp.end());
    std::copy(tmp.begin(), tmp.end(), mem.begin() + ptr[g]);
  }
  out->n_groups = n;
  out->grp_ptr = dup_array(ptr);
  out->members = dup_array(mem);
  return 0;
}

int gst_synth_groups_uniform(int64_t V, int32_t n_groups, int32_t smin, int32_t smax,
                             uint64_t seed, gst_host_groups* out) {
  if (!out || n_groups < 1 || smin < 1 || smax < smin || smax > V) return 1;
  Rng rng(seed);
  std::vector<int32_t> sizes(n_groups);
  for (auto& s : sizes) s = smin + (int32_t)rng.below((uint64_t)(smax - smin + 1));
  return fill_groups(V, sizes, rng, out);
}

int gst_synth_groups_zipf(int64_t V, int32_t n_groups, double s, int32_t smin, int32_t smax,
                          uint64_t seed, gst_host_groups* out) {
  if (!out || n_groups < 1 || s <= 1.0 || smin < 1 || smax < smin || smax > V) return 1;
  Rng rng(seed);
  // Zipf(s) on {1,2,...} by Devroye's rejection method (Non-Uniform Random
  // Variate Generation, 1986, X.6.1), then clamped to [smin, smax].
  const double am1 = s - 1.0, bb = std::pow(2.0, am1);
  std::vector<int32_t> sizes(n_groups);
  for (auto& sz : sizes) {
    double X;
    for (;;) {
      double U = 1.0 - rng.unit(), Vv = rng.unit();
      X = std::floor(std::pow(U, -1.0 / am1));
      if (X > 1e9 || X < 1.0) continue;
      double T = std::pow(1.0 + 1.0 / X, am1);
      if (Vv * X * (T - 1.0) / (bb - 1.0) <= T / bb) break;
    }
    int64_t xi = (int64_t)X;
    sz = (int32_t)std::min<int64_t>(std::max<int64_t>(xi, smin), smax);
  }
  return fill_groups(V, sizes, rng, out);
}

int gst_synth_queries(int32_t n_groups, int32_t n_queries, int32_t k, uint64_t seed,
                      int32_t* out) {
  if (!out || k < 1 || k > n_groups || n_queries < 0) return 1;
  Rng rng(seed);
  for (int32_t q = 0; q < n_queries; q++) {
    int32_t* row = out + (int64_t)q * k;
    for (int32_t j = 0; j < k; j++) {
      int32_t g;
      bool dup;
      do {
        g = (int32_t)rng.below((uint64_t)n_groups);
        dup = false;
        for (int32_t t = 0; t < j; t++) dup |= (row[t] == g);
      } while (dup);
      row[j] = g;
    }
  }
  return 0;
}

}  // extern "C"
