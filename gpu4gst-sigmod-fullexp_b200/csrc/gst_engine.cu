// Host side of the GST engine and its C ABI (include/gst.h).
//
// A gst_graph owns the device CSR and a pool of query slots (state slab,
// one-label distances, worklists).  gst_solve runs one query in slot 0;
// gst_solve_batch runs up to cfg.max_batch queries at once in as many slots,
// refilling a slot as soon as its query finishes.  The level loop is a fixed
// launch sequence (sssp, ctrl, rows, ctrl, grow, ctrl) that the host issues a few
// levels ahead of the device; every kernel reads its work counts from the
// device-side contexts, so extra launches after a query finishes are no-ops.
#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <utility>
#include <vector>

#include <cuda_runtime.h>

#include "gst.h"
#include "gst_device.cuh"

using namespace gst;

namespace {

thread_local std::string tl_err;

struct Slot {
  size_t rw_cap = 0;     // cells per row the slab was sized for
  int64_t V = 0;
  uint64_t* table = nullptr;
  uint32_t* dist = nullptr;
  uint32_t* rowbits = nullptr;
  uint32_t* tour = nullptr;
  uint4* q[2] = {nullptr, nullptr};
  uint4* far[2] = {nullptr, nullptr};
  uint32_t* rows = nullptr;
  int32_t* out = nullptr;
  uint64_t* stack = nullptr;
  uint32_t qcap = 0, farcap = 0, rowcap = 0, outcap = 0, stackcap = 0;
  size_t bytes = 0;
};

}  // namespace

// Counters of one gst_solve_batch call.
struct CallStats {
  int64_t launches = 0, h2d = 0, d2h = 0;
  std::vector<std::pair<int, int>> prof;  // (kernel kind, event-pair index)
  size_t next_ev = 0;
};

struct gst_engine {
  int device = 0;
  gst_config cfg{};
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  std::vector<cudaEvent_t> prof_events;  // reused pairs for cfg.profile_kernels
  CallStats cs;
  int sms = 148;
  int grow_blocks = 0, sssp_blocks = 0;
  std::string err;
  std::mutex mu;
};

struct gst_graph {
  gst_engine* eng = nullptr;
  int64_t V = 0, E = 0;
  int64_t* d_beg = nullptr;
  int2* d_edges = nullptr;   // per vertex sorted by neighbour (tree extraction)
  int2* d_wedges = nullptr;  // per vertex sorted by (weight, neighbour) (grow, SSSP)
  uint32_t* d_widx = nullptr;
  std::vector<int64_t> h_beg;
  std::vector<Slot> slots;
  Ctx* d_ctx = nullptr;       // MAXB contexts
  Ctx* h_ctx = nullptr;       // pinned mirror
};

struct gst_groups {
  gst_graph* g = nullptr;
  int32_t n = 0;
  int64_t* d_ptr = nullptr;
  int32_t* d_mem = nullptr;
  std::vector<int64_t> h_ptr;
};

namespace {

gst_status fail(gst_engine* e, gst_status s, const std::string& msg) {
  if (e) e->err = msg;
  tl_err = msg;
  return s;
}

#define CK(call)                                                                      \
  do {                                                                                \
    cudaError_t _e = (call);                                                          \
    if (_e != cudaSuccess)                                                            \
      return fail(eng, GST_DEVICE_ERROR,                                              \
                  std::string(#call) + ": " + cudaGetErrorString(_e));                \
  } while (0)

void free_slot(Slot& s) {
  cudaFree(s.table);
  cudaFree(s.dist);
  cudaFree(s.rowbits);
  cudaFree(s.tour);
  cudaFree(s.q[0]);
  cudaFree(s.q[1]);
  cudaFree(s.far[0]);
  cudaFree(s.far[1]);
  cudaFree(s.rows);
  cudaFree(s.out);
  cudaFree(s.stack);
  s = Slot();
}

// worklist capacity for a slab of V rows of rw cells
uint32_t list_cap(int64_t V, size_t rw) {
  const uint64_t want = (uint64_t)V * rw + 4ull * (uint64_t)V + 4096;
  return (uint32_t)std::min<uint64_t>(want, 1ull << 26);
}

constexpr size_t kTourWords = ((size_t)1 << KMAX) * (TOUR_STRIDE + KMAX);

size_t slot_bytes(int64_t V, size_t rw) {
  const uint64_t cap = list_cap(V, rw);
  return (size_t)V * rw * 8 + (size_t)V * DIST_STRIDE * 4 + ((size_t)V + 31) / 32 * 4 +
         kTourWords * 4 +
         4 * (size_t)cap * 16 + (size_t)V * 4 + (size_t)(1 << 16) * 12 + (size_t)(1 << 18) * 8;
}

gst_status ensure_slot(gst_engine* eng, gst_graph* g, size_t idx, size_t rw) {
  if (g->slots.size() <= idx) g->slots.resize(idx + 1);
  Slot& s = g->slots[idx];
  if (s.table && s.rw_cap >= rw && s.V == g->V) return GST_OK;
  free_slot(s);
  const int64_t V = g->V;
  s.V = V;
  s.rw_cap = rw;
  s.qcap = s.farcap = list_cap(V, rw);
  s.rowcap = (uint32_t)V;
  s.outcap = 1 << 16;
  s.stackcap = 1 << 18;
  CK(cudaMalloc(&s.table, (size_t)V * rw * 8));
  CK(cudaMalloc(&s.dist, (size_t)V * DIST_STRIDE * 4));
  CK(cudaMalloc(&s.rowbits, ((size_t)V + 31) / 32 * 4));
  CK(cudaMalloc(&s.tour, kTourWords * 4));
  for (int i = 0; i < 2; i++) {
    CK(cudaMalloc(&s.q[i], (size_t)s.qcap * 16));
    CK(cudaMalloc(&s.far[i], (size_t)s.farcap * 16));
  }
  CK(cudaMalloc(&s.rows, (size_t)V * 4));
  CK(cudaMalloc(&s.out, (size_t)s.outcap * 12));
  CK(cudaMalloc(&s.stack, (size_t)s.stackcap * 8));
  CK(cudaMemsetAsync(s.rowbits, 0, ((size_t)V + 31) / 32 * 4, eng->stream));
  s.bytes = slot_bytes(V, rw);
  return GST_OK;
}

size_t row_width(int k, int D) { return ((size_t)1 << k) * (size_t)(D >= 0 ? D + 1 : 1); }

gst_status validate_query(gst_engine* eng, gst_groups* grp, const gst_query* q) {
  if (!q || q->k < 1 || q->k > KMAX || !q->group_ids)
    return fail(eng, GST_BAD_INPUT, "query: k must be in [1,8] with group ids");
  if (q->hop_bound > 30) return fail(eng, GST_BAD_INPUT, "query: hop bound must be <= 30");
  for (int i = 0; i < q->k; i++) {
    const int32_t a = q->group_ids[i];
    if (a < 0 || a >= grp->n) return fail(eng, GST_BAD_INPUT, "query: group id out of range");
    if (grp->h_ptr[a + 1] == grp->h_ptr[a])
      return fail(eng, GST_BAD_INPUT, "query: group has no members");
    for (int j = 0; j < i; j++)
      if (q->group_ids[j] == a) return fail(eng, GST_BAD_INPUT, "query: duplicate group id");
  }
  return GST_OK;
}

// Host copy of a fresh context for query q in slot s.
void prep_ctx(gst_engine* eng, gst_graph* g, Slot& s, const gst_query* q, Ctx& c) {
  memset(&c, 0, sizeof(c));
  const int hop = q->hop_bound >= 0;
  c.table = s.table;
  c.dist = s.dist;
  c.rowbits = s.rowbits;
  c.tour = s.tour;
  c.q[0] = s.q[0];
  c.q[1] = s.q[1];
  c.far[0] = s.far[0];
  c.far[1] = s.far[1];
  c.rows = s.rows;
  c.out = s.out;
  c.stack = s.stack;
  c.qcap = s.qcap;
  c.farcap = s.farcap;
  c.rowcap = s.rowcap;
  c.outcap = s.outcap;
  c.stackcap = s.stackcap;
  c.k = q->k;
  c.W = 1 << q->k;
  c.full = c.W - 1;
  c.D = hop ? q->hop_bound : 0;
  c.DD = hop ? q->hop_bound + 1 : 1;
  c.RW = c.W * c.DD;
  c.hop = hop;
  c.use_lb = hop ? 0 : 1;
  c.use_tour = c.use_lb;
  for (int i = 0; i < q->k; i++) c.gid[i] = q->group_ids[i];
  memset(c.vv, 0xFF, sizeof(c.vv));
  c.delta = (uint32_t)std::max(0, eng->cfg.bucket_delta);
  c.max_levels = (uint32_t)eng->cfg.max_levels;
  c.in_ptr = nullptr;
  c.in_n = 0;
  c.in_kind = 0;
  c.in_idx = 1;
  c.no = 0;
  c.f = 0;
  c.far_min = 0xFFFFFFFFu;
  c.bucket_end = c.delta ? c.delta : 0xFFFFFFFFu;
  c.ub = 0xFFFFFFFFu;
  c.ub_cell = 0xFFFFFFFFu;
  c.best = ~0ull;
  c.phase = c.use_lb ? PH_SSSP : PH_DP;
}

// Clear the slot's slab and distances for a query with row width rw.
gst_status reset_slot(gst_engine* eng, gst_graph* g, Slot& s, size_t rw, bool need_dist) {
  CK(cudaMemsetAsync(s.table, 0xFF, (size_t)g->V * rw * 8, eng->stream));
  CK(cudaMemsetAsync(s.rowbits, 0, ((size_t)g->V + 31) / 32 * 4, eng->stream));
  if (need_dist) CK(cudaMemsetAsync(s.dist, 0xFF, (size_t)g->V * DIST_STRIDE * 4, eng->stream));
  return GST_OK;
}

struct LoopShape {
  bool sssp = true;
  int rw_max = 1;
};

enum ProfKind { PROF_GROW = 0, PROF_ROWS = 1, PROF_SSSP = 2 };

// Record the start event of a profiled launch; returns the pair index or -1.
int prof_begin(gst_engine* eng, int kind) {
  if (!((eng->cfg.profile_kernels >> kind) & 1)) return -1;
  const size_t i = eng->cs.next_ev++;
  while (eng->prof_events.size() < 2 * (i + 1)) {
    cudaEvent_t e;
    if (cudaEventCreate(&e) != cudaSuccess) return -1;
    eng->prof_events.push_back(e);
  }
  cudaEventRecord(eng->prof_events[2 * i], eng->stream);
  eng->cs.prof.push_back({kind, (int)i});
  return (int)i;
}
void prof_end(gst_engine* eng, int i) {
  if (i >= 0) cudaEventRecord(eng->prof_events[2 * i + 1], eng->stream);
}

DevGraph dev_graph(const gst_graph* g) {
  return DevGraph{g->V, g->E, g->d_beg, g->d_edges, g->d_wedges, g->d_widx};
}

gst_status launch_level(gst_engine* eng, gst_graph* g, int nctx, const LoopShape& sh) {
  cudaStream_t st = eng->stream;
  const DevGraph G = dev_graph(g);
  const int split = eng->cfg.split_degree;
  const int tpb = eng->cfg.threads_per_block;
  if (sh.sssp) {
    const int pe = prof_begin(eng, PROF_SSSP);
    k_sssp<<<eng->sssp_blocks, 256, 0, st>>>(g->d_ctx, nctx, G, split);
    prof_end(eng, pe);
    k_ctrl<<<nctx, 128, 0, st>>>(g->d_ctx, nctx, CTRL_SSSP);
    eng->cs.launches += 2;
  }
  const size_t per_warp = rows_smem_per_warp(sh.rw_max);
  const int warps = std::max(1, tpb / 32);
  int pe = prof_begin(eng, PROF_ROWS);
  k_rows<<<eng->grow_blocks, warps * 32, per_warp * warps, st>>>(g->d_ctx, nctx, G, split,
                                                                  sh.rw_max);
  prof_end(eng, pe);
  k_ctrl<<<nctx, 128, 0, st>>>(g->d_ctx, nctx, CTRL_DP_ROWS);
  pe = prof_begin(eng, PROF_GROW);
  k_grow<<<eng->grow_blocks, 256, 0, st>>>(g->d_ctx, nctx, G, split);
  prof_end(eng, pe);
  k_ctrl<<<nctx, 128, 0, st>>>(g->d_ctx, nctx, CTRL_DP_GROW);
  eng->cs.launches += 4;
  CK(cudaGetLastError());
  return GST_OK;
}

gst_status status_of(const Ctx& c) {
  if (c.error & ERR_TIMEOUT) return GST_TIMEOUT;
  if (c.error & (ERR_QCAP | ERR_FARCAP | ERR_ROWCAP)) return GST_CAPACITY;
  if (c.error) return GST_DEVICE_ERROR;
  if (c.phase != PH_DONE) return GST_DEVICE_ERROR;
  if (c.best == ~0ull) return GST_INFEASIBLE;
  return GST_OK;
}

void fill_result(gst_graph* g, const Ctx& c, const gst_query* q, const std::vector<int32_t>& raw,
                 gst_result* r) {
  memset(r, 0, sizeof(*r));
  r->user_tag = q->user_tag;
  r->status = status_of(c);
  r->stats.levels = c.levels;
  r->stats.states_expanded = (int64_t)c.st_items;
  r->stats.edge_relaxations = (int64_t)c.st_relax;
  r->stats.merge_pairs = (int64_t)c.st_merge;
  r->stats.rows_merged = (int64_t)c.st_rows;
  r->stats.sssp_relaxations = (int64_t)c.st_sssp;
  if (r->status != GST_OK) return;
  r->cost = (int32_t)(c.best >> 32);
  r->root = (int32_t)(c.best & 0x7FFFFFFull);
  r->root_hop = (int32_t)((c.best >> 27) & 31u);
  // distinct edges, (min, max) orientation
  std::vector<std::pair<std::pair<int32_t, int32_t>, int32_t>> es;
  const size_t n = std::min<size_t>(c.n_out, raw.size() / 3);
  es.reserve(n);
  for (size_t i = 0; i < n; i++) {
    int32_t a = raw[3 * i], b = raw[3 * i + 1];
    if (a > b) std::swap(a, b);
    es.push_back({{a, b}, raw[3 * i + 2]});
  }
  std::sort(es.begin(), es.end());
  es.erase(std::unique(es.begin(), es.end(),
                       [](const auto& x, const auto& y) { return x.first == y.first; }),
           es.end());
  r->n_edges = (int64_t)es.size();
  if (!es.empty()) {
    r->edge_u = (int32_t*)malloc(sizeof(int32_t) * es.size());
    r->edge_v = (int32_t*)malloc(sizeof(int32_t) * es.size());
    r->edge_w = (int32_t*)malloc(sizeof(int32_t) * es.size());
    for (size_t i = 0; i < es.size(); i++) {
      r->edge_u[i] = es[i].first.first;
      r->edge_v[i] = es[i].first.second;
      r->edge_w[i] = es[i].second;
    }
  }
}

}  // namespace

extern "C" {

void gst_config_default(gst_config* cfg) {
  if (!cfg) return;
  memset(cfg, 0, sizeof(*cfg));
  cfg->mem_budget_bytes = 0;
  cfg->split_degree = 256;
  cfg->bucket_delta = 0;
  cfg->max_levels = 1 << 20;
  cfg->threads_per_block = 256;
  cfg->blocks_per_sm = 4;
  cfg->max_batch = 16;
  cfg->use_graphs = 0;
  cfg->verbose = 0;
}

gst_status gst_engine_create(int32_t device, const gst_config* cfg, gst_engine** out) {
  if (!out) return fail(nullptr, GST_BAD_INPUT, "engine: null output");
  *out = nullptr;
  int ndev = 0;
  cudaError_t e = cudaGetDeviceCount(&ndev);
  if (e != cudaSuccess || ndev == 0)
    return fail(nullptr, GST_DEVICE_ERROR, "engine: no CUDA device available");
  if (device < 0 || device >= ndev) return fail(nullptr, GST_BAD_INPUT, "engine: bad device");
  gst_engine* eng = new gst_engine();
  eng->device = device;
  gst_config_default(&eng->cfg);
  if (cfg) {
    gst_config d = eng->cfg;
    eng->cfg = *cfg;
    if (eng->cfg.split_degree <= 0) eng->cfg.split_degree = d.split_degree;
    if (eng->cfg.max_levels <= 0) eng->cfg.max_levels = d.max_levels;
    if (eng->cfg.threads_per_block <= 0) eng->cfg.threads_per_block = d.threads_per_block;
    if (eng->cfg.blocks_per_sm <= 0) eng->cfg.blocks_per_sm = d.blocks_per_sm;
    if (eng->cfg.max_batch <= 0) eng->cfg.max_batch = d.max_batch;
  }
  eng->cfg.max_batch = std::min(eng->cfg.max_batch, MAXB);
  if (cudaSetDevice(device) != cudaSuccess) {
    delete eng;
    return fail(nullptr, GST_DEVICE_ERROR, "engine: cudaSetDevice failed");
  }
  cudaDeviceProp prop;
  cudaGetDeviceProperties(&prop, device);
  eng->sms = prop.multiProcessorCount;
  eng->grow_blocks = eng->sms * eng->cfg.blocks_per_sm;
  eng->sssp_blocks = eng->sms * eng->cfg.blocks_per_sm;
  if (cudaStreamCreateWithFlags(&eng->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreate(&eng->ev0) != cudaSuccess || cudaEventCreate(&eng->ev1) != cudaSuccess) {
    delete eng;
    return fail(nullptr, GST_DEVICE_ERROR, "engine: stream/event creation failed");
  }
  cudaFuncSetAttribute(k_rows, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
  *out = eng;
  return GST_OK;
}

gst_status gst_engine_destroy(gst_engine* eng) {
  if (!eng) return GST_OK;
  cudaSetDevice(eng->device);
  if (eng->stream) cudaStreamDestroy(eng->stream);
  if (eng->ev0) cudaEventDestroy(eng->ev0);
  if (eng->ev1) cudaEventDestroy(eng->ev1);
  for (auto e : eng->prof_events) cudaEventDestroy(e);
  delete eng;
  return GST_OK;
}

const char* gst_last_error_string(gst_engine* eng) {
  if (eng) {
    tl_err = eng->err;
    return tl_err.c_str();
  }
  return tl_err.c_str();
}

static gst_status graph_create_impl(gst_engine* eng, int64_t V, int64_t E, const int64_t* beg,
                                    const int32_t* adj, const int32_t* wt, gst_graph** out) {
  if (!eng || !out) return fail(eng, GST_BAD_INPUT, "graph: null argument");
  *out = nullptr;
  if (V < 1 || V >= (int64_t)1 << 27 || E < 0 || !beg || (E > 0 && (!adj || !wt)))
    return fail(eng, GST_BAD_INPUT, "graph: need 1 <= V < 2^27, E >= 0 and non-null arrays");
  if (beg[0] != 0 || beg[V] != E) return fail(eng, GST_BAD_INPUT, "graph: beg_pos[0] must be 0 and beg_pos[V] == E");
  for (int64_t v = 0; v < V; v++)
    if (beg[v + 1] < beg[v]) return fail(eng, GST_BAD_INPUT, "graph: beg_pos not monotone");
  // Two device copies of the adjacency: sorted by neighbour (edge-weight lookups
  // of the tree walk) and sorted by weight, with per vertex the number of edges of
  // weight <= 2^j (j < WIDX), so that a grow step reads only the edges light enough
  // to keep its target under the upper bound.
  std::vector<int2> edges((size_t)E), wedges((size_t)E);
  std::vector<uint32_t> widx((size_t)V * WIDX);
  int bad = 0;
#pragma omp parallel
  {
    std::vector<std::pair<int32_t, int32_t>> tmp;
#pragma omp for schedule(dynamic, 1024) reduction(| : bad)
    for (int64_t v = 0; v < V; v++) {
      tmp.clear();
      for (int64_t i = beg[v]; i < beg[v + 1]; i++) {
        if (adj[i] < 0 || adj[i] >= V) bad |= 1;
        else if (wt[i] < 1 || wt[i] > (1 << 24)) bad |= 2;
        else tmp.push_back({adj[i], wt[i]});
      }
      if (!std::is_sorted(tmp.begin(), tmp.end())) std::sort(tmp.begin(), tmp.end());
      for (size_t j = 0; j < tmp.size(); j++)
        edges[beg[v] + j] = make_int2(tmp[j].first, tmp[j].second);
      for (auto& x : tmp) std::swap(x.first, x.second);
      std::sort(tmp.begin(), tmp.end());
      size_t j = 0;
      for (int t = 0; t < WIDX; t++) {
        while (j < tmp.size() && tmp[j].first <= (1 << t)) j++;
        widx[(size_t)v * WIDX + t] = (uint32_t)j;
      }
      for (size_t i = 0; i < tmp.size(); i++)
        wedges[beg[v] + i] = make_int2(tmp[i].second, tmp[i].first);
    }
  }
  if (bad & 1) return fail(eng, GST_BAD_INPUT, "graph: neighbour id out of range");
  if (bad & 2) return fail(eng, GST_BAD_INPUT, "graph: weights must be in [1, 2^24]");
  std::lock_guard<std::mutex> lk(eng->mu);
  CK(cudaSetDevice(eng->device));
  gst_graph* g = new gst_graph();
  g->eng = eng;
  g->V = V;
  g->E = E;
  g->h_beg.assign(beg, beg + V + 1);
  CK(cudaMalloc(&g->d_beg, sizeof(int64_t) * (V + 1)));
  CK(cudaMalloc(&g->d_edges, sizeof(int2) * std::max<int64_t>(E, 1)));
  CK(cudaMalloc(&g->d_wedges, sizeof(int2) * std::max<int64_t>(E, 1)));
  CK(cudaMalloc(&g->d_widx, sizeof(uint32_t) * V * WIDX));
  CK(cudaMalloc(&g->d_ctx, sizeof(Ctx) * MAXB));
  CK(cudaMallocHost(&g->h_ctx, sizeof(Ctx) * MAXB));
  // stream-ordered copies, completed before returning: the level kernels run on a
  // non-blocking stream that does not wait for the legacy default stream
  CK(cudaMemcpyAsync(g->d_beg, beg, sizeof(int64_t) * (V + 1), cudaMemcpyHostToDevice,
                     eng->stream));
  if (E) {
    CK(cudaMemcpyAsync(g->d_edges, edges.data(), sizeof(int2) * E, cudaMemcpyHostToDevice,
                       eng->stream));
    CK(cudaMemcpyAsync(g->d_wedges, wedges.data(), sizeof(int2) * E, cudaMemcpyHostToDevice,
                       eng->stream));
  }
  CK(cudaMemcpyAsync(g->d_widx, widx.data(), sizeof(uint32_t) * V * WIDX,
                     cudaMemcpyHostToDevice, eng->stream));
  CK(cudaStreamSynchronize(eng->stream));
  *out = g;
  return GST_OK;
}

gst_status gst_graph_create(gst_engine* eng, int64_t V, int64_t E, const int64_t* beg_pos,
                            const int32_t* csr, const int32_t* weight, gst_graph** out) {
  return graph_create_impl(eng, V, E, beg_pos, csr, weight, out);
}

gst_status gst_graph_create_i64(gst_engine* eng, int64_t V, int64_t E, const int64_t* beg_pos,
                                const int64_t* csr, const int64_t* weight, gst_graph** out) {
  if (E < 0 || (E > 0 && (!csr || !weight))) return fail(eng, GST_BAD_INPUT, "graph: bad arrays");
  std::vector<int32_t> a((size_t)E), w((size_t)E);
  for (int64_t i = 0; i < E; i++) {
    if (csr[i] < 0 || csr[i] >= V) return fail(eng, GST_BAD_INPUT, "graph: neighbour id out of range");
    if (weight[i] < 1 || weight[i] > (1 << 24))
      return fail(eng, GST_BAD_INPUT, "graph: weights must be in [1, 2^24]");
    a[i] = (int32_t)csr[i];
    w[i] = (int32_t)weight[i];
  }
  return graph_create_impl(eng, V, E, beg_pos, a.data(), w.data(), out);
}

gst_status gst_graph_destroy(gst_graph* g) {
  if (!g) return GST_OK;
  gst_engine* eng = g->eng;
  std::lock_guard<std::mutex> lk(eng->mu);
  cudaSetDevice(eng->device);
  cudaStreamSynchronize(eng->stream);
  for (auto& s : g->slots) free_slot(s);
  cudaFree(g->d_beg);
  cudaFree(g->d_edges);
  cudaFree(g->d_wedges);
  cudaFree(g->d_widx);
  cudaFree(g->d_ctx);
  cudaFreeHost(g->h_ctx);
  delete g;
  return GST_OK;
}

gst_status gst_groups_create(gst_graph* g, int32_t n_groups, const int64_t* grp_ptr,
                             const int32_t* members, gst_groups** out) {
  gst_engine* eng = g ? g->eng : nullptr;
  if (!g || !out || n_groups < 1 || !grp_ptr) return fail(eng, GST_BAD_INPUT, "groups: bad arguments");
  *out = nullptr;
  if (grp_ptr[0] != 0) return fail(eng, GST_BAD_INPUT, "groups: grp_ptr[0] must be 0");
  for (int32_t i = 0; i < n_groups; i++)
    if (grp_ptr[i + 1] < grp_ptr[i]) return fail(eng, GST_BAD_INPUT, "groups: grp_ptr not monotone");
  const int64_t M = grp_ptr[n_groups];
  if (M > 0 && !members) return fail(eng, GST_BAD_INPUT, "groups: null members");
  for (int64_t j = 0; j < M; j++)
    if (members[j] < 0 || members[j] >= g->V) return fail(eng, GST_BAD_INPUT, "groups: member out of range");
  std::lock_guard<std::mutex> lk(eng->mu);
  CK(cudaSetDevice(eng->device));
  gst_groups* gr = new gst_groups();
  gr->g = g;
  gr->n = n_groups;
  gr->h_ptr.assign(grp_ptr, grp_ptr + n_groups + 1);
  CK(cudaMalloc(&gr->d_ptr, sizeof(int64_t) * (n_groups + 1)));
  CK(cudaMalloc(&gr->d_mem, sizeof(int32_t) * std::max<int64_t>(M, 1)));
  CK(cudaMemcpyAsync(gr->d_ptr, grp_ptr, sizeof(int64_t) * (n_groups + 1),
                     cudaMemcpyHostToDevice, eng->stream));
  if (M)
    CK(cudaMemcpyAsync(gr->d_mem, members, sizeof(int32_t) * M, cudaMemcpyHostToDevice,
                       eng->stream));
  CK(cudaStreamSynchronize(eng->stream));
  *out = gr;
  return GST_OK;
}

gst_status gst_groups_destroy(gst_groups* gr) {
  if (!gr) return GST_OK;
  cudaSetDevice(gr->g->eng->device);
  cudaFree(gr->d_ptr);
  cudaFree(gr->d_mem);
  delete gr;
  return GST_OK;
}

gst_status gst_solve_batch(gst_graph* g, gst_groups* grp, int32_t n, const gst_query* queries,
                           gst_result* results) {
  gst_engine* eng = g ? g->eng : nullptr;
  if (!g || !grp || grp->g != g || n < 0 || (n > 0 && (!queries || !results)))
    return fail(eng, GST_BAD_INPUT, "solve: bad arguments");
  for (int32_t i = 0; i < n; i++) memset(&results[i], 0, sizeof(gst_result));
  std::lock_guard<std::mutex> lk(eng->mu);
  CK(cudaSetDevice(eng->device));
  const int B = std::max(1, std::min<int>(eng->cfg.max_batch, n));
  // admission: slots sized for the widest query, bounded by the memory budget
  size_t rw_max = 1;
  for (int32_t i = 0; i < n; i++) {
    gst_status s = validate_query(eng, grp, &queries[i]);
    if (s != GST_OK) {
      results[i].status = s;
      results[i].user_tag = queries[i].user_tag;
      continue;
    }
    rw_max = std::max(rw_max, row_width(queries[i].k, queries[i].hop_bound));
  }
  size_t free_b = 0, total_b = 0;
  CK(cudaMemGetInfo(&free_b, &total_b));
  size_t held = 0;
  for (auto& s : g->slots) held += s.bytes;
  const size_t budget = eng->cfg.mem_budget_bytes > 0 ? (size_t)eng->cfg.mem_budget_bytes
                                                      : (size_t)((free_b + held) * 0.85);
  const size_t per = slot_bytes(g->V, rw_max);
  int nslots = (int)std::min<size_t>((size_t)B, budget / std::max<size_t>(per, 1));
  if (nslots < 1) {
    for (int32_t i = 0; i < n; i++)
      if (results[i].status == 0) {
        results[i].status = GST_OOM_ADMISSION;
        results[i].user_tag = queries[i].user_tag;
      }
    return fail(eng, GST_OOM_ADMISSION, "solve: state table does not fit the memory budget");
  }
  for (int s = 0; s < nslots; s++) {
    gst_status st = ensure_slot(eng, g, (size_t)s, rw_max);
    if (st != GST_OK) return st;
  }
  // slot -> query index; -1 = free
  std::vector<int> owner(nslots, -1);
  std::vector<int32_t> raw((size_t)(1 << 16) * 3);
  int32_t next = 0;
  auto next_valid = [&]() {
    while (next < n && results[next].status != 0) next++;
    return next < n ? next++ : -1;
  };
  eng->cs = CallStats();
  const auto t_call = std::chrono::steady_clock::now();
  std::vector<double> lat(n > 0 ? n : 1, 0.0);
  CK(cudaEventRecord(eng->ev0, eng->stream));
  int active = 0;
  // fill and run in waves of refills: a finished slot is refilled at the next check
  for (;;) {
    for (int s = 0; s < nslots; s++) {
      if (owner[s] >= 0) continue;
      int qi = next_valid();
      if (qi < 0) break;
      const gst_query* q = &queries[qi];
      Slot& sl = g->slots[s];
      Ctx& hc = g->h_ctx[s];
      prep_ctx(eng, g, sl, q, hc);
      gst_status st = reset_slot(eng, g, sl, (size_t)hc.RW, hc.use_lb != 0);
      if (st != GST_OK) return st;
      CK(cudaMemcpyAsync(g->d_ctx + s, &hc, sizeof(Ctx), cudaMemcpyHostToDevice, eng->stream));
      eng->cs.h2d += sizeof(Ctx);
      eng->cs.launches += 2;
      // k_init for this slot alone: grid.y selects the context
      const DevGraph G = dev_graph(g);
      k_init<<<dim3(64, 1), 256, 0, eng->stream>>>(g->d_ctx + s, 1, G, grp->d_ptr, grp->d_mem,
                                                   eng->cfg.split_degree);
      k_ctrl<<<1, 32, 0, eng->stream>>>(g->d_ctx + s, 1, CTRL_SSSP);
      owner[s] = qi;
      active++;
    }
    if (active == 0) break;
    // contexts of free slots must look finished to the level kernels
    for (int s = 0; s < nslots; s++)
      if (owner[s] < 0) {
        Ctx& idle = g->h_ctx[s];
        memset(&idle, 0, sizeof(idle));
        idle.phase = PH_DONE;
        idle.best = ~0ull;
        CK(cudaMemcpyAsync(g->d_ctx + s, &idle, sizeof(Ctx), cudaMemcpyHostToDevice, eng->stream));
        eng->cs.h2d += sizeof(Ctx);
      }
    LoopShape sh;
    sh.sssp = true;
    sh.rw_max = (int)rw_max;
    // run until at least one query finishes
    const int ahead = 6;
    bool any_done = false;
    while (!any_done) {
      for (int i = 0; i < ahead; i++) {
        gst_status st = launch_level(eng, g, nslots, sh);
        if (st != GST_OK) return st;
      }
      CK(cudaMemcpyAsync(g->h_ctx, g->d_ctx, sizeof(Ctx) * nslots, cudaMemcpyDeviceToHost,
                         eng->stream));
      eng->cs.d2h += (int64_t)sizeof(Ctx) * nslots;
      CK(cudaStreamSynchronize(eng->stream));
      bool any_sssp = false;
      for (int s = 0; s < nslots; s++) {
        if (owner[s] < 0) continue;
        any_sssp |= g->h_ctx[s].phase == PH_SSSP || g->h_ctx[s].phase == PH_PREP;
        any_done |= g->h_ctx[s].phase >= PH_DONE;
      }
      sh.sssp = any_sssp;
    }
    // harvest finished queries
    const DevGraph G = dev_graph(g);
    k_extract<<<1, MAXB, 0, eng->stream>>>(g->d_ctx, nslots, G);
    eng->cs.launches += 1;
    CK(cudaMemcpyAsync(g->h_ctx, g->d_ctx, sizeof(Ctx) * nslots, cudaMemcpyDeviceToHost,
                       eng->stream));
    eng->cs.d2h += (int64_t)sizeof(Ctx) * nslots;
    CK(cudaStreamSynchronize(eng->stream));
    for (int s = 0; s < nslots; s++) {
      if (owner[s] < 0 || g->h_ctx[s].phase < PH_DONE) continue;
      const Ctx c = g->h_ctx[s];
      const uint32_t nout = std::min(c.n_out, g->slots[s].outcap);
      if (nout) {
        CK(cudaMemcpyAsync(raw.data(), g->slots[s].out, (size_t)nout * 12,
                           cudaMemcpyDeviceToHost, eng->stream));
        eng->cs.d2h += (int64_t)nout * 12;
        CK(cudaStreamSynchronize(eng->stream));
      }
      fill_result(g, c, &queries[owner[s]], raw, &results[owner[s]]);
      if (c.error || c.phase != PH_DONE) {
        char msg[160];
        snprintf(msg, sizeof msg, "query %d: phase %u error bits 0x%x bounds site %u levels %u",
                 owner[s], c.phase, c.error, c.bad_site, c.levels);
        fail(eng, (gst_status)results[owner[s]].status, msg);
      }
      if (c.error & ERR_EXTRACT) results[owner[s]].status = GST_DEVICE_ERROR;
      lat[owner[s]] = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() -
                                                               t_call).count();
      owner[s] = -1;
      active--;
    }
  }
  CK(cudaEventRecord(eng->ev1, eng->stream));
  CK(cudaEventSynchronize(eng->ev1));
  float ms = 0;
  cudaEventElapsedTime(&ms, eng->ev0, eng->ev1);
  double kms[3] = {0, 0, 0};
  for (auto& pr : eng->cs.prof) {
    float e = 0;
    if (cudaEventElapsedTime(&e, eng->prof_events[2 * pr.second],
                             eng->prof_events[2 * pr.second + 1]) == cudaSuccess)
      kms[pr.first] += e;
  }
  for (int32_t i = 0; i < n; i++) {
    gst_stats& st = results[i].stats;
    st.device_ms = ms;
    st.latency_ms = lat[i];
    st.kernel_launches = eng->cs.launches;
    st.h2d_bytes = eng->cs.h2d;
    st.d2h_bytes = eng->cs.d2h;
    st.grow_ms = kms[PROF_GROW];
    st.rows_ms = kms[PROF_ROWS];
    st.sssp_ms = kms[PROF_SSSP];
  }
  return GST_OK;
}

gst_status gst_solve(gst_graph* g, gst_groups* grp, const gst_query* q, gst_result* res) {
  gst_engine* eng = g ? g->eng : nullptr;
  if (!g || !grp || !q || !res) return fail(eng, GST_BAD_INPUT, "solve: null argument");
  gst_status s = validate_query(eng, grp, q);
  if (s != GST_OK) {
    memset(res, 0, sizeof(*res));
    res->status = s;
    res->user_tag = q->user_tag;
    return s;
  }
  const int32_t saved = eng->cfg.max_batch;
  eng->cfg.max_batch = 1;
  s = gst_solve_batch(g, grp, 1, q, res);
  eng->cfg.max_batch = saved;
  if (s != GST_OK) return s;
  return (gst_status)res->status;
}

gst_status gst_debug_slot_state(gst_graph* g, int32_t slot, uint64_t* cells, int64_t n_cells,
                                uint64_t* best_out) {
  gst_engine* eng = g ? g->eng : nullptr;
  if (!g || slot < 0 || (size_t)slot >= g->slots.size() || n_cells < 0)
    return fail(eng, GST_BAD_INPUT, "debug: bad slot");
  std::lock_guard<std::mutex> lk(eng->mu);
  CK(cudaSetDevice(eng->device));
  const Slot& s = g->slots[slot];
  const int64_t have = (int64_t)(s.V * s.rw_cap);
  if (cells && n_cells)
    CK(cudaMemcpyAsync(cells, s.table, (size_t)std::min(n_cells, have) * 8,
                       cudaMemcpyDeviceToHost, eng->stream));
  CK(cudaMemcpyAsync(g->h_ctx + slot, g->d_ctx + slot, sizeof(Ctx), cudaMemcpyDeviceToHost,
                     eng->stream));
  CK(cudaStreamSynchronize(eng->stream));
  if (best_out) *best_out = g->h_ctx[slot].best;
  return GST_OK;
}

void gst_result_free(gst_result* r) {
  if (!r) return;
  free(r->edge_u);
  free(r->edge_v);
  free(r->edge_w);
  r->edge_u = r->edge_v = r->edge_w = nullptr;
  r->n_edges = 0;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// No-allocation solve.
//
// Some callers cannot let a library call cudaMalloc: a host application that
// owns all device memory through its own pool (a database engine's GPU memory
// manager, a framework's caching allocator, a serving process that carves HBM up
// front) forbids stray allocations, and cudaMalloc / cudaFree also synchronise
// the device, stalling the caller's other streams.  gst_solve_noalloc serves
// them: the caller passes the graph and groups already in device memory and
// host buffers for the tree; every scratch buffer of the solve (query context,
// state table, one-label distances, worklists, extraction stack) lives in the
// file-scope array below, which the CUDA module reserves when it is loaded and
// keeps until the process exits — on every GPU that loads this library.
//
// The array is shared by every call on a device and keeps the previous call's
// contents; each call clears the parts that must start empty (state table,
// distances, dirty-row bitmap) before its kernels run.  Two calls whose work
// overlaps on the same GPU (different streams or host threads) race on the array
// and corrupt each other: serialise them.  The first call on a device looks up
// the array's device address (cudaGetSymbolAddress, with that device current)
// and caches it; make that first call before any stream capture.
// ---------------------------------------------------------------------------
namespace {

constexpr size_t kNoallocScratchBytes = (size_t)64 << 20;  // GST_NOALLOC_SCRATCH_BYTES
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoallocScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mu;
void* g_noalloc_ptr[kMaxDevices] = {nullptr};

size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

// Device address of the scratch array on `device` (must be current).  Host code
// cannot use the symbol itself: on the host it names a stand-in object, not
// device memory.
gst_status noalloc_scratch(int device, void** out) {
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  if (!g_noalloc_ptr[device]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) {
      tl_err = std::string("noalloc: cudaGetSymbolAddress: ") + cudaGetErrorString(e);
      return GST_DEVICE_ERROR;
    }
    g_noalloc_ptr[device] = p;
  }
  *out = g_noalloc_ptr[device];
  return GST_OK;
}

gst_status noalloc_fail(gst_status s, const char* msg) {
  tl_err = msg;
  return s;
}

gst_status noalloc_solve(int device, cudaStream_t st, int64_t V, int64_t E, const int64_t* d_beg,
                         const int32_t* d_edges, int32_t n_groups, const int64_t* d_grp_ptr,
                         const int32_t* d_members, const gst_query* q, int64_t edge_cap,
                         gst_result* res) {
  gst_engine* eng = nullptr;  // for CK()
  if (!res) return noalloc_fail(GST_BAD_INPUT, "noalloc: null result");
  int32_t* eu = res->edge_u;
  int32_t* ev = res->edge_v;
  int32_t* ew = res->edge_w;
  memset(res, 0, sizeof(*res));
  res->edge_u = eu;
  res->edge_v = ev;
  res->edge_w = ew;
  if (!q || !d_beg || !d_grp_ptr || !d_members || (E > 0 && !d_edges) || V < 1 ||
      V >= ((int64_t)1 << 27) || E < 0 || n_groups < 1 || edge_cap < 0 ||
      (edge_cap > 0 && (!eu || !ev || !ew)))
    return noalloc_fail(GST_BAD_INPUT, "noalloc: bad arguments");
  res->user_tag = q->user_tag;
  if (q->k < 1 || q->k > KMAX || !q->group_ids || q->hop_bound > 30)
    return res->status = GST_BAD_INPUT,
           noalloc_fail(GST_BAD_INPUT, "noalloc: k must be in [1,8], hop bound <= 30");
  for (int i = 0; i < q->k; i++) {
    const int32_t a = q->group_ids[i];
    if (a < 0 || a >= n_groups)
      return res->status = GST_BAD_INPUT, noalloc_fail(GST_BAD_INPUT, "noalloc: group id out of range");
    for (int j = 0; j < i; j++)
      if (q->group_ids[j] == a)
        return res->status = GST_BAD_INPUT, noalloc_fail(GST_BAD_INPUT, "noalloc: duplicate group id");
  }
  // scratch layout; reject what does not fit
  const int hop = q->hop_bound >= 0;
  const size_t RW = row_width(q->k, q->hop_bound);
  const uint32_t outcap = 1u << 14, stackcap = 1u << 16;
  size_t off = align256(sizeof(Ctx));
  const size_t o_table = off;
  off = align256(off + (size_t)V * RW * 8);
  const size_t o_dist = off;
  off = align256(off + (size_t)V * DIST_STRIDE * 4);
  const size_t o_bits = off;
  off = align256(off + ((size_t)V + 31) / 32 * 4);
  const size_t o_rows = off;
  off = align256(off + (size_t)V * 4);
  const size_t o_out = off;
  off = align256(off + (size_t)outcap * 12);
  const size_t o_stack = off;
  off = align256(off + (size_t)stackcap * 8);
  const size_t o_tour = off;
  off = align256(off + kTourWords * 4);
  const size_t min_lists = 4 * (size_t)(4 * V + 4096) * 16;
  if (off + min_lists > kNoallocScratchBytes) {
    char msg[200];
    snprintf(msg, sizeof msg,
             "noalloc: this query needs more than the %zu-byte static scratch "
             "(V=%lld, row width %zu); use gst_solve",
             kNoallocScratchBytes, (long long)V, RW);
    res->status = GST_OOM_ADMISSION;
    return noalloc_fail(GST_OOM_ADMISSION, msg);
  }
  const uint64_t want = (uint64_t)V * RW + 4ull * (uint64_t)V + 4096;
  const uint64_t fit = (kNoallocScratchBytes - off) / (4 * 16);
  const uint32_t cap = (uint32_t)std::min<uint64_t>(std::min<uint64_t>(want, fit), 1ull << 26);

  int prev_dev = 0;
  CK(cudaGetDevice(&prev_dev));
  CK(cudaSetDevice(device));
  void* scratch = nullptr;
  gst_status s = noalloc_scratch(device, &scratch);
  if (s != GST_OK) {
    cudaSetDevice(prev_dev);
    res->status = s;
    return s;
  }
  unsigned char* base = (unsigned char*)scratch;
  // empty-group check: members of each queried group
  for (int i = 0; i < q->k; i++) {
    int64_t be[2];
    CK(cudaMemcpyAsync(be, d_grp_ptr + q->group_ids[i], sizeof(be), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    if (be[1] <= be[0]) {
      cudaSetDevice(prev_dev);
      res->status = GST_BAD_INPUT;
      return noalloc_fail(GST_BAD_INPUT, "noalloc: group has no members");
    }
  }
  int sms = 148;
  CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
  gst_config cfg;
  gst_config_default(&cfg);
  const int split = cfg.split_degree;
  Ctx c;
  memset(&c, 0, sizeof(c));
  c.table = (uint64_t*)(base + o_table);
  c.dist = (uint32_t*)(base + o_dist);
  c.rowbits = (uint32_t*)(base + o_bits);
  c.tour = (uint32_t*)(base + o_tour);
  c.q[0] = (uint4*)(base + off);
  c.q[1] = (uint4*)(base + off + (size_t)cap * 16);
  c.far[0] = (uint4*)(base + off + 2 * (size_t)cap * 16);
  c.far[1] = (uint4*)(base + off + 3 * (size_t)cap * 16);
  c.rows = (uint32_t*)(base + o_rows);
  c.out = (int32_t*)(base + o_out);
  c.stack = (uint64_t*)(base + o_stack);
  c.qcap = c.farcap = cap;
  c.rowcap = (uint32_t)V;
  c.outcap = outcap;
  c.stackcap = stackcap;
  c.k = q->k;
  c.W = 1 << q->k;
  c.full = c.W - 1;
  c.D = hop ? q->hop_bound : 0;
  c.DD = hop ? q->hop_bound + 1 : 1;
  c.RW = c.W * c.DD;
  c.hop = hop;
  c.use_lb = hop ? 0 : 1;
  c.use_tour = c.use_lb;
  for (int i = 0; i < q->k; i++) c.gid[i] = q->group_ids[i];
  memset(c.vv, 0xFF, sizeof(c.vv));
  c.delta = 0;
  c.max_levels = (uint32_t)cfg.max_levels;
  c.in_idx = 1;
  c.far_min = 0xFFFFFFFFu;
  c.bucket_end = 0xFFFFFFFFu;
  c.ub = 0xFFFFFFFFu;
  c.ub_cell = 0xFFFFFFFFu;
  c.best = ~0ull;
  c.phase = c.use_lb ? PH_SSSP : PH_DP;
  Ctx* d_ctx = (Ctx*)base;
  // clear what must start empty, then upload the context
  CK(cudaMemsetAsync(c.table, 0xFF, (size_t)V * RW * 8, st));
  CK(cudaMemsetAsync(c.dist, 0xFF, (size_t)V * DIST_STRIDE * 4, st));
  CK(cudaMemsetAsync(c.rowbits, 0, ((size_t)V + 31) / 32 * 4, st));
  CK(cudaMemcpyAsync(d_ctx, &c, sizeof(Ctx), cudaMemcpyHostToDevice, st));
  // the caller's edges are sorted by neighbour only: no light-edge index
  DevGraph G{V, E, d_beg, (const int2*)d_edges, (const int2*)d_edges, nullptr};
  k_init<<<dim3(64, 1), 256, 0, st>>>(d_ctx, 1, G, d_grp_ptr, d_members, split);
  k_ctrl<<<1, 32, 0, st>>>(d_ctx, 1, CTRL_SSSP);
  const int blocks = sms * cfg.blocks_per_sm;
  const size_t per_warp = rows_smem_per_warp((int)RW);
  const int warps = cfg.threads_per_block / 32;
  cudaFuncSetAttribute(k_rows, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
  int64_t launches = 2;
  Ctx h;
  const auto t0 = std::chrono::steady_clock::now();
  for (;;) {
    for (int i = 0; i < 6; i++) {
      k_sssp<<<blocks, 256, 0, st>>>(d_ctx, 1, G, split);
      k_ctrl<<<1, 32, 0, st>>>(d_ctx, 1, CTRL_SSSP);
      k_rows<<<blocks, warps * 32, per_warp * warps, st>>>(d_ctx, 1, G, split, (int)RW);
      k_ctrl<<<1, 32, 0, st>>>(d_ctx, 1, CTRL_DP_ROWS);
      k_grow<<<blocks, 256, 0, st>>>(d_ctx, 1, G, split);
      k_ctrl<<<1, 32, 0, st>>>(d_ctx, 1, CTRL_DP_GROW);
      launches += 6;
    }
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(&h, d_ctx, sizeof(Ctx), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    if (h.phase >= PH_DONE) break;
  }
  k_extract<<<1, 32, 0, st>>>(d_ctx, 1, G);
  launches++;
  CK(cudaMemcpyAsync(&h, d_ctx, sizeof(Ctx), cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  res->status = status_of(h);
  if (h.error & ERR_EXTRACT) res->status = GST_DEVICE_ERROR;
  res->stats.levels = h.levels;
  res->stats.states_expanded = (int64_t)h.st_items;
  res->stats.edge_relaxations = (int64_t)h.st_relax;
  res->stats.merge_pairs = (int64_t)h.st_merge;
  res->stats.rows_merged = (int64_t)h.st_rows;
  res->stats.sssp_relaxations = (int64_t)h.st_sssp;
  res->stats.kernel_launches = launches;
  res->stats.latency_ms =
      std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  res->stats.device_ms = res->stats.latency_ms;
  if (res->status == GST_OK) {
    res->cost = (int32_t)(h.best >> 32);
    res->root = (int32_t)(h.best & 0x7FFFFFFull);
    res->root_hop = (int32_t)((h.best >> 27) & 31u);
    const int64_t nraw = std::min<int64_t>(h.n_out, outcap);
    if (nraw > edge_cap) {
      res->status = GST_CAPACITY;
    } else if (nraw > 0) {
      // scatter the interleaved (u, v, w) triples into the caller's three arrays
      CK(cudaMemcpy2DAsync(eu, 4, c.out + 0, 12, 4, (size_t)nraw, cudaMemcpyDeviceToHost, st));
      CK(cudaMemcpy2DAsync(ev, 4, c.out + 1, 12, 4, (size_t)nraw, cudaMemcpyDeviceToHost, st));
      CK(cudaMemcpy2DAsync(ew, 4, c.out + 2, 12, 4, (size_t)nraw, cudaMemcpyDeviceToHost, st));
      CK(cudaStreamSynchronize(st));
      // in place: orient u < v, drop repeated edges, sort by (u, v)
      int64_t m = 0;
      for (int64_t i = 0; i < nraw; i++) {
        int32_t a = eu[i], b = ev[i];
        if (a > b) std::swap(a, b);
        bool dup = false;
        for (int64_t j = 0; j < m && !dup; j++) dup = eu[j] == a && ev[j] == b;
        if (dup) continue;
        const int32_t w = ew[i];
        int64_t p = m++;
        while (p > 0 && (eu[p - 1] > a || (eu[p - 1] == a && ev[p - 1] > b))) {
          eu[p] = eu[p - 1];
          ev[p] = ev[p - 1];
          ew[p] = ew[p - 1];
          p--;
        }
        eu[p] = a;
        ev[p] = b;
        ew[p] = w;
      }
      res->n_edges = m;
    }
  }
  cudaSetDevice(prev_dev);
  return res->status == GST_OK ? GST_OK : (gst_status)res->status;
}

}  // namespace

extern "C" gst_status gst_solve_noalloc(int32_t device, void* stream, int64_t V, int64_t E,
                                        const int64_t* d_beg_pos, const int32_t* d_edges,
                                        int32_t n_groups, const int64_t* d_grp_ptr,
                                        const int32_t* d_members, const gst_query* q,
                                        int64_t edge_cap, gst_result* res) {
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev ||
      device >= kMaxDevices)
    return noalloc_fail(GST_BAD_INPUT, "noalloc: bad device");
  return noalloc_solve(device, (cudaStream_t)stream, V, E, d_beg_pos, d_edges, n_groups,
                       d_grp_ptr, d_members, q, edge_cap, res);
}
