// Host side of the GST engine and its C ABI (include/gst.h).
//
// A gst_graph owns the device CSR.  Queries run in a Runner: a set of resident
// query slots (state slab, one-label distances, worklists, control context) that
// share every launch of the level loop.  gst_solve_batch drives a runner from a
// list of queries; a gst_server drives its own runner from a submission queue on a
// host thread, admitting new queries at level boundaries (continuous batching).
// Slot memory comes from the engine's stream-ordered memory pool and is admitted
// against a memory budget by the size of each query's state table.
//
// The level loop is a fixed launch sequence (sssp, ctrl, rows, ctrl, grow, ctrl)
// that every resident query steps through together; each kernel reads its work
// counts from the device-side contexts, so launches after a query finishes are
// no-ops for it.  The host either issues a few levels ahead and then reads the
// contexts back, or (cfg.use_graphs) launches one CUDA graph whose conditional
// WHILE node repeats the level body on the device until a query finishes.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <utility>
#include <vector>

#include <cuda_runtime.h>

#include "gst.h"
#include "gst_device.cuh"
#include "gst_bsearch.cuh"

using namespace gst;

namespace {

thread_local std::string tl_err;

using Clock = std::chrono::steady_clock;

// Device memory of one query slot: one pool allocation carved into the buffers.
struct SlotMem {
  void* base = nullptr;
  size_t bytes = 0;
  size_t table_bytes = 0; // state rows (the row pool) of the slot
  size_t table_dirty = 0; // bytes at the table's start that may hold written cells
  uint32_t cap = 0;       // near-list capacity (items)
  uint32_t farcap = 0;    // far-list capacity (0 when the frontier has one bucket)
  uint64_t* table = nullptr;
  uint32_t* rowmap = nullptr;  // vertex -> pool row
  uint32_t* dist = nullptr;
  uint32_t* rowbits = nullptr;
  uint32_t* fm[2] = {nullptr, nullptr};
  uint32_t* snap = nullptr;
  uint32_t* dist_h = nullptr;  // hop budgets 1..nhb of the one-label distances
  int nhb = 0;
  uint32_t ds = 0;             // uint32 per distance row the buffers were carved for
  uint32_t* tour = nullptr;
  uint4* q[2] = {nullptr, nullptr};
  uint4* far[2] = {nullptr, nullptr};
  uint32_t* rows = nullptr;
  int32_t* out = nullptr;
  uint64_t* stack = nullptr;
  uint32_t rowcap = 0, outcap = 0, stackcap = 0;
};

constexpr size_t kTourWords = ((size_t)1 << KMAX) * (TOUR_STRIDE + KMAX);
constexpr uint32_t kOutCap = 1u << 16;
constexpr uint32_t kStackCap = 1u << 18;

size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

// Frontier bytes of the distance search: one per vertex (four to a word), padded to
// whole 16-byte words.
size_t fm_bytes(int64_t V) { return ((size_t)V + 15) / 16 * 16; }

// Rows of a query's row pool: an eighth of the vertices (at least 64k rows), four times
// more per capacity retry.  A query writes rows for a few percent of the vertices (its
// pruning keeps the DP near the optimal trees).  A pool of half the vertices or more
// becomes the dense layout (one row per vertex, no map): small graphs, last retries.
uint32_t pool_rows(int64_t V, int boost) {
  uint64_t r = std::max<uint64_t>(1u << 16, (uint64_t)V / 8);
  for (int i = 0; i < boost; i++) r *= 4;
  return r * 2 >= (uint64_t)V ? (uint32_t)V : (uint32_t)r;
}

// Lay out (or, with base == nullptr, only size) a slot of V vertices: a row pool of
// `rows` rows of rw cells and the per-vertex buffers.
size_t carve_slot(SlotMem& m, unsigned char* base, int64_t V, size_t rw, uint32_t rows,
                  uint32_t cap, uint32_t farcap, int nhb, uint32_t ds) {
  size_t off = 0;
  auto take = [&](size_t n) {
    unsigned char* p = base ? base + off : nullptr;
    off = align256(off + n);
    return p;
  };
  m.table_bytes = (size_t)rows * rw * 8;
  m.table_dirty = m.table_bytes;  // fresh memory: cleared before first use
  m.table = (uint64_t*)take(m.table_bytes);
  m.rowmap = (uint32_t*)take((size_t)V * 4);
  m.dist = (uint32_t*)take((size_t)V * ds * 4);
  m.ds = ds;
  m.rowbits = (uint32_t*)take(((size_t)V + 31) / 32 * 4);
  m.fm[0] = (uint32_t*)take(fm_bytes(V));
  m.fm[1] = (uint32_t*)take(fm_bytes(V));
  m.snap = (uint32_t*)take((size_t)V * ds * 4);
  m.dist_h = (uint32_t*)take((size_t)nhb * (size_t)V * ds * 4);
  m.nhb = nhb;
  m.tour = (uint32_t*)take(kTourWords * 4);
  m.q[0] = (uint4*)take((size_t)cap * 16);
  m.q[1] = (uint4*)take((size_t)cap * 16);
  m.far[0] = (uint4*)take((size_t)farcap * 16);
  m.far[1] = (uint4*)take((size_t)farcap * 16);
  m.rows = (uint32_t*)take((size_t)V * 4);
  m.out = (int32_t*)take((size_t)kOutCap * 12);
  m.stack = (uint64_t*)take((size_t)kStackCap * 8);
  m.cap = cap;
  m.farcap = farcap;
  m.rowcap = (uint32_t)V;
  m.outcap = kOutCap;
  m.stackcap = kStackCap;
  return off;
}

size_t row_width(int k, int D) { return ((size_t)1 << k) * (size_t)(D >= 0 ? D + 1 : 1); }

// Hop budgets 1..n of the one-label distances kept for a hop bound D (budget D is the
// distance table itself, budget 0 the group members).
int hop_budgets(int D) { return D > 1 ? std::min(D - 1, HOP_BUDGETS_MAX) : 0; }

// Worklist capacity.  A level appends at most one item per edge chunk of every
// state it settles, which in the worst case is every cell of the slab; queries
// use a small fraction of that, so a slot starts at `base` items and a query that
// overflows is re-run with four times the room (up to the worst case).
uint32_t list_cap(int64_t V, int64_t E, size_t rw, int split, int boost) {
  const uint64_t worst = std::min<uint64_t>((uint64_t)V * rw + (uint64_t)E / split * rw + 4096,
                                            (1ull << 31));
  uint64_t c = std::max<uint64_t>(1ull << 16, 8ull * (uint64_t)V + 2ull * (uint64_t)E / split);
  for (int i = 0; i < boost; i++) c *= 4;
  return (uint32_t)std::min(c, worst);
}
bool cap_is_worst(int64_t V, int64_t E, size_t rw, int split, uint32_t cap) {
  return cap >= std::min<uint64_t>((uint64_t)V * rw + (uint64_t)E / split * rw + 4096, 1ull << 31);
}

}  // namespace

struct gst_engine {
  int device = 0;
  gst_config cfg{};
  cudaStream_t stream = nullptr;
  cudaMemPool_t pool = nullptr;
  std::vector<cudaEvent_t> prof_events;  // reused start/stop pairs for cfg.profile_kernels
  int sms = 148;
  int grow_blocks = 0, sssp_blocks = 0;
  std::vector<std::pair<uint64_t, int>> rows_occ;  // (threads<<32 | smem) -> grid
  size_t rows_smem = 0;                            // dynamic shared memory a rows CTA may take
  std::atomic<int> graphs{0};                      // live graphs (the engine outlives them)
  cudaEvent_t bs_ev[2] = {nullptr, nullptr};       // timing of batch-shared searches
  std::string err;
  std::mutex mu;                                   // serialises all GPU work of the engine
};

namespace {
struct Runner;
}

struct gst_graph {
  gst_engine* eng = nullptr;
  int64_t V = 0, E = 0;
  int64_t* d_beg = nullptr;
  int2* d_edges = nullptr;   // per vertex sorted by neighbour (tree extraction)
  int2* d_wedges = nullptr;  // per vertex sorted by (weight, neighbour) (grow, SSSP)
  uint32_t* d_widx = nullptr;
  int64_t max_deg = 0;       // shape of the graph (autotuner cache key)
  int32_t max_w = 0;
  // Vertices are renumbered on the device by degree, highest first (ties by id), so that
  // the rows of the vertices most relaxations land on (the high-degree ones) pack into
  // few cache lines; groups and results are translated at the boundary.
  std::vector<int32_t> to_dev;    // caller's vertex id -> device id
  std::vector<int32_t> to_host;   // device id -> caller's vertex id
  std::unique_ptr<Runner> batch;  // runner of gst_solve / gst_solve_batch (slots kept)
};

struct gst_groups {
  gst_graph* g = nullptr;
  int32_t n = 0;
  int64_t* d_ptr = nullptr;
  int32_t* d_mem = nullptr;
  std::vector<int64_t> h_ptr;
  // One-label distance caches: the distances of a group to every vertex depend on the
  // group only, not on the query, so hot groups keep theirs on the device (least
  // recently warmed replaced first).  `cache`: unlimited distances, V uint32 per group.
  // `hop_cache`: the distances within hop budgets 1..n (n = min(D-1, 7)) and within D
  // for one hop bound D, (n+1) x V uint32 per group in that order.
  struct Cache {
    uint32_t* d_vec = nullptr;       // cap x stride
    int32_t cap = 0;
    int32_t D = -1;                  // hop bound of the entries (-1: unlimited)
    size_t stride = 0;               // uint32 per entry
    std::vector<int32_t> slot_of;    // group id -> slot, -1 if not cached
    std::vector<int32_t> gid_of;     // slot -> group id, -1 if empty
    std::vector<uint64_t> used;      // slot -> last warm call that listed it
    uint64_t clock = 0;
    const uint32_t* vec(int32_t gid) const {
      const int32_t s = gid >= 0 && gid < (int32_t)slot_of.size() ? slot_of[gid] : -1;
      return s < 0 ? nullptr : d_vec + (size_t)s * stride;
    }
  } cache, hop_cache;
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

// Dynamic shared memory a rows-kernel CTA may take on `device`: the opt-in maximum
// per block less the kernel's static shared memory.
size_t rows_smem_limit(int device) {
  int optin = 0;
  if (cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device) != cudaSuccess)
    optin = 48 * 1024;
  cudaFuncAttributes fa{};
  cudaFuncGetAttributes(&fa, k_rows);
  return optin > (int)fa.sharedSizeBytes ? (size_t)optin - fa.sharedSizeBytes : 0;
}

// Warps per CTA of the rows kernel when the widest resident row has rwm cells: the
// configured CTA size (threads_per_block, at most 8 warps), fewer when that many
// warps' rows do not fit the shared memory; 0 when not even one does.
int rows_warps(size_t smem_limit, int threads_per_block, int rwm) {
  const size_t per = rows_smem_per_warp(rwm);
  const int want = std::max(1, std::min(8, threads_per_block / 32));
  return (int)std::min<size_t>((size_t)want, smem_limit / per);
}

gst_status validate_query(gst_engine* eng, const gst_groups* grp, const gst_query* q) {
  if (!q || q->k < 1 || q->k > KMAX || !q->group_ids)
    return fail(eng, GST_BAD_INPUT, "query: k must be in [1,8] with group ids");
  if (q->hop_bound > 30) return fail(eng, GST_BAD_INPUT, "query: hop bound must be <= 30");
  // one row of the query's states must fit one warp's shared memory in the rows kernel
  // (2^k x (D+1) cells; every k <= 8, D <= 30 row fits the 227 KB of a B200 CTA)
  if (rows_warps(eng->rows_smem, 32, (int)(((size_t)1 << q->k) * (q->hop_bound >= 0 ? q->hop_bound + 1 : 1))) < 1)
    return fail(eng, GST_BAD_INPUT, "query: its state row does not fit the rows kernel's shared memory");
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

gst_status status_of(const Ctx& c) {
  if (c.error & ERR_TIMEOUT) return GST_TIMEOUT;
  if (c.error & (ERR_QCAP | ERR_FARCAP | ERR_ROWCAP | ERR_POOL)) return GST_CAPACITY;
  if (c.error) return GST_DEVICE_ERROR;
  if (c.phase != PH_DONE) return GST_DEVICE_ERROR;
  if (c.best == ~0ull) return GST_INFEASIBLE;
  return GST_OK;
}

DevGraph dev_graph(const gst_graph* g) {
  return DevGraph{g->V, g->E, g->d_beg, g->d_edges, g->d_wedges, g->d_widx};
}

// Grid of the rows kernel: every SM filled with as many CTAs as its registers and
// shared memory allow (the dynamic shared memory grows with the row width), capped
// at cfg.blocks_per_sm.
int rows_blocks(gst_engine* eng, int threads, size_t smem) {
  const uint64_t key = ((uint64_t)threads << 32) | (uint64_t)smem;
  for (auto& kv : eng->rows_occ)
    if (kv.first == key) return kv.second;
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_rows, threads, smem) != cudaSuccess ||
      per_sm < 1)
    per_sm = 1;
  const int blocks = eng->sms * std::min(per_sm, std::max(1, eng->cfg.blocks_per_sm));
  eng->rows_occ.push_back({key, blocks});
  return blocks;
}

// Launch geometry derived from the configuration (grids sized by occupancy).
void apply_launch_config(gst_engine* eng) {
  int occ_grow = 1, occ_sssp = 1;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_grow, k_grow, 256, 0);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_sssp, k_sssp, 256, 0);
  eng->grow_blocks = eng->sms * std::max(1, std::min(occ_grow, eng->cfg.blocks_per_sm));
  eng->sssp_blocks = eng->sms * std::max(1, std::min(occ_sssp, eng->cfg.blocks_per_sm));
  eng->rows_occ.clear();
}

// The query-dependent fields of a fresh context (zeroed by the caller), shared by the
// runner's slots and the no-allocation solve: sizes, pruning switches, bounds, phase
// and the distance search's item form.
void init_query_ctx(Ctx& c, const gst_query* q, const gst_config& cfg) {
  const int hop = q->hop_bound >= 0;
  c.k = q->k;
  c.W = 1 << q->k;
  c.full = c.W - 1;
  c.D = hop ? q->hop_bound : 0;
  c.DD = hop ? q->hop_bound + 1 : 1;
  c.RW = c.W * c.DD;
  c.hop = hop;
  // The one-label and tour bounds of the unbounded problem are lower bounds of the
  // hop-bounded one too (a hop-feasible completion is also an unbounded one), so
  // hop-bounded queries prune with them against their own bound ub_cell.
  c.use_lb = 1;
  c.use_tour = 1;
  c.cut_pm = hop ? (cfg.hop_cut_permille > 0
                       ? (uint32_t)cfg.hop_cut_permille
                       : 1000u * (uint32_t)(cfg.hop_cut_mult > 0 ? cfg.hop_cut_mult : 1))
                 : (uint32_t)(cfg.search_cut_permille > 0 ? cfg.search_cut_permille : 1000);
  // A tree of diameter <= D reaches every missing group within D edges of any of its
  // vertices, so hop-bounded queries bound with the cheapest paths of at most D
  // edges (a level-synchronous search of D rounds), tighter than unlimited ones.
  c.sssp_hops = hop && q->hop_bound > 0 ? (uint32_t)q->hop_bound : 0u;
  for (int i = 0; i < q->k; i++) c.gid[i] = q->group_ids[i];
  memset(c.vv, 0xFF, sizeof(c.vv));
  c.delta = (uint32_t)std::max(0, cfg.bucket_delta);
  c.max_levels = (uint32_t)cfg.max_levels;
  c.in_idx = 1;
  c.far_min = 0xFFFFFFFFu;
  // the hop-limited search runs one round per step, in one cost bucket
  c.bucket_end = c.delta && !c.sssp_hops ? c.delta : 0xFFFFFFFFu;
  c.ub = 0xFFFFFFFFu;
  c.cut = 0xFFFFFFFFu;
  c.ub_cell = 0xFFFFFFFFu;
  c.ub_hop = 0xFFFFFFFFu;
  c.best = ~0ull;
  c.phase = c.use_lb ? PH_SSSP : PH_DP;
  // one distance-search item per (vertex, groups): hop-limited distances in rounds,
  // unlimited ones when the search runs in one bucket
  c.sssp_mask = c.sssp_hops ? 2u : (c.bucket_end == 0xFFFFFFFFu ? 1u : 0u);
}

enum ProfKind { PROF_GROW = 0, PROF_ROWS = 1, PROF_SSSP = 2, PROF_BSRELAX = 3, PROF_KINDS = 4 };

// A query waiting for, or holding, a slot.
struct Job {
  gst_query q{};
  int32_t gids[KMAX] = {0};
  gst_result* out = nullptr;     // destination of the result
  uint64_t ticket = 0;
  Clock::time_point t_submit;
  int boost = 0;                 // worklist capacity boost (capacity retries)
  size_t rw = 0;
  int nhb = 0;                   // hop budgets of the one-label distances
  uint32_t ds = DIST_STRIDE;     // uint32 per distance row
  uint32_t* cache_dst = nullptr; // a group-cache fill: the distances of group gids[0] to
                                 // every vertex go here (V entries), no DP
  // batch-shared search: 1 when a shared table of the runner holds this query's distances
  // (its groups in columns ss_cols), exact up to ss_cut; 2 when its table was given back
  // before it was admitted (it searches on its own)
  int ss = 0;
  uint16_t ss_cols[KMAX] = {0};
  uint32_t ss_cut = 0;
  std::atomic<bool> done{false};
};

// Per-call accounting (launches, bytes moved, profiled kernel time).
struct CallStats {
  int64_t launches = 0, h2d = 0, d2h = 0;
  int64_t graph_launches = 0, graph_levels = 0;
  int64_t allocs = 0, alloc_bytes = 0;
  double alloc_ms = 0;
  int64_t bs_sectors = 0, bs_launches = 0, bs_relax = 0;  // batch-shared searches of the call
  double bs_ms = 0;
  std::vector<std::pair<int, int>> prof;  // (kernel kind, event-pair index)
  size_t next_ev = 0;
};

// Resident query slots and the level loop over them.
struct Runner {
  gst_engine* eng;
  gst_graph* g;
  gst_groups* grp = nullptr;
  int max_slots;
  size_t budget = 0;            // bytes of slot memory the runner may hold
  size_t held = 0;              // bytes reserved from the pool (arenas)
  // Slot memory is carved from a few large arenas taken from the pool (first fit,
  // freed ranges coalesced): the pool maps physical memory for an allocation of a
  // new size, which costs far more than a query at these sizes, so slots of
  // varying size are sub-allocated from memory mapped once.
  struct Arena {
    unsigned char* base = nullptr;
    size_t size = 0;
    std::vector<std::pair<size_t, size_t>> free_;  // (offset, size), sorted by offset
  };
  std::vector<Arena> arenas;
  Ctx* d_ctx = nullptr;         // MAXB contexts
  Ctx* h_ctx = nullptr;         // pinned mirror
  uint32_t* d_loop = nullptr;   // graph loop: {iterations left, any query finished}
  uint32_t* loop_init = nullptr;  // pinned: values for d_loop before a launch
  uint32_t* loop_left = nullptr;  // pinned: iterations left after it
  std::vector<SlotMem> mem;
  std::vector<Job*> owner;      // slot -> job (nullptr = free)
  std::vector<uint8_t> idle_written;
  int nctx = 0;                 // slots the kernels scan (high-water mark)
  int active = 0;
  CallStats cs;
  // CUDA graphs of the level loop, by (nctx, rw_max)
  struct LoopGraph {
    int nctx;
    int rw_max;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
  };
  std::vector<LoopGraph> graphs;
  // Batch-shared distance search (gst_bsearch.cuh): its table lives in the arenas until
  // every query of its chunk has been admitted (and gathered its columns).
  struct Shared {
    void* mem = nullptr;
    size_t bytes = 0;
    BsCtx* d_b = nullptr;
    int remaining = 0;
    int D = 0;                       // 0: unbounded distances; else the hop bound
    uint32_t Gp = 0;                 // columns of the tables
    uint32_t* tab[KMAX + 1] = {};    // hop-bounded: d^{<=h} tables (device); tab[D] = dist
    uint32_t* dist = nullptr;        // the distance table (device)
  };
  std::vector<Shared> shs;           // pending shared tables, at most one per kind (D)
  Shared* shared_of(int D) {
    for (Shared& x : shs)
      if (x.D == D && x.d_b) return &x;
    return nullptr;
  }

  Runner(gst_engine* e, gst_graph* gr, int slots) : eng(e), g(gr), max_slots(slots) {}
  ~Runner() { release(); }

  void release() {
    cudaSetDevice(eng->device);
    cudaStreamSynchronize(eng->stream);
    for (auto& lg : graphs) {
      if (lg.exec) cudaGraphExecDestroy(lg.exec);
      if (lg.graph) cudaGraphDestroy(lg.graph);
    }
    graphs.clear();
    shs.clear();  // their memory is in the arenas
    for (auto& a : arenas) cudaFreeAsync(a.base, eng->stream);
    cudaStreamSynchronize(eng->stream);
    arenas.clear();
    mem.clear();
    held = 0;
    if (d_ctx) cudaFree(d_ctx);
    if (h_ctx) cudaFreeHost(h_ctx);
    if (d_loop) cudaFree(d_loop);
    if (loop_init) cudaFreeHost(loop_init);
    loop_init = loop_left = nullptr;
    d_ctx = nullptr;
    h_ctx = nullptr;
    d_loop = nullptr;
  }

  gst_status init() {
    CK(cudaMalloc(&d_ctx, sizeof(Ctx) * MAXB));
    CK(cudaMallocHost(&h_ctx, sizeof(Ctx) * MAXB));
    CK(cudaMalloc(&d_loop, sizeof(uint32_t) * 4));
    CK(cudaMallocHost(&loop_init, sizeof(uint32_t) * 4));
    loop_left = loop_init + 2;
    mem.assign(max_slots, SlotMem());
    owner.assign(max_slots, nullptr);
    idle_written.assign(max_slots, 0);
    size_t free_b = 0, total_b = 0;
    CK(cudaMemGetInfo(&free_b, &total_b));
    // memory the engine's pool keeps but no allocation uses (arenas released by another
    // runner) is free for this one's slots too
    unsigned long long reserved = 0, used = 0;
    CK(cudaMemPoolGetAttribute(eng->pool, cudaMemPoolAttrReservedMemCurrent, &reserved));
    CK(cudaMemPoolGetAttribute(eng->pool, cudaMemPoolAttrUsedMemCurrent, &used));
    const size_t avail = free_b + (size_t)(reserved > used ? reserved - used : 0);
    budget = eng->cfg.mem_budget_bytes > 0 ? (size_t)eng->cfg.mem_budget_bytes
                                           : (size_t)(avail * 0.85);
    return GST_OK;
  }

  size_t job_bytes(const Job& j) const {
    SlotMem tmp;
    const int split = eng->cfg.split_degree;
    const uint32_t cap = list_cap(g->V, g->E, j.rw, split, j.boost);
    return carve_slot(tmp, nullptr, g->V, j.rw, pool_rows(g->V, j.boost), cap,
                      eng->cfg.bucket_delta > 0 ? cap : 0, j.nhb, j.ds);
  }

  int rw_max() const {
    size_t r = 1;
    for (int s = 0; s < nctx; s++)
      if (owner[s]) r = std::max(r, owner[s]->rw);
    return (int)r;
  }

  // A range of `need` bytes from the arenas, or nullptr.
  void* arena_take(size_t need) {
    // best fit: the smallest free range that holds `need`, so that the large ranges
    // that large slots (k = 7 hop-bounded tables run to 12 GB) leave behind stay whole
    Arena* ba = nullptr;
    size_t bi = 0;
    for (auto& a : arenas)
      for (size_t i = 0; i < a.free_.size(); i++)
        if (a.free_[i].second >= need && (!ba || a.free_[i].second < ba->free_[bi].second)) {
          ba = &a;
          bi = i;
        }
    if (!ba) return nullptr;
    const size_t off = ba->free_[bi].first;
    ba->free_[bi].first += need;
    ba->free_[bi].second -= need;
    if (ba->free_[bi].second == 0) ba->free_.erase(ba->free_.begin() + (long)bi);
    return ba->base + off;
  }
  // Return a range to its arena, merging it with free neighbours.
  void arena_give(void* p, size_t n) {
    for (auto& a : arenas) {
      unsigned char* q = (unsigned char*)p;
      if (q < a.base || q >= a.base + a.size) continue;
      const size_t off = (size_t)(q - a.base);
      auto it = std::lower_bound(a.free_.begin(), a.free_.end(), std::make_pair(off, (size_t)0));
      it = a.free_.insert(it, {off, n});
      const size_t i = (size_t)(it - a.free_.begin());
      if (i + 1 < a.free_.size() && a.free_[i].first + a.free_[i].second == a.free_[i + 1].first) {
        a.free_[i].second += a.free_[i + 1].second;
        a.free_.erase(a.free_.begin() + (long)i + 1);
      }
      if (i > 0 && a.free_[i - 1].first + a.free_[i - 1].second == a.free_[i].first) {
        a.free_[i - 1].second += a.free_[i].second;
        a.free_.erase(a.free_.begin() + (long)i);
      }
      return;
    }
  }
  // Reserve a new arena of at least `need` bytes within the budget: at least 4 GB, and
  // at least what is held already (geometric growth: mixed batches stop growing the
  // arenas after their first few, since new physical memory costs ~8-9 ms per GB).
  gst_status arena_grow(size_t need, bool* grown) {
    *grown = false;
    if (held + need > budget) return GST_OK;
    const size_t chunk = std::max(need, std::min(std::max((size_t)4 << 30, held), budget - held));
    void* p = nullptr;
    const auto ta = Clock::now();
    CK(cudaMallocFromPoolAsync(&p, chunk, eng->pool, eng->stream));
    cs.alloc_ms += std::chrono::duration<double, std::milli>(Clock::now() - ta).count();
    cs.allocs++;
    cs.alloc_bytes += (int64_t)chunk;
    Arena a;
    a.base = (unsigned char*)p;
    a.size = chunk;
    a.free_.push_back({0, chunk});
    arenas.push_back(a);
    held += chunk;
    *grown = true;
    return GST_OK;
  }
  // Memory of `need` bytes for a slot: a free range, else after returning idle
  // slots' memory (largest first), else from a new arena; nullptr if none fits.
  gst_status slot_memory(size_t need, void** out) {
    *out = arena_take(need);
    while (!*out) {
      int best = -1;
      for (int s = 0; s < (int)mem.size(); s++)
        if (!owner[s] && mem[s].base && (best < 0 || mem[s].bytes > mem[best].bytes)) best = s;
      if (best < 0) break;
      arena_give(mem[best].base, mem[best].bytes);
      mem[best] = SlotMem();
      *out = arena_take(need);
    }
    if (!*out) {
      // hand wholly free arenas back to the pool while a new one would not fit
      bool freed = false;
      for (size_t i = 0; i < arenas.size() && held + need > budget;) {
        Arena& a = arenas[i];
        if (a.free_.size() == 1 && a.free_[0].first == 0 && a.free_[0].second == a.size) {
          cudaFreeAsync(a.base, eng->stream);
          held -= a.size;
          arenas.erase(arenas.begin() + (long)i);
          freed = true;
        } else {
          i++;
        }
      }
      if (freed) {
        // the pool keeps freed memory reserved (its release threshold is unlimited):
        // give it back to the device before a new arena is mapped, or the pool would
        // hold both and run the device out of memory within the budget
        CK(cudaStreamSynchronize(eng->stream));
        CK(cudaMemPoolTrimTo(eng->pool, held));
      }
      bool grown = false;
      gst_status st = arena_grow(need, &grown);
      if (st != GST_OK) return st;
      if (grown) *out = arena_take(need);
    }
    return GST_OK;
  }

  // Put job j into a free slot.  GST_OK: admitted.  GST_NOT_READY: no slot or
  // memory free now (retry after a query finishes).  GST_OOM_ADMISSION: the
  // query's state table can never fit the budget.
  gst_status admit(Job* j) {
    const int split = eng->cfg.split_degree;
    const uint32_t cap = list_cap(g->V, g->E, j->rw, split, j->boost);
    const uint32_t farcap = eng->cfg.bucket_delta > 0 ? cap : 0;
    const size_t need = job_bytes(*j);
    if (need > budget) return GST_OOM_ADMISSION;
    const size_t need_table = (size_t)pool_rows(g->V, j->boost) * j->rw * 8;
    // the free slot whose memory already fits with the least to spare (a small query
    // does not take a large slot that a large one will want; among equals the lowest,
    // which keeps the contexts the kernels scan few), else the lowest free slot
    int s = -1;
    for (int i = 0; i < max_slots; i++)
      if (!owner[i] && mem[i].base && mem[i].table_bytes >= need_table && mem[i].cap >= cap &&
          mem[i].farcap >= farcap && mem[i].nhb >= j->nhb && mem[i].ds >= j->ds &&
          (s < 0 || mem[i].bytes < mem[s].bytes))
        s = i;
    if (s < 0) {
      for (int i = 0; i < max_slots && s < 0; i++)
        if (!owner[i]) s = i;
      if (s < 0) return GST_NOT_READY;
      if (mem[s].base) {
        arena_give(mem[s].base, mem[s].bytes);
        mem[s] = SlotMem();
      }
      void* p = nullptr;
      gst_status st = slot_memory(need, &p);
      if (st != GST_OK) return st;
      if (!p) return GST_NOT_READY;
      SlotMem m;
      carve_slot(m, (unsigned char*)p, g->V, j->rw, pool_rows(g->V, j->boost), cap, farcap, j->nhb,
                 j->ds);
      m.base = p;
      m.bytes = need;
      mem[s] = m;
    }
    SlotMem& m = mem[s];
    // fresh context
    Ctx& c = h_ctx[s];
    memset(&c, 0, sizeof(c));
    const gst_query* q = &j->q;
    const int hop = q->hop_bound >= 0;
    c.table = m.table;
    c.rowmap = m.rowmap;
    c.dist = m.dist;
    c.ds = j->ds;
    c.rowbits = m.rowbits;
    c.fm[0] = m.fm[0];
    c.fm[1] = m.fm[1];
    c.snap = m.snap;
    c.dist_h = m.dist_h;
    c.nhb = j->nhb;
    c.tour = m.tour;
    c.q[0] = m.q[0];
    c.q[1] = m.q[1];
    c.far[0] = m.far[0];
    c.far[1] = m.far[1];
    c.rows = m.rows;
    c.out = m.out;
    c.stack = m.stack;
    c.qcap = cap;
    c.farcap = farcap;
    c.rowcap = m.rowcap;
    c.outcap = m.outcap;
    c.stackcap = m.stackcap;
    init_query_ctx(c, q, eng->cfg);
    // a group-cache fill: the distances of one group, exact everywhere, then done
    if (j->cache_dst) {
      c.dist_only = 1;
      c.sssp_full = 1;
      c.bucket_end = 0xFFFFFFFFu;
      c.use_tour = 0;
    }
    // An unbounded query with cached groups: their distances are gathered from the
    // cache (exact everywhere; a member's distance 0 keeps its group out of the search).
    // With every group cached the query starts at the bounds pass; otherwise the search
    // runs for the other groups, its star bound already counting the cached ones.  A
    // hop-bounded query takes its cached groups from the hop cache of its bound, every
    // hop budget's table with them.  (The search's tentative star of D/2-edge paths may
    // then count a cached distance of more edges and come out low; it only sets the
    // search cutoff, which stays non-increasing, so every distance below the final
    // cutoff is still exact and the bounds stay valid.)
    GroupVecs gv{};
    const uint32_t* hv[KMAX] = {};
    int n_cached = 0;
    const size_t V = (size_t)g->V;
    if (!hop && !j->cache_dst) {
      for (int i = 0; i < q->k; i++) n_cached += (gv.v[i] = grp->cache.vec(c.gid[i])) != nullptr;
    } else if (hop && q->hop_bound > 0 && !j->cache_dst && grp->hop_cache.cap > 0 &&
               grp->hop_cache.D == q->hop_bound) {
      for (int i = 0; i < q->k; i++) n_cached += (hv[i] = grp->hop_cache.vec(c.gid[i])) != nullptr;
      for (int i = 0; i < q->k; i++) gv.v[i] = hv[i] ? hv[i] + (size_t)c.nhb * V : nullptr;
    }
    // a query of the batch-shared search: its distances are in the runner's shared
    // table, exact up to its cutoff; it starts at the bounds pass
    Shared* S = j->ss == 1 ? shared_of(hop ? q->hop_bound : 0) : nullptr;
    const bool shared = S != nullptr;
    if (shared) {
      n_cached = 0;
      c.cut_fix = std::max(1u, j->ss_cut);
      c.phase = PH_PREP;
    }
    const bool cached = n_cached > 0 || shared;
    if (n_cached == q->k) {
      c.sssp_full = 1;
      c.phase = PH_PREP;
    }
    c.sssp_mask = c.sssp_hops ? 2u : (c.bucket_end == 0xFFFFFFFFu ? 1u : 0u);
    cudaStream_t st = eng->stream;
    // the pool takes every row the slot's table holds; only the rows the slot's last
    // query wrote need clearing
    c.pool_cap = (uint32_t)std::min<uint64_t>((uint64_t)g->V, m.table_bytes / ((size_t)c.RW * 8));
    c.pool_n = 0;
    if (c.pool_cap >= (uint32_t)g->V) c.rowmap = nullptr;  // a row for every vertex: dense
    if (m.table_dirty) CK(cudaMemsetAsync(m.table, 0xFF, m.table_dirty, st));
    m.table_dirty = 0;
    if (c.rowmap) CK(cudaMemsetAsync(m.rowmap, 0xFF, (size_t)g->V * 4, st));
    CK(cudaMemsetAsync(m.rowbits, 0, ((size_t)g->V + 31) / 32 * 4, st));
    if (c.use_lb && !cached) CK(cudaMemsetAsync(m.dist, 0xFF, (size_t)g->V * c.ds * 4, st));
    CK(cudaMemsetAsync(m.fm[0], 0, fm_bytes(g->V), st));
    CK(cudaMemsetAsync(m.fm[1], 0, fm_bytes(g->V), st));
    if (c.nhb && !cached)
      CK(cudaMemsetAsync(m.dist_h, 0xFF, (size_t)c.nhb * (size_t)g->V * c.ds * 4, st));
    CK(cudaMemcpyAsync(d_ctx + s, &c, sizeof(Ctx), cudaMemcpyHostToDevice, st));
    cs.h2d += sizeof(Ctx) + sizeof(int32_t) * q->k;
    const DevGraph G = dev_graph(g);
    if (shared) {
      // the distance table, and for a hop-bounded query its budgets 1..nhb
      const uint16_t* sc = j->ss_cols;
      const ushort4 c0 = make_ushort4(sc[0], sc[1], sc[2], sc[3]);
      const ushort4 c1 = make_ushort4(sc[4], sc[5], sc[6], sc[7]);
      k_bs_gather<<<eng->sssp_blocks, 256, 0, st>>>(m.dist, c.ds, q->k, S->dist, S->Gp, c0, c1, g->V);
      cs.launches += 1;
      for (int h = 1; h <= c.nhb; h++) {
        k_bs_gather<<<eng->sssp_blocks, 256, 0, st>>>(m.dist_h + (size_t)(h - 1) * V * c.ds, c.ds,
                                                      q->k, S->tab[h], S->Gp, c0, c1, g->V);
        cs.launches += 1;
      }
      S->remaining--;
    } else if (cached) {
      k_gather_dist<<<eng->sssp_blocks, 256, 0, st>>>(m.dist, c.ds, q->k, gv, g->V);
      cs.launches += 1;
      if (hop)
        for (int h = 1; h <= c.nhb; h++) {
          GroupVecs gh{};
          for (int i = 0; i < q->k; i++) gh.v[i] = hv[i] ? hv[i] + (size_t)(h - 1) * V : nullptr;
          k_gather_dist<<<eng->sssp_blocks, 256, 0, st>>>(
              m.dist_h + (size_t)(h - 1) * V * c.ds, c.ds, q->k, gh, g->V);
          cs.launches += 1;
        }
    }
    k_init<<<dim3(64, 1), 256, 0, st>>>(d_ctx + s, 1, G, grp->d_ptr, grp->d_mem,
                                       eng->cfg.split_degree);
    if (n_cached == q->k || shared) {
      // the bounds pass over the distance rows (star bound, group distances), which
      // the control step after it turns into the tour table
      k_sssp<<<eng->sssp_blocks, 256, 0, st>>>(d_ctx + s, 1, G, eng->cfg.split_degree);
      cs.launches += 1;
    }
    k_ctrl<<<1, 32, 0, st>>>(d_ctx + s, 1, CTRL_SSSP);
    cs.launches += 2;
    owner[s] = j;
    idle_written[s] = 0;
    nctx = std::max(nctx, s + 1);
    active++;
    return GST_OK;
  }

  // Give back the shared tables whose queries have all been admitted (all of them with
  // `all`).
  void shared_release(bool all) {
    for (size_t i = 0; i < shs.size();) {
      if (all || shs[i].remaining <= 0) {
        if (shs[i].mem) arena_give(shs[i].mem, shs[i].bytes);
        shs.erase(shs.begin() + (std::ptrdiff_t)i);
      } else {
        i++;
      }
    }
  }

  // One batch-shared distance search for the queries `jobs`, all unbounded (D = 0) or all
  // of hop bound D (1..KMAX), over their distinct groups `cols` (at most BS_COLS groups,
  // BS_MAXQ queries).  On success every job is marked (ss = 1) with its columns and
  // cutoff; without memory for the tables, or when the search reports an error, the jobs
  // keep their own searches.
  gst_status shared_search(const std::vector<Job*>& jobs, const std::vector<int32_t>& cols, int D) {
    const int64_t V = g->V;
    const uint32_t ncols = (uint32_t)cols.size();
    const uint32_t Gp = (ncols + 7u) / 8u * 8u, Wm = (Gp + 31u) / 32u;
    if (D < 0 || D > KMAX) return GST_OK;
    const uint64_t item_cap = (uint64_t)V + (uint64_t)g->E / BS_CHUNK + 1024;
    if (item_cap >= (1ull << 32)) return GST_OK;
    size_t off = 0;
    auto take = [&](size_t n) {
      const size_t o = off;
      off = align256(off + n);
      return o;
    };
    const size_t o_b = take(sizeof(BsCtx));
    const size_t o_dist = take((size_t)V * Gp * 4 * (size_t)std::max(D, 1));  // tables 1..D
    const size_t o_fm0 = take((size_t)V * Wm * 4);
    const size_t o_fm1 = take((size_t)V * Wm * 4);
    const size_t o_am = take((size_t)V * Wm * 4);
    const size_t o_items = take((size_t)item_cap * 8);
    const size_t o_cols = take((size_t)BS_COLS * 4);
    void* p = nullptr;
    gst_status s = slot_memory(off, &p);
    if (s != GST_OK) return s;
    if (!p) return GST_OK;  // no room: the queries search on their own
    unsigned char* base = (unsigned char*)p;
    // held by the runner from here on (an error below gives it back with the others)
    shs.emplace_back();
    shs.back().mem = p;
    shs.back().bytes = off;
    shs.back().D = D;
    BsCtx h;
    memset(&h, 0, sizeof(h));
    h.D = (uint32_t)D;
    for (int t = 1; t <= D; t++) h.tab[t] = (uint32_t*)(base + o_dist + (size_t)(t - 1) * V * Gp * 4);
    h.dist = D ? h.tab[D] : (uint32_t*)(base + o_dist);
    h.fm[0] = (uint32_t*)(base + o_fm0);
    h.fm[1] = (uint32_t*)(base + o_fm1);
    h.am = (uint32_t*)(base + o_am);
    h.items = (uint2*)(base + o_items);
    h.item_cap = (uint32_t)item_cap;
    h.Gp = Gp;
    h.Wm = Wm;
    h.max_steps = (uint32_t)std::min(eng->cfg.max_levels, 1 << 16);
    const gst_config& cfg = eng->cfg;
    h.cut_pm = D ? (cfg.hop_cut_permille > 0
                        ? (uint32_t)cfg.hop_cut_permille
                        : 1000u * (uint32_t)(cfg.hop_cut_mult > 0 ? cfg.hop_cut_mult : 1))
                 : (uint32_t)(cfg.search_cut_permille > 0 ? cfg.search_cut_permille : 1000);
    h.nq = (uint32_t)jobs.size();
    for (size_t q = 0; q < jobs.size(); q++) {
      h.qk[q] = (uint32_t)jobs[q]->q.k;
      h.star[q] = COST_INF;
      for (int i = 0; i < jobs[q]->q.k; i++)
        h.qcol[q][i] =
            (uint16_t)(std::find(cols.begin(), cols.end(), jobs[q]->gids[i]) - cols.begin());
    }
    for (int c = 0; c < BS_COLS; c++) h.cutc[c] = COST_INF;
    cudaStream_t st = eng->stream;
    BsCtx* d_b = (BsCtx*)(base + o_b);
    int32_t* d_cols = (int32_t*)(base + o_cols);
    if (!eng->bs_ev[0]) {
      CK(cudaEventCreate(&eng->bs_ev[0]));
      CK(cudaEventCreate(&eng->bs_ev[1]));
    }
    CK(cudaEventRecord(eng->bs_ev[0], st));
    // the seeds' table (table 1 of a hop-bounded search); the copies fill the others
    CK(cudaMemsetAsync(D ? h.tab[1] : h.dist, 0xFF, (size_t)V * Gp * 4, st));
    CK(cudaMemsetAsync(h.fm[0], 0, (size_t)V * Wm * 4, st));
    CK(cudaMemsetAsync(h.fm[1], 0, (size_t)V * Wm * 4, st));
    CK(cudaMemcpyAsync(d_b, &h, sizeof(BsCtx), cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(d_cols, cols.data(), ncols * 4, cudaMemcpyHostToDevice, st));
    cs.h2d += sizeof(BsCtx) + ncols * 4;
    const DevGraph G = dev_graph(g);
    k_bs_seed<<<dim3(16, ncols), 256, 0, st>>>(d_b, G, grp->d_ptr, grp->d_mem, d_cols, (int)ncols);
    int64_t launches = 1, relax_launches = 0;
    const int64_t n4 = V * (int64_t)Gp / 4;
    int occ = 1;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_bs_relax, 256, 0);
    const int relax_blocks = eng->sms * std::max(1, std::min(occ, 4));
    BsCtx hb;
    for (;;) {
      for (int i = 0; i < 6; i++) {
        if (D) {
          k_bs_copy<<<eng->sms * 4, 256, 0, st>>>(d_b, n4, 0);
          launches++;
        }
        k_bs_scan<<<eng->sms * 4, 256, 0, st>>>(d_b, G);
        k_bs_star<<<eng->sms * 4, 256, 0, st>>>(d_b);
        k_bs_ctrl<<<1, 256, 0, st>>>(d_b, 0);
        const int pe = prof_begin(PROF_BSRELAX);
        k_bs_relax<<<relax_blocks, 256, 0, st>>>(d_b, G);
        prof_end(pe);
        relax_launches++;
        k_bs_ctrl<<<1, 256, 0, st>>>(d_b, 1);
        launches += 5;
      }
      CK(cudaGetLastError());
      CK(cudaMemcpyAsync(&hb, d_b, sizeof(BsCtx), cudaMemcpyDeviceToHost, st));
      cs.d2h += sizeof(BsCtx);
      CK(cudaStreamSynchronize(st));
      if (hb.done) break;
    }
    if (D && hb.round + 1u < (uint32_t)D) {
      k_bs_copy<<<eng->sms * 4, 256, 0, st>>>(d_b, n4, 1);
      launches++;
      CK(cudaGetLastError());
    }
    CK(cudaEventRecord(eng->bs_ev[1], st));
    CK(cudaEventSynchronize(eng->bs_ev[1]));
    float ms = 0;
    cudaEventElapsedTime(&ms, eng->bs_ev[0], eng->bs_ev[1]);
    cs.bs_ms += ms;
    cs.bs_sectors += (int64_t)hb.st_relax;
    cs.bs_launches += launches;
    cs.bs_relax += relax_launches;
    cs.launches += launches;
    Shared& S = shs.back();
    if (hb.error) {  // the queries search on their own
      S.remaining = 0;
      shared_release(false);
      return GST_OK;
    }
    S.d_b = d_b;
    S.Gp = Gp;
    S.dist = h.dist;
    for (int t = 0; t <= KMAX; t++) S.tab[t] = h.tab[t];
    // a query's cutoff: the smallest final cutoff of its columns
    for (size_t q = 0; q < jobs.size(); q++) {
      uint32_t cut = COST_INF;
      for (int i = 0; i < jobs[q]->q.k; i++) cut = std::min(cut, hb.cutc[hb.qcol[q][i]]);
      for (int i = 0; i < KMAX; i++) jobs[q]->ss_cols[i] = i < jobs[q]->q.k ? hb.qcol[q][i] : 0;
      jobs[q]->ss_cut = cut;
      jobs[q]->ss = 1;
    }
    S.remaining = (int)jobs.size();
    return GST_OK;
  }

  // Contexts of free slots below nctx must look idle to the kernels.
  gst_status write_idle() {
    for (int s = 0; s < nctx; s++)
      if (!owner[s] && !idle_written[s]) {
        Ctx& c = h_ctx[s];
        memset(&c, 0, sizeof(c));
        c.phase = PH_DONE;
        c.idle = 1;
        c.best = ~0ull;
        CK(cudaMemcpyAsync(d_ctx + s, &c, sizeof(Ctx), cudaMemcpyHostToDevice, eng->stream));
        cs.h2d += sizeof(Ctx);
        idle_written[s] = 1;
      }
    return GST_OK;
  }

  int prof_begin(int kind) {
    if (!((eng->cfg.profile_kernels >> kind) & 1)) return -1;
    const size_t i = cs.next_ev++;
    while (eng->prof_events.size() < 2 * (i + 1)) {
      cudaEvent_t e;
      if (cudaEventCreate(&e) != cudaSuccess) return -1;
      eng->prof_events.push_back(e);
    }
    cudaEventRecord(eng->prof_events[2 * i], eng->stream);
    cs.prof.push_back({kind, (int)i});
    return (int)i;
  }
  void prof_end(int i) {
    if (i >= 0) cudaEventRecord(eng->prof_events[2 * i + 1], eng->stream);
  }

  // One level of every resident query: sssp, ctrl, rows, ctrl, grow, ctrl.
  void launch_level(cudaStream_t st, int rwm, bool sssp, bool prof) {
    const DevGraph G = dev_graph(g);
    const int split = eng->cfg.split_degree;
    const int tpb = eng->cfg.threads_per_block;
    if (sssp) {
      const int pe = prof ? prof_begin(PROF_SSSP) : -1;
      k_sssp<<<eng->sssp_blocks, 256, 0, st>>>(d_ctx, nctx, G, split);
      prof_end(pe);
      k_ctrl<<<nctx, 128, 0, st>>>(d_ctx, nctx, CTRL_SSSP);
    }
    const size_t per_warp = rows_smem_per_warp(rwm);
    // k_rows: at most 256 threads, as many warps as the widest row lets fit
    const int warps = rows_warps(eng->rows_smem, tpb, rwm);
    int pe = prof ? prof_begin(PROF_ROWS) : -1;
    k_rows<<<rows_blocks(eng, warps * 32, per_warp * warps), warps * 32, per_warp * warps, st>>>(
        d_ctx, nctx, G, split, rwm);
    prof_end(pe);
    k_ctrl<<<nctx, 128, 0, st>>>(d_ctx, nctx, CTRL_DP_ROWS);
    pe = prof ? prof_begin(PROF_GROW) : -1;
    k_grow<<<eng->grow_blocks, 256, 0, st>>>(d_ctx, nctx, G, split);
    prof_end(pe);
    k_ctrl<<<nctx, 128, 0, st>>>(d_ctx, nctx, CTRL_DP_GROW);
  }

  // The level loop as a CUDA graph: a WHILE node whose body is one level plus a
  // kernel that decides whether to go on (no query finished, iterations left).
  gst_status loop_graph(int rwm, cudaGraphExec_t* out) {
    for (auto& lg : graphs)
      if (lg.nctx == nctx && lg.rw_max == rwm) {
        *out = lg.exec;
        return GST_OK;
      }
    LoopGraph lg;
    lg.nctx = nctx;
    lg.rw_max = rwm;
    CK(cudaGraphCreate(&lg.graph, 0));
    cudaGraphConditionalHandle handle;
    CK(cudaGraphConditionalHandleCreate(&handle, lg.graph, 1, cudaGraphCondAssignDefault));
    cudaGraphNodeParams cp = {};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = handle;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    cudaGraphNode_t node;
    CK(cudaGraphAddNode(&node, lg.graph, nullptr, 0, &cp));
    cudaGraph_t body = cp.conditional.phGraph_out[0];
    {
      // occupancy queries before the capture
      const int warps = rows_warps(eng->rows_smem, eng->cfg.threads_per_block, rwm);
      rows_blocks(eng, warps * 32, rows_smem_per_warp(rwm) * warps);
    }
    cudaStream_t cap;
    CK(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking));
    CK(cudaStreamBeginCaptureToGraph(cap, body, nullptr, nullptr, 0,
                                     cudaStreamCaptureModeThreadLocal));
    launch_level(cap, rwm, true, false);
    k_loop_cond<<<1, 64, 0, cap>>>(d_ctx, nctx, d_loop, handle);
    cudaGraph_t captured = nullptr;
    cudaError_t ce = cudaStreamEndCapture(cap, &captured);
    cudaStreamDestroy(cap);
    if (ce != cudaSuccess) {
      cudaGraphDestroy(lg.graph);
      return fail(eng, GST_DEVICE_ERROR, std::string("graph capture: ") + cudaGetErrorString(ce));
    }
    CK(cudaGraphInstantiate(&lg.exec, lg.graph, 0));
    graphs.push_back(lg);
    *out = lg.exec;
    return GST_OK;
  }

  // Run levels until at least one resident query has finished (or, with
  // max_levels > 0, at most about that many levels), then read the contexts.
  gst_status run(int max_levels) {
    {
      gst_status s = write_idle();
      if (s != GST_OK) return s;
    }
    const int rwm = rw_max();
    bool any_sssp = true;
    const bool prof = eng->cfg.profile_kernels != 0;
    const bool graphs_on = eng->cfg.use_graphs && !prof;
    for (;;) {
      int levels = 0;
      if (graphs_on) {
        cudaGraphExec_t ex;
        gst_status s = loop_graph(rwm, &ex);
        if (s != GST_OK) return s;
        const uint32_t iters = max_levels > 0 ? (uint32_t)max_levels : 4096u;
        loop_init[0] = iters;
        loop_init[1] = 0u;
        CK(cudaMemcpyAsync(d_loop, loop_init, 2 * sizeof(uint32_t), cudaMemcpyHostToDevice,
                           eng->stream));
        CK(cudaGraphLaunch(ex, eng->stream));
        CK(cudaMemcpyAsync(loop_left, d_loop, sizeof(uint32_t), cudaMemcpyDeviceToHost,
                           eng->stream));
        levels = (int)iters;
      } else {
        const int ahead = 6;
        for (int i = 0; i < ahead; i++) launch_level(eng->stream, rwm, any_sssp, prof);
        cs.launches += (int64_t)ahead * (any_sssp ? 6 : 4);
        levels = ahead;
      }
      CK(cudaGetLastError());
      CK(cudaMemcpyAsync(h_ctx, d_ctx, sizeof(Ctx) * nctx, cudaMemcpyDeviceToHost, eng->stream));
      cs.d2h += (int64_t)sizeof(Ctx) * nctx;
      CK(cudaStreamSynchronize(eng->stream));
      if (graphs_on) {
        // levels the device loop ran: each is 7 kernels (sssp, rows, grow, 3 ctrl, loop test)
        const int64_t ran = (int64_t)levels - (int64_t)loop_left[0];
        cs.launches += 7 * ran;
        cs.graph_launches++;
        cs.graph_levels += ran;
        levels = (int)ran;
      }
      bool any_done = false;
      any_sssp = false;
      for (int s = 0; s < nctx; s++) {
        if (!owner[s]) continue;
        any_sssp |= h_ctx[s].phase == PH_SSSP || h_ctx[s].phase == PH_PREP;
        any_done |= h_ctx[s].phase >= PH_DONE;
        if (eng->cfg.verbose > 1)
          fprintf(stderr, "[gst run] slot %d k %d phase %u levels %u err %x ub %u n_rows %u in_n %u\n",
                  s, h_ctx[s].k, h_ctx[s].phase, h_ctx[s].levels, h_ctx[s].error, h_ctx[s].ub,
                  h_ctx[s].n_rows, h_ctx[s].in_n);
      }
      if (any_done || active == 0) return GST_OK;
      if (max_levels > 0 && levels >= max_levels) return GST_OK;
    }
  }

  // Extract the trees of finished queries, fill their results and free their
  // slots; finished jobs are appended to `done` (capacity overflows are returned
  // in `retry` with a larger worklist boost instead, unless already at the worst case).
  gst_status harvest(std::vector<Job*>& done, std::vector<Job*>& retry) {
    bool any = false;
    for (int s = 0; s < nctx; s++) any |= owner[s] && h_ctx[s].phase >= PH_DONE;
    if (!any) return GST_OK;
    const DevGraph G = dev_graph(g);
    k_extract<<<1, MAXB, 0, eng->stream>>>(d_ctx, nctx, G);
    cs.launches += 1;
    CK(cudaMemcpyAsync(h_ctx, d_ctx, sizeof(Ctx) * nctx, cudaMemcpyDeviceToHost, eng->stream));
    cs.d2h += (int64_t)sizeof(Ctx) * nctx;
    CK(cudaStreamSynchronize(eng->stream));
    std::vector<int32_t> raw;
    for (int s = 0; s < nctx; s++) {
      Job* j = owner[s];
      if (!j || h_ctx[s].phase < PH_DONE) continue;
      const Ctx c = h_ctx[s];
      owner[s] = nullptr;
      active--;
      // pool rows this query may have written: cleared before the slot's next query
      mem[s].table_dirty = std::max(mem[s].table_dirty,
                                    (size_t)(c.rowmap ? std::min(c.pool_n, c.pool_cap) : c.pool_cap) *
                                        (size_t)c.RW * 8);
      const bool list_full = (c.error & (ERR_QCAP | ERR_FARCAP)) &&
                             !cap_is_worst(g->V, g->E, j->rw, eng->cfg.split_degree, c.qcap);
      const bool pool_full = (c.error & ERR_POOL) && c.rowmap != nullptr;
      if (list_full || pool_full) {
        j->boost++;
        j->ss = 0;  // a retry searches on its own
        retry.push_back(j);
        continue;
      }
      if (j->cache_dst) {
        // a group-cache fill: column 0 of the distance rows is the group's vector; a hop
        // fill stores its budgets 1..nhb first, then the full bound
        if (!c.error && c.phase == PH_DONE) {
          const size_t V = (size_t)g->V;
          CK(cudaMemcpy2DAsync(j->cache_dst + (size_t)c.nhb * V, sizeof(uint32_t), mem[s].dist,
                               (size_t)c.ds * sizeof(uint32_t), sizeof(uint32_t), V,
                               cudaMemcpyDeviceToDevice, eng->stream));
          for (int h = 1; h <= c.nhb; h++)
            CK(cudaMemcpy2DAsync(j->cache_dst + (size_t)(h - 1) * V, sizeof(uint32_t),
                                 mem[s].dist_h + (size_t)(h - 1) * V * c.ds,
                                 (size_t)c.ds * sizeof(uint32_t), sizeof(uint32_t), V,
                                 cudaMemcpyDeviceToDevice, eng->stream));
        }
        memset(j->out, 0, sizeof(gst_result));
        j->out->status = c.error ? status_of(c) : GST_OK;
        j->done = true;
        done.push_back(j);
        continue;
      }
      const uint32_t nout = std::min(c.n_out, mem[s].outcap);
      raw.resize((size_t)nout * 3);
      if (nout) {
        CK(cudaMemcpyAsync(raw.data(), mem[s].out, (size_t)nout * 12, cudaMemcpyDeviceToHost,
                           eng->stream));
        cs.d2h += (int64_t)nout * 12;
        CK(cudaStreamSynchronize(eng->stream));
      }
      fill(c, j, raw, nout);
      if (c.error || c.phase != PH_DONE) {
        char msg[160];
        snprintf(msg, sizeof msg, "query tag %llu: phase %u error bits 0x%x bounds site %u levels %u",
                 (unsigned long long)j->q.user_tag, c.phase, c.error, c.bad_site, c.levels);
        fail(eng, (gst_status)j->out->status, msg);
      }
      j->done = true;
      done.push_back(j);
    }
    // idle contexts for the slots just freed
    return write_idle();
  }

  // Result of job j from its context and its raw tree edges (device numbering), in the
  // caller's vertex ids.
  void fill(const Ctx& c, Job* j, const std::vector<int32_t>& raw, uint32_t nout) const {
    const std::vector<int32_t>& host_id = g->to_host;
    gst_result* r = j->out;
    memset(r, 0, sizeof(*r));
    r->user_tag = j->q.user_tag;
    r->status = status_of(c);
    if (c.error & ERR_EXTRACT) r->status = GST_DEVICE_ERROR;
    r->stats.levels = c.levels;
    r->stats.states_expanded = (int64_t)c.st_items;
    r->stats.edge_relaxations = (int64_t)c.st_relax;
    r->stats.merge_pairs = (int64_t)c.st_merge;
    r->stats.rows_merged = (int64_t)c.st_rows;
    r->stats.sssp_relaxations = (int64_t)c.st_sssp;
    r->stats.queue_max = c.st_qmax;
    r->stats.latency_ms =
        std::chrono::duration<double, std::milli>(Clock::now() - j->t_submit).count();
    if (r->status != GST_OK) return;
    r->cost = (int32_t)(c.best >> 32);
    r->root = host_id[(size_t)(c.best & 0x7FFFFFFull)];
    r->root_hop = (int32_t)((c.best >> 27) & 31u);
    // distinct edges, (min, max) orientation
    std::vector<std::pair<std::pair<int32_t, int32_t>, int32_t>> es;
    es.reserve(nout);
    for (size_t i = 0; i < nout; i++) {
      int32_t a = host_id[(size_t)raw[3 * i]], b = host_id[(size_t)raw[3 * i + 1]];
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

  // Summed profiled kernel time of this call per ProfKind, in ms, and launches.
  void kernel_ms(double out[PROF_KINDS], int64_t n[PROF_KINDS]) {
    for (int i = 0; i < PROF_KINDS; i++) {
      out[i] = 0;
      n[i] = 0;
    }
    for (auto& pr : cs.prof) {
      float e = 0;
      if (cudaEventElapsedTime(&e, eng->prof_events[2 * pr.second],
                               eng->prof_events[2 * pr.second + 1]) == cudaSuccess) {
        out[pr.first] += e;
        n[pr.first]++;
      }
    }
  }
};

// Fill job j from query q (copying the group ids) with result destination r.
void make_job(Job& j, const gst_query* q, gst_result* r) {
  j.q = *q;
  for (int i = 0; i < q->k && i < KMAX; i++) j.gids[i] = q->group_ids[i];
  j.q.group_ids = j.gids;
  j.out = r;
  j.t_submit = Clock::now();
  j.rw = row_width(q->k, q->hop_bound);
  j.nhb = hop_budgets(q->hop_bound);
  j.ds = dist_stride(q->k);
}

}  // namespace

// ---- serving -------------------------------------------------------------------
struct gst_server {
  gst_graph* g = nullptr;
  gst_groups* grp = nullptr;
  std::unique_ptr<Runner> run;
  std::thread th;
  std::mutex mu;                       // guards everything below
  std::condition_variable cv_work;     // submissions / stop
  std::condition_variable cv_done;     // completions
  std::deque<Job*> pending;
  std::map<uint64_t, std::unique_ptr<Job>> jobs;        // ticket -> job (owns the result)
  std::map<uint64_t, std::unique_ptr<gst_result>> res;  // ticket -> result storage
  uint64_t next_ticket = 1;
  bool stop = false;
  gst_status fatal = GST_OK;
  std::string fatal_msg;
  int64_t admitted = 0, completed = 0;
};

namespace {
gst_status maybe_shared_search(Runner& R, std::deque<Job*>& pending);  // with the batch driver
}  // namespace

namespace {

void server_loop(gst_server* sv) {
  gst_engine* eng = sv->g->eng;
  Runner& R = *sv->run;
  std::vector<Job*> done, retry;
  for (;;) {
    // admit what fits, in arrival order (a query that must wait blocks the ones
    // behind it, so that a large query is not starved by small ones)
    {
      std::unique_lock<std::mutex> lk(sv->mu);
      if (R.active == 0)
        sv->cv_work.wait(lk, [&] { return sv->stop || !sv->pending.empty(); });
      if (eng->cfg.verbose)
        fprintf(stderr, "[gst server] top: stop %d active %d pending %zu\n", (int)sv->stop,
                R.active, sv->pending.size());
      if (sv->stop && sv->pending.empty() && R.active == 0) return;
    }
    done.clear();
    retry.clear();
    {
      std::lock_guard<std::mutex> elk(eng->mu);
      cudaSetDevice(eng->device);
      // the waiting arrivals' distances: one shared search per kind, as in a batch call
      gst_status s_pre = GST_OK;
      if (eng->cfg.batch_search) {
        std::deque<Job*> snap;
        {
          std::lock_guard<std::mutex> lk(sv->mu);
          snap = sv->pending;
        }
        s_pre = maybe_shared_search(R, snap);
      }
      for (;;) {
        if (s_pre != GST_OK) break;
        Job* j = nullptr;
        {
          std::lock_guard<std::mutex> lk(sv->mu);
          if (sv->pending.empty()) break;
          j = sv->pending.front();
        }
        gst_status s = R.admit(j);
        if (s == GST_NOT_READY) break;
        std::lock_guard<std::mutex> lk(sv->mu);
        sv->pending.pop_front();
        if (s == GST_OK) {
          sv->admitted++;
          continue;
        }
        memset(j->out, 0, sizeof(gst_result));
        j->out->status = s;
        j->out->user_tag = j->q.user_tag;
        j->done = true;
        sv->completed++;
        sv->cv_done.notify_all();
      }
      bool waiting;
      {
        std::lock_guard<std::mutex> lk(sv->mu);
        waiting = !sv->pending.empty();
      }
      gst_status s = s_pre;
      if (s == GST_OK && R.active == 0 && waiting && !R.shs.empty()) {
        // nothing runs and the shared tables hold memory the next arrival needs: give
        // them back; the waiting queries search on their own
        std::lock_guard<std::mutex> lk(sv->mu);
        for (Job* j : sv->pending)
          if (j->ss == 1) j->ss = 2;
        R.shared_release(true);
      }
      if (eng->cfg.verbose) {
        std::lock_guard<std::mutex> lk(sv->mu);
        fprintf(stderr, "[gst server] active %d pending %zu held %zu budget %zu\n", R.active,
                sv->pending.size(), R.held, R.budget);
      }
      if (s == GST_OK && R.active > 0) {
        // with arrivals waiting for a slot, come back at the next finished query;
        // with free slots and arrivals possible, check every few levels
        const bool free_slot = R.active < R.max_slots;
        s = R.run(waiting || !free_slot ? 0 : 8);
        if (s == GST_OK) s = R.harvest(done, retry);
      }
      std::lock_guard<std::mutex> lk(sv->mu);
      if (s != GST_OK) {
        sv->fatal = s;
        sv->fatal_msg = eng->err;
        for (int i = 0; i < R.max_slots; i++)
          if (R.owner[i]) {
            R.owner[i]->out->status = s;
            R.owner[i]->done = true;
            R.owner[i] = nullptr;
          }
        for (Job* j : sv->pending) {
          j->out->status = s;
          j->done = true;
        }
        sv->pending.clear();
        R.active = 0;
        sv->cv_done.notify_all();
        return;
      }
      for (Job* j : retry) sv->pending.push_front(j);
      sv->completed += (int64_t)done.size();
      if (!done.empty()) sv->cv_done.notify_all();
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
  cfg->blocks_per_sm = 8;
  cfg->max_batch = 16;
  cfg->use_graphs = 1;
  cfg->verbose = 0;
  cfg->hop_cut_mult = 1;
  cfg->search_cut_permille = 1000;
  cfg->batch_search = 1;
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
    if (eng->cfg.use_graphs < 0) eng->cfg.use_graphs = 0;
    if (eng->cfg.hop_cut_mult <= 0) eng->cfg.hop_cut_mult = 1;
    if (eng->cfg.search_cut_permille <= 0) eng->cfg.search_cut_permille = 1000;
  }
  // the rows kernel is compiled for at most 256 threads per CTA (4 CTAs per SM)
  eng->cfg.threads_per_block = std::max(64, std::min(256, eng->cfg.threads_per_block / 32 * 32));
  eng->cfg.max_batch = std::min(eng->cfg.max_batch, MAXB);
  if (cudaSetDevice(device) != cudaSuccess) {
    delete eng;
    return fail(nullptr, GST_DEVICE_ERROR, "engine: cudaSetDevice failed");
  }
  cudaDeviceProp prop;
  cudaGetDeviceProperties(&prop, device);
  eng->sms = prop.multiProcessorCount;
  apply_launch_config(eng);
  // a pool of our own, keeping freed slot memory for the next query
  cudaMemPoolProps pp = {};
  pp.allocType = cudaMemAllocationTypePinned;
  pp.location.type = cudaMemLocationTypeDevice;
  pp.location.id = device;
  if (cudaStreamCreateWithFlags(&eng->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaMemPoolCreate(&eng->pool, &pp) != cudaSuccess) {
    if (eng->stream) cudaStreamDestroy(eng->stream);
    delete eng;
    return fail(nullptr, GST_DEVICE_ERROR, "engine: stream / memory pool creation failed");
  }
  uint64_t keep = ~0ull;
  cudaMemPoolSetAttribute(eng->pool, cudaMemPoolAttrReleaseThreshold, &keep);
  eng->rows_smem = rows_smem_limit(device);
  if (cudaFuncSetAttribute(k_rows, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)eng->rows_smem) != cudaSuccess) {
    cudaStreamDestroy(eng->stream);
    cudaMemPoolDestroy(eng->pool);
    delete eng;
    return fail(nullptr, GST_DEVICE_ERROR, "engine: cannot size the rows kernel's shared memory");
  }
  *out = eng;
  return GST_OK;
}

gst_status gst_engine_destroy(gst_engine* eng) {
  if (!eng) return GST_OK;
  if (eng->graphs.load() > 0)
    return fail(eng, GST_BAD_INPUT, "engine: destroy its graphs first (gst_graph_destroy)");
  cudaSetDevice(eng->device);
  if (eng->stream) {
    cudaStreamSynchronize(eng->stream);
    cudaStreamDestroy(eng->stream);
  }
  for (auto e : eng->prof_events) cudaEventDestroy(e);
  for (auto e : eng->bs_ev)
    if (e) cudaEventDestroy(e);
  if (eng->pool) cudaMemPoolDestroy(eng->pool);
  delete eng;
  return GST_OK;
}

gst_status gst_engine_set_profiling(gst_engine* eng, int32_t bits) {
  if (!eng || bits < 0 || bits > 15) return fail(eng, GST_BAD_INPUT, "profiling: bits must be in [0, 15]");
  std::lock_guard<std::mutex> lk(eng->mu);
  eng->cfg.profile_kernels = bits;
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
  for (int64_t i = 0; i < E; i++)
    if (adj[i] < 0 || adj[i] >= V) return fail(eng, GST_BAD_INPUT, "graph: neighbour id out of range");
  // device numbering: by degree, highest first, ties by id
  std::vector<int32_t> to_host((size_t)V), to_dev((size_t)V);
  for (int64_t v = 0; v < V; v++) to_host[v] = (int32_t)v;
  std::stable_sort(to_host.begin(), to_host.end(), [&](int32_t a, int32_t b) {
    return beg[a + 1] - beg[a] > beg[b + 1] - beg[b];
  });
  for (int64_t n = 0; n < V; n++) to_dev[to_host[n]] = (int32_t)n;
  std::vector<int64_t> nbeg((size_t)V + 1, 0);
  for (int64_t n = 0; n < V; n++) nbeg[n + 1] = nbeg[n] + (beg[to_host[n] + 1] - beg[to_host[n]]);
  std::vector<int32_t> nadj((size_t)E), nwt((size_t)E);
#pragma omp parallel for schedule(dynamic, 4096)
  for (int64_t n = 0; n < V; n++) {
    const int64_t o = to_host[n];
    for (int64_t i = beg[o], j = nbeg[n]; i < beg[o + 1]; i++, j++) {
      nadj[j] = to_dev[adj[i]];
      nwt[j] = wt[i];
    }
  }
  beg = nbeg.data();
  adj = nadj.data();
  wt = nwt.data();
  // Two device copies of the adjacency: sorted by neighbour (edge-weight lookups
  // of the tree walk) and sorted by weight, with per vertex the number of edges of
  // weight <= widx_threshold(t) (t < WIDX), so that a grow step reads only the edges light enough
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
        while (j < tmp.size() && (uint32_t)tmp[j].first <= widx_threshold(t)) j++;
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
  g->to_dev.swap(to_dev);
  g->to_host.swap(to_host);
  for (int64_t v = 0; v < V; v++) g->max_deg = std::max(g->max_deg, beg[v + 1] - beg[v]);
  for (int64_t i = 0; i < E; i++) g->max_w = std::max(g->max_w, wt[i]);
  CK(cudaMalloc(&g->d_beg, sizeof(int64_t) * (V + 1)));
  CK(cudaMalloc(&g->d_edges, sizeof(int2) * std::max<int64_t>(E, 1)));
  CK(cudaMalloc(&g->d_wedges, sizeof(int2) * std::max<int64_t>(E, 1)));
  CK(cudaMalloc(&g->d_widx, sizeof(uint32_t) * V * WIDX));
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
  eng->graphs++;
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
  g->batch.reset();
  cudaFree(g->d_beg);
  cudaFree(g->d_edges);
  cudaFree(g->d_wedges);
  cudaFree(g->d_widx);
  cudaMemPoolTrimTo(eng->pool, 0);
  delete g;
  eng->graphs--;
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
  std::vector<int32_t> dm((size_t)M);  // members in the graph's device numbering
  for (int64_t j = 0; j < M; j++) dm[j] = g->to_dev[members[j]];
  CK(cudaMalloc(&gr->d_ptr, sizeof(int64_t) * (n_groups + 1)));
  CK(cudaMalloc(&gr->d_mem, sizeof(int32_t) * std::max<int64_t>(M, 1)));
  CK(cudaMemcpyAsync(gr->d_ptr, grp_ptr, sizeof(int64_t) * (n_groups + 1),
                     cudaMemcpyHostToDevice, eng->stream));
  if (M)
    CK(cudaMemcpyAsync(gr->d_mem, dm.data(), sizeof(int32_t) * M, cudaMemcpyHostToDevice,
                       eng->stream));
  CK(cudaStreamSynchronize(eng->stream));
  *out = gr;
  return GST_OK;
}

gst_status gst_groups_destroy(gst_groups* gr) {
  if (!gr) return GST_OK;
  gst_engine* eng = gr->g->eng;
  std::lock_guard<std::mutex> lk(eng->mu);
  cudaSetDevice(eng->device);
  cudaStreamSynchronize(eng->stream);
  cudaFree(gr->d_ptr);
  cudaFree(gr->d_mem);
  if (gr->cache.d_vec) cudaFree(gr->cache.d_vec);
  if (gr->hop_cache.d_vec) cudaFree(gr->hop_cache.d_vec);
  delete gr;
  return GST_OK;
}

}  // extern "C"

namespace {
// Run the pending jobs on R with at most B resident (admitting beyond the batch size
// would change it), refilling slots as queries finish; capacity overflows are re-run
// with more room.  A job that does not fit the free memory yet does not hold back the
// smaller ones behind it (a batch has no arrival order to keep).
// A query the batch-shared search may serve: unbounded or of hop bound 1..KMAX, a first
// attempt, not a cache fill, not every group in the group cache of its kind (those start
// from exact distances; with only some cached, the shared table serves all of them).
// Returns its kind (0 unbounded, else D), -1 if none.
int shared_kind(const Runner& R, const Job* j) {
  if (j->cache_dst || j->boost > 0 || j->ss) return -1;
  const int D = j->q.hop_bound;
  if (D == 0 || D > KMAX) return -1;
  const auto& hc = R.grp->hop_cache;
  int cached = 0;
  for (int i = 0; i < j->q.k; i++) {
    if (D < 0) cached += R.grp->cache.vec(j->gids[i]) != nullptr;
    if (D > 0) cached += hc.cap > 0 && hc.D == D && hc.vec(j->gids[i]) != nullptr;
  }
  if (cached == j->q.k) return -1;
  return D < 0 ? 0 : D;
}

// One shared search over the first waiting queries of one kind (0 unbounded, else D).
gst_status shared_search_kind(Runner& R, std::deque<Job*>& pending, int kind) {
  std::vector<Job*> chunk;
  std::vector<int32_t> cols;
  for (Job* j : pending) {
    if (shared_kind(R, j) != kind) continue;
    int add = 0;
    for (int i = 0; i < j->q.k; i++)
      add += std::find(cols.begin(), cols.end(), j->gids[i]) == cols.end();
    if ((int)cols.size() + add > BS_COLS || (int)chunk.size() >= BS_MAXQ) break;
    for (int i = 0; i < j->q.k; i++)
      if (std::find(cols.begin(), cols.end(), j->gids[i]) == cols.end()) cols.push_back(j->gids[i]);
    chunk.push_back(j);
  }
  if (chunk.empty()) return GST_OK;
  return R.shared_search(chunk, cols, kind);
}

// Before admitting: for every kind (unbounded, or one hop bound D) with no shared table
// pending and an eligible query waiting, search the groups of that kind's first
// queries together (in order, up to BS_COLS distinct groups and BS_MAXQ queries).  A
// lone query takes the same path: its search over k columns on these kernels is faster
// than the per-query group-mask search on large graphs.  Kinds are searched in the
// order their first queries wait.
gst_status maybe_shared_search(Runner& R, std::deque<Job*>& pending) {
  if (!R.eng->cfg.batch_search) return GST_OK;
  R.shared_release(false);
  std::vector<int> kinds;
  for (Job* j : pending) {
    const int jk = shared_kind(R, j);
    if (jk >= 0 && !R.shared_of(jk) && std::find(kinds.begin(), kinds.end(), jk) == kinds.end())
      kinds.push_back(jk);
  }
  for (int kind : kinds) {
    gst_status s = shared_search_kind(R, pending, kind);
    if (s != GST_OK) return s;
  }
  return GST_OK;
}

gst_status drive(Runner& R, std::deque<Job*>& pending, int B) {
  gst_engine* eng = R.eng;
  const int saved = R.max_slots;
  R.max_slots = B;
  gst_status st = GST_OK;
  std::vector<Job*> done, retry;
  while (st == GST_OK && (!pending.empty() || R.active > 0)) {
    st = maybe_shared_search(R, pending);
    if (st != GST_OK) break;
    for (auto it = pending.begin(); it != pending.end() && R.active < R.max_slots;) {
      gst_status s = R.admit(*it);
      if (s == GST_NOT_READY) {
        ++it;
        continue;
      }
      if (s == GST_OOM_ADMISSION) {
        Job* j = *it;
        if (j->ss == 1) {  // never gathers its columns
          Runner::Shared* S = R.shared_of(j->q.hop_bound < 0 ? 0 : j->q.hop_bound);
          if (S) S->remaining--;
        }
        j->out->status = GST_OOM_ADMISSION;
        j->out->user_tag = j->q.user_tag;
        fail(eng, GST_OOM_ADMISSION, "solve: the query's state table does not fit the memory budget");
      } else if (s != GST_OK) {
        st = s;
        break;
      }
      it = pending.erase(it);
    }
    if (st == GST_OK && R.active == 0 && !pending.empty() && !R.shs.empty()) {
      // nothing runs and the shared tables hold memory a waiting query needs: give them
      // back; the waiting queries search on their own
      for (Job* j : pending)
        if (j->ss == 1) j->ss = 2;
      R.shared_release(true);
      continue;
    }
    if (st != GST_OK || R.active == 0) break;
    st = R.run(0);
    done.clear();
    retry.clear();
    if (st == GST_OK) st = R.harvest(done, retry);
    for (Job* j : retry) pending.push_front(j);
  }
  R.shared_release(true);
  R.max_slots = saved;
  return st;
}

// The graph's batch runner with at least B slots, created on first use.
gst_status batch_runner(gst_graph* g, int B) {
  if (!g->batch || g->batch->max_slots < B) {
    const int slots = std::max(B, g->batch ? g->batch->max_slots : 0);
    g->batch.reset(new Runner(g->eng, g, slots));
    gst_status s = g->batch->init();
    if (s != GST_OK) {
      g->batch.reset();
      return s;
    }
  }
  return GST_OK;
}
}  // namespace

extern "C" {

}  // extern "C"

namespace {
// Warm cache C of groups grp for hop bound D (-1: unlimited distances): see
// gst_groups_cache_warm / gst_groups_cache_warm_hop.  Caller holds the engine lock.
gst_status cache_warm(gst_groups* grp, gst_groups::Cache& C, int32_t D, int32_t n,
                      const int32_t* group_ids, int64_t max_bytes, int32_t* n_cached) {
  gst_graph* g = grp->g;
  gst_engine* eng = g->eng;
  const size_t stride = (size_t)g->V * (size_t)(D > 0 ? hop_budgets(D) + 1 : 1);
  const size_t eb = stride * sizeof(uint32_t);
  const int32_t cap = (int32_t)std::min<int64_t>(max_bytes / (int64_t)eb, grp->n);
  if (cap != C.cap || D != C.D) {
    CK(cudaStreamSynchronize(eng->stream));
    if (C.d_vec) cudaFree(C.d_vec);
    C = gst_groups::Cache();
    if (cap > 0) {
      CK(cudaMalloc(&C.d_vec, (size_t)cap * eb));
      C.cap = cap;
      C.D = D;
      C.stride = stride;
      C.slot_of.assign(grp->n, -1);
      C.gid_of.assign(cap, -1);
      C.used.assign(cap, 0);
    }
  }
  if (n_cached) *n_cached = 0;
  if (C.cap == 0) return GST_OK;
  C.clock++;
  // the listed groups, in list order; at most cap of them stay
  std::vector<int32_t> want;
  for (int32_t i = 0; i < n && (int32_t)want.size() < C.cap; i++)
    if (std::find(want.begin(), want.end(), group_ids[i]) == want.end()) want.push_back(group_ids[i]);
  for (int32_t gid : want)
    if (C.slot_of[gid] >= 0) C.used[C.slot_of[gid]] = C.clock;
  std::vector<int32_t> todo;
  for (int32_t gid : want)
    if (C.slot_of[gid] < 0) todo.push_back(gid);
  if (!todo.empty()) {
    // a slot for each missing group: empty ones first, then the least recently used
    // among groups this call does not list; one distance-only job per group
    std::unique_ptr<Job[]> jobs(new Job[todo.size()]);
    std::vector<gst_result> res(todo.size());
    std::deque<Job*> pending;
    for (size_t t = 0; t < todo.size(); t++) {
      int32_t best = -1;
      for (int32_t sl = 0; sl < C.cap; sl++)
        if (C.used[sl] != C.clock && (best < 0 || C.used[sl] < C.used[best])) best = sl;
      if (C.gid_of[best] >= 0) C.slot_of[C.gid_of[best]] = -1;
      C.gid_of[best] = todo[t];
      C.used[best] = C.clock;
      gst_query q{};
      q.k = 1;
      q.group_ids = &todo[t];
      q.hop_bound = D;
      make_job(jobs[t], &q, &res[t]);
      jobs[t].cache_dst = C.d_vec + (size_t)best * C.stride;
      pending.push_back(&jobs[t]);
    }
    const int B = std::max(1, std::min<int>(eng->cfg.max_batch, (int)todo.size()));
    gst_status st = batch_runner(g, B);
    if (st == GST_OK) {
      Runner& R = *g->batch;
      R.grp = grp;
      R.cs = CallStats();
      R.nctx = 0;
      st = drive(R, pending, B);
    }
    CK(cudaStreamSynchronize(eng->stream));
    bool ok = st == GST_OK;
    for (size_t t = 0; t < todo.size(); t++) ok = ok && jobs[t].done && res[t].status == GST_OK;
    if (!ok) {
      // forget the slots this call was filling (their groups were never visible)
      for (int32_t sl = 0; sl < C.cap; sl++)
        if (C.gid_of[sl] >= 0 && std::find(todo.begin(), todo.end(), C.gid_of[sl]) != todo.end()) {
          C.gid_of[sl] = -1;
          C.used[sl] = 0;
        }
      if (st != GST_OK) {
        // a device failure ends the call; the runner is rebuilt on the next call
        g->batch.reset();
        cudaGetLastError();
      } else {
        st = GST_DEVICE_ERROR;
      }
      return fail(eng, st, "cache: a group's distance search failed: " + eng->err);
    }
    for (int32_t sl = 0; sl < C.cap; sl++)
      if (C.gid_of[sl] >= 0) C.slot_of[C.gid_of[sl]] = sl;
  }
  if (n_cached)
    for (int32_t gid : want) *n_cached += C.slot_of[gid] >= 0;
  return GST_OK;
}
}  // namespace

extern "C" {

gst_status gst_groups_cache_warm(gst_groups* grp, int32_t n, const int32_t* group_ids,
                                 int64_t max_bytes, int32_t* n_cached) {
  gst_engine* eng = grp ? grp->g->eng : nullptr;
  if (!grp || n < 0 || (n > 0 && !group_ids) || max_bytes < 0)
    return fail(eng, GST_BAD_INPUT, "cache: bad arguments");
  for (int32_t i = 0; i < n; i++)
    if (group_ids[i] < 0 || group_ids[i] >= grp->n) return fail(eng, GST_BAD_INPUT, "cache: group id out of range");
  std::lock_guard<std::mutex> lk(eng->mu);
  CK(cudaSetDevice(eng->device));
  return cache_warm(grp, grp->cache, -1, n, group_ids, max_bytes, n_cached);
}

gst_status gst_groups_cache_warm_hop(gst_groups* grp, int32_t n, const int32_t* group_ids,
                                     int32_t hop_bound, int64_t max_bytes, int32_t* n_cached) {
  gst_engine* eng = grp ? grp->g->eng : nullptr;
  if (!grp || n < 0 || (n > 0 && !group_ids) || max_bytes < 0 || hop_bound < 1 || hop_bound > 30)
    return fail(eng, GST_BAD_INPUT, "cache: bad arguments (hop bound must be in [1, 30])");
  for (int32_t i = 0; i < n; i++)
    if (group_ids[i] < 0 || group_ids[i] >= grp->n) return fail(eng, GST_BAD_INPUT, "cache: group id out of range");
  std::lock_guard<std::mutex> lk(eng->mu);
  CK(cudaSetDevice(eng->device));
  return cache_warm(grp, grp->hop_cache, hop_bound, n, group_ids, max_bytes, n_cached);
}

gst_status gst_solve_batch(gst_graph* g, gst_groups* grp, int32_t n, const gst_query* queries,
                           gst_result* results) {
  gst_engine* eng = g ? g->eng : nullptr;
  if (!g || !grp || grp->g != g || n < 0 || (n > 0 && (!queries || !results)))
    return fail(eng, GST_BAD_INPUT, "solve: bad arguments");
  for (int32_t i = 0; i < n; i++) memset(&results[i], 0, sizeof(gst_result));
  std::lock_guard<std::mutex> lk(eng->mu);
  CK(cudaSetDevice(eng->device));
  const int B = std::max(1, std::min<int>(eng->cfg.max_batch, std::max<int32_t>(n, 1)));
  {
    gst_status s = batch_runner(g, B);
    if (s != GST_OK) return s;
  }
  Runner& R = *g->batch;
  R.grp = grp;
  R.cs = CallStats();
  R.nctx = 0;  // no query is resident between calls
  std::unique_ptr<Job[]> jobs(new Job[(size_t)std::max<int32_t>(n, 1)]);
  std::deque<Job*> pending;
  for (int32_t i = 0; i < n; i++) {
    gst_status s = validate_query(eng, grp, &queries[i]);
    if (s != GST_OK) {
      results[i].status = s;
      results[i].user_tag = queries[i].user_tag;
      continue;
    }
    make_job(jobs[i], &queries[i], &results[i]);
    pending.push_back(&jobs[i]);
  }
  cudaEvent_t ev0, ev1;
  CK(cudaEventCreate(&ev0));
  CK(cudaEventCreate(&ev1));
  CK(cudaEventRecord(ev0, eng->stream));
  gst_status st = drive(R, pending, B);
  CK(cudaEventRecord(ev1, eng->stream));
  CK(cudaEventSynchronize(ev1));
  float ms = 0;
  cudaEventElapsedTime(&ms, ev0, ev1);
  cudaEventDestroy(ev0);
  cudaEventDestroy(ev1);
  if (st != GST_OK) {
    // a device failure ends the call; the runner is rebuilt on the next call
    std::string msg = eng->err;
    g->batch.reset();
    cudaGetLastError();
    for (int32_t i = 0; i < n; i++)
      if (!jobs[i].done && results[i].status == GST_OK) results[i].status = st;
    return fail(eng, st, msg);
  }
  if (eng->cfg.verbose)
    fprintf(stderr, "[gst batch] %d queries: %.3f ms, %lld launches, %lld graph launches, %lld graph levels, "
            "%lld slot allocations (%.1f GB, %.1f ms host)\n",
            n, ms, (long long)R.cs.launches, (long long)R.cs.graph_launches,
            (long long)R.cs.graph_levels, (long long)R.cs.allocs, R.cs.alloc_bytes / 1e9, R.cs.alloc_ms);
  double kms[PROF_KINDS];
  int64_t kn[PROF_KINDS];
  R.kernel_ms(kms, kn);
  for (int32_t i = 0; i < n; i++) {
    gst_stats& s = results[i].stats;
    s.device_ms = ms;
    s.kernel_launches = R.cs.launches;
    s.h2d_bytes = R.cs.h2d;
    s.d2h_bytes = R.cs.d2h;
    s.grow_ms = kms[PROF_GROW];
    s.rows_ms = kms[PROF_ROWS];
    s.sssp_ms = kms[PROF_SSSP];
    s.grow_launches = kn[PROF_GROW];
    s.rows_launches = kn[PROF_ROWS];
    s.sssp_launches = kn[PROF_SSSP];
    s.shared_relax_ms = kms[PROF_BSRELAX];
    s.shared_sectors = R.cs.bs_sectors;
    s.shared_ms = R.cs.bs_ms;
    s.shared_launches = R.cs.bs_launches;
    s.shared_relax_launches = R.cs.bs_relax;
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
  int32_t saved;
  {
    std::lock_guard<std::mutex> lk(eng->mu);
    saved = eng->cfg.max_batch;
    eng->cfg.max_batch = 1;
  }
  s = gst_solve_batch(g, grp, 1, q, res);
  {
    std::lock_guard<std::mutex> lk(eng->mu);
    eng->cfg.max_batch = saved;
  }
  if (s != GST_OK) return s;
  return (gst_status)res->status;
}

gst_status gst_debug_slot_state(gst_graph* g, int32_t slot, uint64_t* cells, int64_t n_cells,
                                uint64_t* best_out) {
  gst_engine* eng = g ? g->eng : nullptr;
  if (!g || !g->batch || slot < 0 || slot >= g->batch->max_slots || n_cells < 0 ||
      !g->batch->mem[slot].base)
    return fail(eng, GST_BAD_INPUT, "debug: bad slot");
  std::lock_guard<std::mutex> lk(eng->mu);
  CK(cudaSetDevice(eng->device));
  Runner& R = *g->batch;
  const SlotMem& m = R.mem[slot];
  const int64_t have = (int64_t)(m.table_bytes / 8);
  if (cells && n_cells)
    CK(cudaMemcpyAsync(cells, m.table, (size_t)std::min(n_cells, have) * 8,
                       cudaMemcpyDeviceToHost, eng->stream));
  CK(cudaMemcpyAsync(R.h_ctx + slot, R.d_ctx + slot, sizeof(Ctx), cudaMemcpyDeviceToHost,
                     eng->stream));
  CK(cudaStreamSynchronize(eng->stream));
  if (best_out) *best_out = R.h_ctx[slot].best;
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

// ---- autotuner ----------------------------------------------------------------------
// Launch parameters are chosen per graph shape by coordinate descent on a sample of
// queries: for each parameter in turn every candidate value is timed (device time
// of gst_solve_batch on the sample, best of two) with the others held, and the
// fastest is kept.  Every candidate must return the same costs; the result is
// cached as one line per shape in a text file, so later runs on a graph of the same
// shape skip the search.

}  // extern "C"

namespace {

std::string shape_key(const gst_graph* g, int32_t max_batch) {
  char b[160];
  snprintf(b, sizeof b, "V=%lld E=%lld dmax=%lld wmax=%d batch=%d sms=%d", (long long)g->V,
           (long long)g->E, (long long)g->max_deg, g->max_w, max_batch, g->eng->sms);
  return b;
}

struct TuneParams {
  int32_t split_degree, bucket_delta, threads_per_block, blocks_per_sm, max_batch, search_cut,
      batch_search;
};

void set_params(gst_graph* g, const TuneParams& p) {
  gst_engine* eng = g->eng;
  eng->cfg.split_degree = p.split_degree;
  eng->cfg.bucket_delta = p.bucket_delta;
  eng->cfg.threads_per_block = std::max(64, std::min(256, p.threads_per_block / 32 * 32));
  eng->cfg.blocks_per_sm = p.blocks_per_sm;
  eng->cfg.max_batch = std::max(1, std::min(MAXB, p.max_batch));
  eng->cfg.search_cut_permille = std::max(1, p.search_cut);
  eng->cfg.batch_search = p.batch_search ? 1 : 0;
  apply_launch_config(eng);
  g->batch.reset();  // its CUDA graphs hold the old launch geometry
}

bool read_cache(const char* path, const std::string& key, TuneParams* p) {
  if (!path) return false;
  FILE* f = fopen(path, "r");
  if (!f) return false;
  char line[512];
  bool hit = false;
  while (fgets(line, sizeof line, f)) {
    char* bar = strchr(line, '|');
    if (!bar) continue;
    *bar = 0;
    if (key != line) continue;
    TuneParams t;
    if (sscanf(bar + 1, "%d %d %d %d %d %d %d", &t.split_degree, &t.bucket_delta,
               &t.threads_per_block, &t.blocks_per_sm, &t.max_batch, &t.search_cut,
               &t.batch_search) == 7) {
      *p = t;
      hit = true;  // the last line for a key wins
    }
  }
  fclose(f);
  return hit;
}

}  // namespace

extern "C" {

extern "C" gst_status gst_autotune(gst_graph* g, gst_groups* grp, int32_t n,
                                   const gst_query* sample, const char* cache_path,
                                   gst_config* chosen) {
  gst_engine* eng = g ? g->eng : nullptr;
  if (!g || !grp || grp->g != g || n < 1 || !sample)
    return fail(eng, GST_BAD_INPUT, "autotune: bad arguments");
  const std::string key = shape_key(g, eng->cfg.max_batch);
  TuneParams cur{eng->cfg.split_degree, eng->cfg.bucket_delta, eng->cfg.threads_per_block,
                 eng->cfg.blocks_per_sm, eng->cfg.max_batch, eng->cfg.search_cut_permille,
                 eng->cfg.batch_search};
  TuneParams hit;
  if (read_cache(cache_path, key, &hit)) {
    std::lock_guard<std::mutex> lk(eng->mu);
    set_params(g, hit);
    if (chosen) *chosen = eng->cfg;
    return GST_OK;
  }
  const int32_t saved_prof = eng->cfg.profile_kernels;
  eng->cfg.profile_kernels = 0;
  std::vector<gst_result> res((size_t)n);
  std::vector<int32_t> ref_cost((size_t)n), ref_status((size_t)n);
  bool have_ref = false;
  // device time of the sample under parameters p (best of two runs), or < 0 on failure
  auto measure = [&](const TuneParams& p, double* ms) -> gst_status {
    {
      std::lock_guard<std::mutex> lk(eng->mu);
      set_params(g, p);
    }
    double best = -1;
    for (int rep = 0; rep < 2; rep++) {
      gst_status st = gst_solve_batch(g, grp, n, sample, res.data());
      if (st != GST_OK) return st;
      const double t = res[0].stats.device_ms;
      for (int32_t i = 0; i < n; i++) {
        if (!have_ref) {
          ref_cost[i] = res[i].cost;
          ref_status[i] = res[i].status;
        } else if (res[i].status != ref_status[i] ||
                   (res[i].status == GST_OK && res[i].cost != ref_cost[i])) {
          for (auto& r : res) gst_result_free(&r);
          return fail(eng, GST_DEVICE_ERROR, "autotune: a candidate changed an optimum");
        }
        gst_result_free(&res[i]);
      }
      have_ref = true;
      if (best < 0 || t < best) best = t;
    }
    *ms = best;
    return GST_OK;
  };
  double best_ms = 0;
  gst_status st = measure(cur, &best_ms);
  const std::vector<int32_t> c_split = {64, 128, 256, 512, 1024};
  const std::vector<int32_t> c_delta = {0, 2, 6, 16};
  const std::vector<int32_t> c_tpb = {128, 256};
  const std::vector<int32_t> c_bps = {2, 4, 8};
  std::vector<int32_t> c_batch;  // resident queries: at most the configured batch
  for (int32_t b : {1, 2, 4, 8, 16, 32, 64})
    if (b < cur.max_batch) c_batch.push_back(b);
  const std::vector<int32_t> c_cut = {1000, 875, 750};  // search cutoff, permille of ub
  const std::vector<int32_t> c_bsearch = {1, 0};  // batch-shared distance search
  for (int param = 0; param < 7 && st == GST_OK; param++) {
    const std::vector<int32_t>& cand = param == 0   ? c_bsearch
                                       : param == 1 ? c_cut
                                       : param == 2 ? c_split
                                       : param == 3 ? c_delta
                                       : param == 4 ? c_tpb
                                       : param == 5 ? c_bps
                                                    : c_batch;
    for (int32_t v : cand) {
      TuneParams p = cur;
      int32_t* field = param == 0   ? &p.batch_search
                       : param == 1 ? &p.search_cut
                       : param == 2 ? &p.split_degree
                       : param == 3 ? &p.bucket_delta
                       : param == 4 ? &p.threads_per_block
                       : param == 5 ? &p.blocks_per_sm
                                    : &p.max_batch;
      if (*field == v) continue;
      *field = v;
      double ms = 0;
      st = measure(p, &ms);
      if (st != GST_OK) break;
      if (ms < best_ms) {
        best_ms = ms;
        cur = p;
      }
    }
  }
  {
    std::lock_guard<std::mutex> lk(eng->mu);
    set_params(g, cur);
    eng->cfg.profile_kernels = saved_prof;
  }
  if (st != GST_OK) return st;
  if (cache_path) {
    FILE* f = fopen(cache_path, "a");
    if (f) {
      fprintf(f, "%s|%d %d %d %d %d %d %d\n", key.c_str(), cur.split_degree, cur.bucket_delta,
              cur.threads_per_block, cur.blocks_per_sm, cur.max_batch, cur.search_cut,
              cur.batch_search);
      fclose(f);
    }
  }
  if (chosen) *chosen = eng->cfg;
  return GST_OK;
}

// ---- serving ---------------------------------------------------------------------

gst_status gst_server_create(gst_graph* g, gst_groups* grp, gst_server** out) {
  gst_engine* eng = g ? g->eng : nullptr;
  if (!g || !grp || grp->g != g || !out) return fail(eng, GST_BAD_INPUT, "server: bad arguments");
  *out = nullptr;
  gst_server* sv = new gst_server();
  sv->g = g;
  sv->grp = grp;
  {
    std::lock_guard<std::mutex> lk(eng->mu);
    CK(cudaSetDevice(eng->device));
    // the graph's batch runner holds no query between calls: hand its slot memory to
    // the server (the next gst_solve* call makes a new one from what is free then)
    g->batch.reset();
    sv->run.reset(new Runner(eng, g, std::max(1, eng->cfg.max_batch)));
    sv->run->grp = grp;
    gst_status s = sv->run->init();
    if (s != GST_OK) {
      delete sv;
      return s;
    }
  }
  sv->th = std::thread(server_loop, sv);
  *out = sv;
  return GST_OK;
}

gst_status gst_submit(gst_server* sv, const gst_query* q, uint64_t* ticket) {
  if (!sv || !q || !ticket) return fail(nullptr, GST_BAD_INPUT, "submit: bad arguments");
  gst_engine* eng = sv->g->eng;
  std::unique_ptr<Job> j(new Job());
  std::unique_ptr<gst_result> r(new gst_result());
  memset(r.get(), 0, sizeof(gst_result));
  gst_status s = validate_query(eng, sv->grp, q);
  std::lock_guard<std::mutex> lk(sv->mu);
  if (sv->fatal != GST_OK) return fail(eng, sv->fatal, "submit: server stopped: " + sv->fatal_msg);
  if (sv->stop) return fail(eng, GST_BAD_INPUT, "submit: server is shutting down");
  const uint64_t t = sv->next_ticket++;
  if (s == GST_OK) make_job(*j, q, r.get());
  j->ticket = t;
  j->out = r.get();
  if (s != GST_OK) {
    r->status = s;
    r->user_tag = q->user_tag;
    j->done = true;
  }
  Job* raw = j.get();
  sv->jobs[t] = std::move(j);
  sv->res[t] = std::move(r);
  if (s == GST_OK) {
    sv->pending.push_back(raw);
    sv->cv_work.notify_one();
  }
  *ticket = t;
  return GST_OK;
}

static gst_status take_result(gst_server* sv, uint64_t ticket, gst_result* res) {
  auto it = sv->jobs.find(ticket);
  *res = *sv->res[ticket];  // ownership of the edge arrays moves to the caller
  sv->jobs.erase(it);
  sv->res.erase(ticket);
  return (gst_status)res->status;
}

gst_status gst_poll(gst_server* sv, uint64_t ticket, gst_result* res) {
  if (!sv || !res) return fail(nullptr, GST_BAD_INPUT, "poll: bad arguments");
  std::lock_guard<std::mutex> lk(sv->mu);
  auto it = sv->jobs.find(ticket);
  if (it == sv->jobs.end()) return fail(sv->g->eng, GST_BAD_INPUT, "poll: unknown ticket");
  if (!it->second->done) return GST_NOT_READY;
  return take_result(sv, ticket, res);
}

gst_status gst_wait(gst_server* sv, uint64_t ticket, gst_result* res) {
  if (!sv || !res) return fail(nullptr, GST_BAD_INPUT, "wait: bad arguments");
  std::unique_lock<std::mutex> lk(sv->mu);
  auto it = sv->jobs.find(ticket);
  if (it == sv->jobs.end()) return fail(sv->g->eng, GST_BAD_INPUT, "wait: unknown ticket");
  Job* j = it->second.get();
  sv->cv_done.wait(lk, [&] { return j->done.load(); });
  return take_result(sv, ticket, res);
}

gst_status gst_server_destroy(gst_server* sv) {
  if (!sv) return GST_OK;
  {
    std::lock_guard<std::mutex> lk(sv->mu);
    sv->stop = true;
    sv->cv_work.notify_all();
  }
  if (sv->th.joinable()) sv->th.join();
  {
    gst_engine* eng = sv->g->eng;
    std::lock_guard<std::mutex> lk(eng->mu);
    sv->run.reset();
  }
  for (auto& kv : sv->res) gst_result_free(kv.second.get());
  delete sv;
  return GST_OK;
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
constexpr uint32_t kNoallocOutCap = 1u << 14;    // tree edges the extraction may write
constexpr uint32_t kNoallocStackCap = 1u << 16;  // its parent-walk stack

// Per-device set-up, done once with the device current: the scratch array's device
// address, the rows kernel's shared-memory limit and two timing events.
struct NoallocDev {
  bool ready = false;
  void* scratch = nullptr;
  size_t rows_smem = 0;
  int sms = 0, grow_blocks = 0, sssp_blocks = 0;
  cudaEvent_t ev[2] = {nullptr, nullptr};
};
std::mutex g_noalloc_mu;
NoallocDev g_noalloc_dev[kMaxDevices];
// Host staging of the raw extracted edges (u, v, w), sorted and deduplicated here before
// they are copied into the caller's arrays; shared by all calls (under g_noalloc_mu).
int32_t g_noalloc_edges[3 * kNoallocOutCap];

// Device address of the scratch array (and the rest of the set-up) on `device`, which
// must be current.  Host code cannot use the symbol itself: on the host it names a
// stand-in object, not device memory.
gst_status noalloc_setup(int device, NoallocDev** out, std::string* err) {
  NoallocDev& d = g_noalloc_dev[device];
  if (!d.ready) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) {
      *err = std::string("noalloc: cudaGetSymbolAddress: ") + cudaGetErrorString(e);
      return GST_DEVICE_ERROR;
    }
    d.scratch = p;
    d.rows_smem = rows_smem_limit(device);
    e = cudaFuncSetAttribute(k_rows, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)d.rows_smem);
    int occ_grow = 1, occ_sssp = 1;
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&d.sms, cudaDevAttrMultiProcessorCount, device);
    if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_grow, k_grow, 256, 0);
    if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_sssp, k_sssp, 256, 0);
    if (e == cudaSuccess) e = cudaEventCreate(&d.ev[0]);
    if (e == cudaSuccess) e = cudaEventCreate(&d.ev[1]);
    if (e != cudaSuccess) {
      *err = std::string("noalloc: device set-up: ") + cudaGetErrorString(e);
      return GST_DEVICE_ERROR;
    }
    gst_config cfg;
    gst_config_default(&cfg);
    d.grow_blocks = d.sms * std::max(1, std::min(occ_grow, cfg.blocks_per_sm));
    d.sssp_blocks = d.sms * std::max(1, std::min(occ_sssp, cfg.blocks_per_sm));
    d.ready = true;
  }
  *out = &d;
  return GST_OK;
}

gst_status noalloc_solve(int device, cudaStream_t st, int64_t V, int64_t E, const int64_t* d_beg,
                         const int32_t* d_edges, int32_t n_groups, const int64_t* d_grp_ptr,
                         const int32_t* d_members, const gst_query* q, int64_t edge_cap,
                         gst_result* res) {
  if (!res) {
    tl_err = "noalloc: null result";
    return GST_BAD_INPUT;
  }
  int32_t* eu = res->edge_u;
  int32_t* ev = res->edge_v;
  int32_t* ew = res->edge_w;
  memset(res, 0, sizeof(*res));
  res->edge_u = eu;
  res->edge_v = ev;
  res->edge_w = ew;
  // every failure leaves its status in res->status as well as in the return value
  auto failed = [&](gst_status s, const std::string& msg) {
    res->status = s;
    tl_err = msg;
    return s;
  };
  if (!q || !d_beg || !d_grp_ptr || !d_members || (E > 0 && !d_edges) || V < 1 ||
      V >= ((int64_t)1 << 27) || E < 0 || n_groups < 1 || edge_cap < 0 ||
      (edge_cap > 0 && (!eu || !ev || !ew)))
    return failed(GST_BAD_INPUT, "noalloc: bad arguments");
  res->user_tag = q->user_tag;
  if (q->k < 1 || q->k > KMAX || !q->group_ids || q->hop_bound > 30)
    return failed(GST_BAD_INPUT, "noalloc: k must be in [1,8], hop bound <= 30");
  for (int i = 0; i < q->k; i++) {
    const int32_t a = q->group_ids[i];
    if (a < 0 || a >= n_groups) return failed(GST_BAD_INPUT, "noalloc: group id out of range");
    for (int j = 0; j < i; j++)
      if (q->group_ids[j] == a) return failed(GST_BAD_INPUT, "noalloc: duplicate group id");
  }
  // scratch layout (the same buffers as a runner slot); reject what does not fit
  gst_config cfg;
  gst_config_default(&cfg);
  Ctx c;
  memset(&c, 0, sizeof(c));
  init_query_ctx(c, q, cfg);
  const size_t RW = (size_t)c.RW;
  const int nhb = c.sssp_hops ? hop_budgets(q->hop_bound) : 0;
  const size_t Vs = (size_t)V;
  size_t off = align256(sizeof(Ctx));
  auto take = [&](size_t n) {
    const size_t o = off;
    off = align256(off + n);
    return o;
  };
  const size_t o_table = take(Vs * RW * 8);
  const size_t ds = dist_stride(q->k);
  const size_t o_dist = take(Vs * ds * 4);
  const size_t o_bits = take((Vs + 31) / 32 * 4);
  const size_t o_rows = take(Vs * 4);
  const size_t o_out = take((size_t)kNoallocOutCap * 12);
  const size_t o_stack = take((size_t)kNoallocStackCap * 8);
  const size_t o_tour = take(kTourWords * 4);
  const size_t o_fm0 = take(fm_bytes(V));
  const size_t o_fm1 = take(fm_bytes(V));
  const size_t o_snap = take(c.sssp_mask == 2u ? Vs * ds * 4 : 0);
  const size_t o_dh = take((size_t)nhb * Vs * ds * 4);
  // four worklists (near and far, ping-pong) of at least 4V + 4096 items each
  const size_t min_lists = 4 * (4 * Vs + 4096) * 16;
  if (off + min_lists > kNoallocScratchBytes) {
    char msg[200];
    snprintf(msg, sizeof msg,
             "noalloc: this query needs more than the %zu-byte static scratch "
             "(V=%lld, row width %zu); use gst_solve",
             kNoallocScratchBytes, (long long)V, RW);
    return failed(GST_OOM_ADMISSION, msg);
  }
  const uint64_t want = (uint64_t)V * RW + 4ull * (uint64_t)V + 4096;
  const uint64_t fit = (kNoallocScratchBytes - off) / (4 * 16);
  const uint32_t cap = (uint32_t)std::min<uint64_t>(std::min<uint64_t>(want, fit), 1ull << 26);

  // the caller's device stays current for the caller: switch, and switch back on every exit
  int prev_dev = 0;
  if (cudaGetDevice(&prev_dev) != cudaSuccess) return failed(GST_DEVICE_ERROR, "noalloc: cudaGetDevice failed");
  if (cudaSetDevice(device) != cudaSuccess) return failed(GST_DEVICE_ERROR, "noalloc: cudaSetDevice failed");
  struct RestoreDevice {
    int dev;
    ~RestoreDevice() { cudaSetDevice(dev); }
  } restore{prev_dev};
#define NCK(call)                                                                         \
  do {                                                                                    \
    cudaError_t _e = (call);                                                              \
    if (_e != cudaSuccess)                                                                \
      return failed(GST_DEVICE_ERROR, std::string(#call) + ": " + cudaGetErrorString(_e)); \
  } while (0)

  // one call at a time per process: the scratch, the set-up and the host staging are shared
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  NoallocDev* nd = nullptr;
  {
    std::string err;
    gst_status s = noalloc_setup(device, &nd, &err);
    if (s != GST_OK) return failed(s, err);
  }
  const int warps = rows_warps(nd->rows_smem, cfg.threads_per_block, (int)RW);
  if (warps < 1) return failed(GST_BAD_INPUT, "noalloc: the query's state row does not fit the rows kernel's shared memory");
  unsigned char* base = (unsigned char*)nd->scratch;
  // empty-group check: members of each queried group
  for (int i = 0; i < q->k; i++) {
    int64_t be[2];
    NCK(cudaMemcpyAsync(be, d_grp_ptr + q->group_ids[i], sizeof(be), cudaMemcpyDeviceToHost, st));
    NCK(cudaStreamSynchronize(st));
    if (be[1] <= be[0]) return failed(GST_BAD_INPUT, "noalloc: group has no members");
  }
  const int split = cfg.split_degree;
  c.table = (uint64_t*)(base + o_table);
  c.dist = (uint32_t*)(base + o_dist);
  c.ds = (uint32_t)ds;
  c.rowbits = (uint32_t*)(base + o_bits);
  c.tour = (uint32_t*)(base + o_tour);
  c.fm[0] = (uint32_t*)(base + o_fm0);
  c.fm[1] = (uint32_t*)(base + o_fm1);
  c.snap = (uint32_t*)(base + o_snap);
  c.dist_h = (uint32_t*)(base + o_dh);
  c.nhb = nhb;
  c.q[0] = (uint4*)(base + off);
  c.q[1] = (uint4*)(base + off + (size_t)cap * 16);
  c.far[0] = (uint4*)(base + off + 2 * (size_t)cap * 16);
  c.far[1] = (uint4*)(base + off + 3 * (size_t)cap * 16);
  c.rows = (uint32_t*)(base + o_rows);
  c.out = (int32_t*)(base + o_out);
  c.stack = (uint64_t*)(base + o_stack);
  c.qcap = c.farcap = cap;
  c.rowcap = (uint32_t)V;
  c.outcap = kNoallocOutCap;
  c.stackcap = kNoallocStackCap;
  Ctx* d_ctx = (Ctx*)base;
  NCK(cudaEventRecord(nd->ev[0], st));
  // clear what must start empty (the array keeps the previous call's contents), then
  // upload the context
  NCK(cudaMemsetAsync(c.table, 0xFF, Vs * RW * 8, st));
  NCK(cudaMemsetAsync(c.dist, 0xFF, Vs * ds * 4, st));
  NCK(cudaMemsetAsync(c.rowbits, 0, (Vs + 31) / 32 * 4, st));
  NCK(cudaMemsetAsync(c.fm[0], 0, fm_bytes(V), st));
  NCK(cudaMemsetAsync(c.fm[1], 0, fm_bytes(V), st));
  if (nhb) NCK(cudaMemsetAsync(c.dist_h, 0xFF, (size_t)nhb * Vs * ds * 4, st));
  NCK(cudaMemcpyAsync(d_ctx, &c, sizeof(Ctx), cudaMemcpyHostToDevice, st));
  // the caller's edges are sorted by neighbour only: no light-edge index
  DevGraph G{V, E, d_beg, (const int2*)d_edges, (const int2*)d_edges, nullptr};
  k_init<<<dim3(64, 1), 256, 0, st>>>(d_ctx, 1, G, d_grp_ptr, d_members, split);
  k_ctrl<<<1, 32, 0, st>>>(d_ctx, 1, CTRL_SSSP);
  const size_t smem = rows_smem_per_warp((int)RW) * (size_t)warps;
  int64_t launches = 2;
  Ctx h;
  for (;;) {
    for (int i = 0; i < 6; i++) {
      k_sssp<<<nd->sssp_blocks, 256, 0, st>>>(d_ctx, 1, G, split);
      k_ctrl<<<1, 128, 0, st>>>(d_ctx, 1, CTRL_SSSP);
      k_rows<<<nd->sms * 4, warps * 32, smem, st>>>(d_ctx, 1, G, split, (int)RW);
      k_ctrl<<<1, 128, 0, st>>>(d_ctx, 1, CTRL_DP_ROWS);
      k_grow<<<nd->grow_blocks, 256, 0, st>>>(d_ctx, 1, G, split);
      k_ctrl<<<1, 128, 0, st>>>(d_ctx, 1, CTRL_DP_GROW);
      launches += 6;
    }
    NCK(cudaGetLastError());
    NCK(cudaMemcpyAsync(&h, d_ctx, sizeof(Ctx), cudaMemcpyDeviceToHost, st));
    NCK(cudaStreamSynchronize(st));
    if (h.phase >= PH_DONE) break;
  }
  k_extract<<<1, 32, 0, st>>>(d_ctx, 1, G);
  launches++;
  NCK(cudaGetLastError());
  NCK(cudaEventRecord(nd->ev[1], st));
  NCK(cudaMemcpyAsync(&h, d_ctx, sizeof(Ctx), cudaMemcpyDeviceToHost, st));
  const uint32_t nraw = std::min(h.n_out, kNoallocOutCap);
  if (status_of(h) == GST_OK && !(h.error & ERR_EXTRACT) && nraw > 0)
    NCK(cudaMemcpyAsync(g_noalloc_edges, c.out, (size_t)nraw * 12, cudaMemcpyDeviceToHost, st));
  NCK(cudaStreamSynchronize(st));
  float ms = 0;
  cudaEventElapsedTime(&ms, nd->ev[0], nd->ev[1]);
  gst_status status = status_of(h);
  if (h.error & ERR_EXTRACT) status = GST_DEVICE_ERROR;
  res->stats.levels = h.levels;
  res->stats.states_expanded = (int64_t)h.st_items;
  res->stats.edge_relaxations = (int64_t)h.st_relax;
  res->stats.merge_pairs = (int64_t)h.st_merge;
  res->stats.rows_merged = (int64_t)h.st_rows;
  res->stats.sssp_relaxations = (int64_t)h.st_sssp;
  res->stats.queue_max = h.st_qmax;
  res->stats.kernel_launches = launches;
  res->stats.device_ms = ms;
  res->stats.h2d_bytes = (int64_t)sizeof(Ctx);
  res->stats.d2h_bytes = 2 * (int64_t)sizeof(Ctx) + (int64_t)nraw * 12 + 16 * q->k;
  if (status != GST_OK) {
    if (status == GST_INFEASIBLE) {
      res->status = status;
      return status;
    }
    char msg[160];
    snprintf(msg, sizeof msg, "noalloc: phase %u error bits 0x%x levels %u", h.phase, h.error, h.levels);
    return failed(status, msg);
  }
  res->cost = (int32_t)(h.best >> 32);
  res->root = (int32_t)(h.best & 0x7FFFFFFull);
  res->root_hop = (int32_t)((h.best >> 27) & 31u);
  // orient each edge u < v, sort by (u, v) and drop repeats (the parent walk reaches
  // an edge once per state that uses it), then copy into the caller's arrays
  struct Tri {
    int32_t u, v, w;
  };
  Tri* t = (Tri*)g_noalloc_edges;
  for (uint32_t i = 0; i < nraw; i++)
    if (t[i].u > t[i].v) std::swap(t[i].u, t[i].v);
  std::sort(t, t + nraw, [](const Tri& a, const Tri& b) { return a.u != b.u ? a.u < b.u : a.v < b.v; });
  Tri* end = std::unique(t, t + nraw, [](const Tri& a, const Tri& b) { return a.u == b.u && a.v == b.v; });
  const int64_t m = end - t;
  if (m > edge_cap) {
    char msg[160];
    snprintf(msg, sizeof msg, "noalloc: the tree has %lld edges, more than edge_cap = %lld",
             (long long)m, (long long)edge_cap);
    return failed(GST_CAPACITY, msg);
  }
  for (int64_t i = 0; i < m; i++) {
    eu[i] = t[i].u;
    ev[i] = t[i].v;
    ew[i] = t[i].w;
  }
  res->n_edges = m;
  res->status = GST_OK;
  return GST_OK;
#undef NCK
}

}  // namespace

extern "C" gst_status gst_solve_noalloc(int32_t device, void* stream, int64_t V, int64_t E,
                                        const int64_t* d_beg_pos, const int32_t* d_edges,
                                        int32_t n_groups, const int64_t* d_grp_ptr,
                                        const int32_t* d_members, const gst_query* q,
                                        int64_t edge_cap, gst_result* res) {
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev ||
      device >= kMaxDevices) {
    tl_err = "noalloc: bad device";
    if (res) res->status = GST_BAD_INPUT;
    return GST_BAD_INPUT;
  }
  return noalloc_solve(device, (cudaStream_t)stream, V, E, d_beg_pos, d_edges, n_groups,
                       d_grp_ptr, d_members, q, edge_cap, res);
}
