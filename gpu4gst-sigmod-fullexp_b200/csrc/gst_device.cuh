// Device side of the GST engine: state layout, worklists and the level kernels.
//
// State table.  One query owns a slab of V rows; row v holds the 2^k x (D+1)
// states (v, p, d) of that vertex (d only for hop-bounded queries), cell d * 2^k + p,
// as packed 64-bit cells
//     cost(32) | pending(1) | parent(31)
// so that one 64-bit atomicMin relaxes cost and parent together (the reference
// writes its int32 cost with atomicMin and the parent separately,
// code/TrimCDP/src/DPQ.cu:136-140, which races).  `pending` marks a cell whose
// value changed since its row was last merged; a pending cell compares larger
// than a settled cell of equal cost, so equal-cost relaxations never reopen a
// settled state.  parent: bit30 = merge; grow -> source vertex (bits 0..29);
// merge -> partner subset Y (bits 0..15), partner hop d2 (16..20), own hop d1
// (21..25); LEAF = a group member's zero-cost singleton.
//
// One level of the DP (per query, all queries of a batch in the same launches):
//   rows kernel   every row dirtied by the previous grow is loaded into shared
//                 memory and closed under merges T(v,X|Y) <= T(v,X)+T(v,Y)
//                 (code/TrimCDP-WB/include/mapper.cuh:416-453; the reference
//                 merges per state with global atomics), then every changed
//                 state is settled, and growable ones are emitted as grow work
//                 items, hubs split into chunks of `split` edges (the virtual
//                 split of code/TrimCDP-WB/include/graph.hpp:128-378, done per
//                 work item instead of by rewriting the CSR).
//   grow kernel   work items are spread over warps by a warp-level load-balanced
//                 search over their edge counts; each edge (v,u,w) relaxes
//                 T(u,X[,d+1]) with one atomicMin; an improved target marks its
//                 row dirty (bitmap + compacted row list)
//                 (code/TrimCDP-WB/include/mapper.cuh:366-413).
//   control       one thread per query swaps worklists, advances the cost bucket
//                 (near/far ordering), counts levels and detects the fixpoint
//                 (replaces the grid barrier loop of mapper_enactor.cuh:158-246).
// Pruning (every test compares with ub, the cost of a feasible tree, so no state of
// an optimal tree is dropped):
//   grow a state only if 2c <= ub (code/TrimCDP-WB/include/mapper_enactor.cuh /
//   reducer.cuh:317-433 use c-1 <= best/2); keep a merged non-full state only if
//   3c <= 2ub (PrunedDP++ CPUNONHOP.h:913 uses 0.667*best+2); drop a state if
//   c + max_{i not in X} dist_i(v) > ub (one-label bound, get_lb mapper.cuh:163-191)
//   or c + ceil(tour/2) > ub (tour bound, PrunedDP++ CPUNONHOP.h:433-493).  A
//   hop-bounded state of height d takes its distances within the hop budget D - d
//   (its deepest vertex is d edges below v, so every missing group lies within
//   D - d edges of v in any tree of diameter <= D that contains it).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace gst {

constexpr uint64_t CELL_INF = ~0ull;
constexpr uint32_t COST_INF = 0xFFFFFFFFu;
constexpr uint32_t PEND = 0x80000000u;
constexpr uint32_t MERGE = 0x40000000u;
constexpr uint32_t LEAF = 0x3FFFFFFFu;
constexpr int MAXB = 64;          // queries per batched launch
constexpr int KMAX = 8;           // groups per query
constexpr int DIST_STRIDE = 8;    // int32 one-label distances per vertex row, at most

// Distance rows are as wide as the query needs: 1, 2, 4 or 8 uint32 (the smallest power
// of two >= k), so the rows of a query with few groups take less memory and cache (a
// k = 3 query's rows of a 4M-vertex graph are 64 MB, most of which the L2 holds).
__host__ __device__ __forceinline__ uint32_t dist_stride(int k) {
  return k <= 1 ? 1u : k <= 2 ? 2u : k <= 4 ? 4u : 8u;
}
// Row v of a distance table of stride ds as eight values (COST_INF past the row).
__device__ __forceinline__ void load_drow(const uint32_t* base, uint32_t ds, uint64_t v, uint4& a,
                                          uint4& b) {
  const uint32_t* p = base + v * ds;
  b = make_uint4(COST_INF, COST_INF, COST_INF, COST_INF);
  if (ds == 8u) {
    a = __ldcg((const uint4*)p);
    b = __ldcg((const uint4*)p + 1);
  } else if (ds == 4u) {
    a = __ldcg((const uint4*)p);
  } else if (ds == 2u) {
    const uint2 x = __ldcg((const uint2*)p);
    a = make_uint4(x.x, x.y, COST_INF, COST_INF);
  } else {
    a = make_uint4(__ldcg(p), COST_INF, COST_INF, COST_INF);
  }
}
__device__ __forceinline__ void store_drow(uint32_t* base, uint32_t ds, uint64_t v, const uint4& a,
                                           const uint4& b) {
  uint32_t* p = base + v * ds;
  if (ds == 8u) {
    ((uint4*)p)[0] = a;
    ((uint4*)p)[1] = b;
  } else if (ds == 4u) {
    *(uint4*)p = a;
  } else if (ds == 2u) {
    *(uint2*)p = make_uint2(a.x, a.y);
  } else {
    *p = a.x;
  }
}

// PH_PREP: distances final; the star bound, group distances and tour table are
// being built (one k_sssp pass over the distance rows, then the control block).
enum Phase : uint32_t { PH_SSSP = 0, PH_PREP = 1, PH_DP = 2, PH_DONE = 3, PH_ERROR = 4 };
enum ErrBits : uint32_t { ERR_QCAP = 1, ERR_FARCAP = 2, ERR_ROWCAP = 4, ERR_TIMEOUT = 8,
                          ERR_EXTRACT = 16, ERR_BOUNDS = 32, ERR_POOL = 64 };
constexpr uint32_t ROW_NONE = 0xFFFFFFFFu;
enum CtrlMode : int { CTRL_SSSP = 0, CTRL_DP_ROWS = 1, CTRL_DP_GROW = 2 };

// Light-edge index: per vertex, the number of edges of weight <= widx_threshold(t)
// for t < WIDX, thresholds 1, 2, 3, 4, 6, 8, 12, ..., 192, 256 (each step x1.5 or
// x1.33), so that one load bounds the edges a relaxation under a weight limit
// needs, over-counting by at most a third.
constexpr int WIDX = 16;
constexpr uint32_t CHUNK = 0x80000000u;  // item flag (in pd): one `split`-edge chunk only
constexpr int RELAX_U = 4;               // edges per lane per round of the grow relax loop
// Hop-limited distance items carry their path's edge count in bits 8..15 of the
// group word (group index in bits 0..7).
constexpr uint32_t SSSP_HOP_SHIFT = 8;
constexpr int TOUR_STRIDE = KMAX * KMAX;
constexpr int HOP_BUDGETS_MAX = 7;       // hop budgets of the one-label distances kept

struct DevGraph {
  int64_t V;
  int64_t E;
  const int64_t* beg;     // V+1
  const int2* edges;      // E x {neighbour, weight}, sorted by neighbour per vertex
  const int2* wedges;     // the same edges sorted by (weight, neighbour) per vertex
  const uint32_t* widx;   // V x WIDX: edges of v with weight <= 2^j (NULL: no index,
                          // wedges then need not be weight-sorted)
};

__host__ __device__ __forceinline__ uint32_t widx_threshold(int t) {
  return t == 0 ? 1u : ((t & 1) ? (2u << (t >> 1)) : (3u << ((t >> 1) - 1)));
}
// Smallest t with widx_threshold(t) >= W (W >= 1); WIDX when W > 256.
__device__ __forceinline__ int widx_slot(uint32_t W) {
  if (W <= 1u) return 0;
  const int b = 31 - __clz(W - 1u);  // 2^b < W <= 2^(b+1)
  if (b == 0) return 1;
  if (b >= 8) return WIDX;
  return W <= (3u << (b - 1)) ? 2 * b : 2 * b + 1;
}

// Edges of v (weight-sorted list, deg entries) worth relaxing under the weight limit
// W: every edge of weight <= W, plus possibly some heavier ones (the per-edge tests
// drop those).  Without an index the list is not weight-sorted and every edge counts.
__device__ __forceinline__ int64_t count_upto(const DevGraph& G, uint32_t v, int64_t deg,
                                              uint32_t W) {
  if (deg <= 0 || W == 0u) return 0;
  if (!G.widx) return deg;
  const int t = widx_slot(W);
  return t >= WIDX ? deg : (int64_t)__ldg(&G.widx[(uint64_t)v * WIDX + t]);
}

// Per-query context.  Fields above `in_ptr` are written by the host before the
// query starts; the rest are updated by the control kernel between launches and
// by atomics inside the level kernels.
struct Ctx {
  uint64_t* table;     // state rows: the dense slab (V rows), or the row pool (pool_cap rows)
  uint32_t* rowmap;    // row pool: vertex -> its pool row (ROW_NONE: none yet); nullptr: dense
  uint32_t pool_cap;   // rows of the pool
  uint32_t pool_n;     // pool rows handed out (may exceed pool_cap: ERR_POOL)
  uint32_t* dist;      // one-label distances: row v at dist + v * ds
  uint32_t ds;         // uint32 per distance row (dist, snap, dist_h): dist_stride(k)
  uint32_t* rowbits;
  uint32_t* fm[2];     // group-mask frontier (one byte per vertex, four to a word): the
                       // groups whose distance at the vertex improved in the step that
                       // wrote fm[no]; read and cleared by the next step through fm[in_idx]
  uint32_t* snap;      // hop-limited group-mask search: the distance rows of a round's
                       // frontier as they stood when the round began (V rows of ds)
  uint32_t* dist_h;    // hop budgets h = 1..nhb: d_i^{<=h}(v), cheapest paths of at most h
                       // edges (nhb x V rows of ds; budget D is dist itself)
  uint32_t* tour;      // 2^k x TOUR_STRIDE path table, then 2^k x KMAX row minima
  uint4* q[2];
  uint4* far[2];
  uint32_t* rows;
  int32_t* out;        // extraction: 3 ints per edge
  uint64_t* stack;     // extraction stack
  uint32_t qcap, farcap, rowcap, outcap, stackcap;
  int32_t k, W, full, D, DD, RW, hop, use_lb;
  int32_t use_tour;     // tour lower bound (needs use_lb)
  int32_t gid[KMAX];
  uint32_t vv[KMAX * KMAX];  // group-to-group distances (min over members of i of d_j)
  uint32_t delta;       // bucket width (0 = one bucket)
  uint32_t max_levels;
  // control state
  uint4* in_ptr;
  uint32_t in_n;
  uint32_t in_kind;     // 0 near list q[in_idx], 1 far list
  uint32_t in_idx;
  uint32_t no;          // near output list index
  uint32_t f;           // far list receiving pushes
  uint32_t n_q[2];
  uint32_t n_far[2];
  uint32_t n_rows;
  uint32_t far_min;
  uint32_t bucket_end;
  uint32_t ub;          // best feasible cost known (one-label solutions and full cells)
  uint32_t cut;         // cutoff when the one-label distances became final: a distance
                        // above it (or unreached) is only known to exceed it
  uint32_t cut_fix;     // nonzero: the distances came from a batch-shared search, exact up
                        // to this cutoff (it replaces the star-bound cutoff below)
  uint32_t cut_pm;      // the distance search stops at cut_pm / 1000 x ub: below 1000 it
                        // searches less and leaves weaker (still valid) bounds to the DP;
                        // hop-bounded queries, which prune against their own larger bound,
                        // may want more than 1000
  uint32_t sssp_hops;   // 0: distances d_i(v); D: hop-limited distances d_i^{<=D}(v), the
                        // cheapest paths of at most D edges (hop-bounded queries)
  int32_t nhb;          // hop budgets kept in dist_h
  uint32_t sssp_full;   // 1: distances exact everywhere (no cutoff): a distance-only job,
                        // or distances gathered from the group cache
  uint32_t dist_only;   // 1: a distance-only job (group cache fill): done at PREP
  uint32_t sssp_mask;   // distance search items: 0 one per (vertex, group); 1 one per
                        // (vertex, group mask), unlimited distances in one cost bucket;
                        // 2 the same for hop-limited distances, one round per two steps
  uint32_t ub_cell;     // best full-state cell
  uint32_t ub_hop;      // hop-bounded queries: best star of paths of at most D/2 edges
                        // found by the distance search (a tree of diameter <= D)
  unsigned long long best;  // cost<<32 | d<<27 | v of the best full-state cell
  uint32_t phase;
  uint32_t error;
  uint32_t levels;
  uint32_t n_out;
  uint32_t bad_site;    // checked builds: first failed bounds check (site id)
  unsigned long long st_items, st_relax, st_merge, st_rows, st_sssp;
  uint32_t st_qmax;     // largest worklist fill seen (near or far), for capacity sizing
  uint32_t idle;        // 1: no query in this slot (the kernels skip it)
};

// Bounds self-check of the checked build (-DGST_CHECKED): a failed check records
// ERR_BOUNDS and the site, and the caller skips the access.  Compiled out otherwise.
#ifdef GST_CHECKED
__device__ __forceinline__ bool in_bounds(Ctx* c, bool ok, uint32_t site) {
  if (!ok) {
    atomicOr(&c->error, (uint32_t)ERR_BOUNDS);
    atomicCAS(&c->bad_site, 0u, site);
  }
  return ok;
}
#else
#define in_bounds(c, ok, site) true
#endif

// ---- state rows ----------------------------------------------------------------------
// A query's states live in rows of RW cells, one row per vertex that holds any finite
// state.  Dense layout (rowmap == nullptr): row v at table + v * RW, all V rows.  Row
// pool: a vertex gets a row from a pool of pool_cap rows (pre-filled with unreached
// cells) the first time one of its states is written; rowmap[v] names it.  A query
// writes rows for a small share of the vertices (its pruned DP settles few states), so
// the pool holds its table in a fraction of the dense slab's memory, and clearing it
// for the next query touches only the rows the last one used.
__device__ __forceinline__ uint64_t* row_of(const Ctx* c, uint32_t v) {
  if (!c->rowmap) return c->table + (uint64_t)v * (uint64_t)c->RW;
  const uint32_t r = __ldcg(&c->rowmap[v]);
  return r == ROW_NONE ? nullptr : c->table + (uint64_t)r * (uint64_t)c->RW;
}
// Row of v given its rowmap entry r (as loaded by the caller), taking a pool row when v
// has none; nullptr when the pool is exhausted (ERR_POOL: the query is re-run with a
// larger pool).  Two lanes taking a row for the same vertex at once both draw a pool
// index; the one whose compare-and-swap loses uses the winner's row, and its own index
// stays unused.
__device__ __forceinline__ uint64_t* row_take(Ctx* c, uint32_t v, uint32_t r) {
  if (!c->rowmap) return c->table + (uint64_t)v * (uint64_t)c->RW;
  if (r == ROW_NONE) {
    const uint32_t mine = atomicAdd(&c->pool_n, 1u);
    if (mine >= c->pool_cap) {
      atomicOr(&c->error, (uint32_t)ERR_POOL);
      return nullptr;
    }
    const uint32_t old = atomicCAS(&c->rowmap[v], ROW_NONE, mine);
    r = old == ROW_NONE ? mine : old;
  }
  return c->table + (uint64_t)r * (uint64_t)c->RW;
}

// One-label distances of v within the hop budget h of a hop-bounded query: d_i^{<=h}(v),
// the cheapest paths of at most h edges.  A state of height d (a tree hanging from v
// whose deepest vertex is d edges below it) reaches every missing group within
// D - d edges in any tree of diameter <= D that contains it: the path from the deepest
// vertex to the group runs through v.  So d^{<=D-d} bounds its completion.  Budget 0
// is the groups' members (distance 0); budgets above the kept ones use d^{<=D}, a
// smaller and so still valid bound.
__device__ __forceinline__ void budget_row(const Ctx* c, int64_t V, uint32_t v, int h, uint4& a,
                                           uint4& b) {
  const uint32_t* base = c->dist;
  if (h >= 1 && h <= c->nhb) base = c->dist_h + (uint64_t)(h - 1) * (uint64_t)V * c->ds;
  load_drow(base, c->ds, v, a, b);
  if (h <= 0) {
    a = make_uint4(a.x ? COST_INF : 0u, a.y ? COST_INF : 0u, a.z ? COST_INF : 0u, a.w ? COST_INF : 0u);
    b = make_uint4(b.x ? COST_INF : 0u, b.y ? COST_INF : 0u, b.z ? COST_INF : 0u, b.w ? COST_INF : 0u);
  }
}

__device__ __forceinline__ uint32_t cost_of(uint64_t c) { return (uint32_t)(c >> 32); }
__device__ __forceinline__ uint64_t pack_cell(uint32_t cost, uint32_t low) {
  return ((uint64_t)cost << 32) | low;
}

// Submask table for masks of up to 8 bits: SUBMASK.v[M][b] is the b-th submask of M,
// the bits of b placed into the set bits of M, lowest first.  Built at compile time,
// so that the merge loop enumerates the submasks of a complement with one cached load.
struct SubmaskTable {
  unsigned char v[256][256];
};
constexpr SubmaskTable make_submask_table() {
  SubmaskTable t{};
  for (int M = 0; M < 256; M++)
    for (int b = 0; b < 256; b++) {
      int r = 0, bb = b, mm = M;
      while (mm) {
        const int low = mm & -mm;
        if (bb & 1) r |= low;
        bb >>= 1;
        mm ^= low;
      }
      t.v[M][b] = (unsigned char)r;
    }
  return t;
}
__device__ const SubmaskTable SUBMASK = make_submask_table();

// x / y for x < 2^22 and 1 <= y, from a float estimate and one correction each way
// (inv = 1.0f / y computed once by the caller).
__device__ __forceinline__ uint32_t udiv_small(uint32_t x, uint32_t y, float inv) {
  uint32_t q = (uint32_t)((float)x * inv);
  if (q * y > x) q--;
  if ((q + 1u) * y <= x) q++;
  return q;
}

// First lane whose inclusive scan value exceeds i (all lanes participate).
__device__ __forceinline__ int warp_owner(uint32_t scan, uint32_t i) {
  int lo = 0;
#pragma unroll
  for (int step = 16; step >= 1; step >>= 1) {
    const uint32_t s = __shfl_sync(0xffffffffu, scan, lo + step - 1);
    if (s <= i) lo += step;
  }
  return lo;
}

__device__ __forceinline__ uint32_t warp_incl_scan(uint32_t x) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  return x;
}

// ---- worklists -----------------------------------------------------------------
// A work item {v, pd, cost, off} asks for the edges of v's weight-sorted list from
// offset `off` on to be relaxed from state (v, pd) of cost `cost` (pd: group index
// in the distance phase, subset | hop << 16 in the DP).  Edges are relaxed in weight
// order and only as far as the current cost bucket [.., bucket_end) and the upper
// bound allow; an item whose next edge lands beyond the bucket waits in the far
// list under the key cost + weight(next edge), so heavy edges are read only once
// the frontier has reached their target cost, by which time ub has usually pruned
// them.  The near list holds items of the current bucket.
// Distance cutoff of the one-label search: cut_pm / 1000 x ub, saturating; for
// hop-limited distances ub is at least the best star of D/2-edge paths, a feasible cost
// of the query.  Both only decrease, so the cutoff never grows during the search.  Any
// cutoff is valid: a stored distance <= the final cutoff is exact (every prefix of its
// shortest path stayed below the cutoff) and any other is only known to exceed it, so
// every bound uses min(d, cut + 1).  A lower cutoff trades search work for DP work.
__device__ __forceinline__ uint32_t sssp_cutoff(const Ctx* c) {
  if (c->sssp_full) return COST_INF;
  if (c->cut_fix) return c->cut_fix;
  uint32_t ub = __ldcg(&c->ub);
  if (c->sssp_hops) {
    const uint32_t h = __ldcg(&c->ub_hop);
    ub = ub > h ? ub : h;
  }
  if (ub == COST_INF) return COST_INF;
  const uint64_t x = (uint64_t)ub * (c->cut_pm ? c->cut_pm : 1000u) / 1000u;
  return x >= COST_INF ? COST_INF : (uint32_t)x;
}

// Largest edge weight a grow step from a state of cost `cost` can still use: a
// target must stay <= ub (unbounded) or < ub_cell (hop-bounded).
__device__ __forceinline__ uint32_t grow_limit(const Ctx* c, uint32_t cost) {
  if (c->hop) {
    const uint32_t b = c->ub_cell;
    return b > cost ? b - cost - 1u : 0u;
  }
  const uint32_t b = c->ub;
  return b >= cost ? b - cost : 0u;
}

__device__ __forceinline__ void mark_row(Ctx* c, uint32_t u) {
  const uint32_t bit = 1u << (u & 31);
  const uint32_t old = atomicOr(&c->rowbits[u >> 5], bit);
  if (!(old & bit)) {
    const uint32_t i = atomicAdd(&c->n_rows, 1u);
    if (i < c->rowcap) c->rows[i] = u;
    else atomicOr(&c->error, (uint32_t)ERR_ROWCAP);
  }
}

// ---- warp-aggregated appends (all 32 lanes call; the loops are warp-uniform) ----
// One worklist counter per query is the hottest address of a level: lanes that
// append to the same list (same query, near or far) reserve their slots with one
// atomicAdd per warp, and far appends lower far_min once per warp.
// Lane with `want` appends item {v, pd, cost, off} to query qi's near list (far ==
// false) or far list (far == true, under `key`).
__device__ __forceinline__ void warp_append(Ctx* ctxs, int qi, bool want, bool far, uint32_t v,
                                            uint32_t pd, uint32_t cost, uint32_t off,
                                            uint32_t key) {
  const int lane = threadIdx.x & 31;
  uint32_t todo = __ballot_sync(0xffffffffu, want);
  while (todo) {
    const int leader = __ffs(todo) - 1;
    const int lq = __shfl_sync(0xffffffffu, qi, leader);
    const int lf = __shfl_sync(0xffffffffu, (int)far, leader);
    const bool mine = want && qi == lq && (int)far == lf;
    const uint32_t grp = __ballot_sync(0xffffffffu, mine);
    const uint32_t kmin = __reduce_min_sync(0xffffffffu, mine ? key : 0xFFFFFFFFu);
    Ctx* c = ctxs + lq;
    uint32_t base = 0;
    if (lane == leader) {
      base = atomicAdd(lf ? &c->n_far[c->f] : &c->n_q[c->no], (uint32_t)__popc(grp));
      if (lf) atomicMin(&c->far_min, kmin);
    }
    base = __shfl_sync(0xffffffffu, base, leader);
    if (mine) {
      const uint32_t i = base + __popc(grp & ((1u << lane) - 1u));
      if (lf) {
        if (i < c->farcap) c->far[c->f][i] = make_uint4(v, pd, cost, off);
        else atomicOr(&c->error, (uint32_t)ERR_FARCAP);
      } else {
        if (i < c->qcap) c->q[c->no][i] = make_uint4(v, pd, cost, off);
        else atomicOr(&c->error, (uint32_t)ERR_QCAP);
      }
    }
    todo &= ~grp;
  }
}

// Lane appends the n chunk items {v, pd | CHUNK, cost, off + j * split}, j < n, to
// query qi's near list.
__device__ __forceinline__ void warp_append_chunks(Ctx* ctxs, int qi, uint32_t n, uint32_t v,
                                                   uint32_t pd, uint32_t cost, uint32_t off,
                                                   int split) {
  const int lane = threadIdx.x & 31;
  uint32_t todo = __ballot_sync(0xffffffffu, n > 0);
  while (todo) {
    const int leader = __ffs(todo) - 1;
    const int lq = __shfl_sync(0xffffffffu, qi, leader);
    const bool mine = n > 0 && qi == lq;
    const uint32_t x = mine ? n : 0u;
    const uint32_t scan = warp_incl_scan(x);
    const uint32_t total = __shfl_sync(0xffffffffu, scan, 31);
    Ctx* c = ctxs + lq;
    uint32_t base = 0;
    if (lane == leader) base = atomicAdd(&c->n_q[c->no], total);
    base = __shfl_sync(0xffffffffu, base, leader);
    if (mine) {
      uint32_t i = base + scan - x;
      for (uint32_t j = 0; j < n; j++, i++) {
        if (i < c->qcap) c->q[c->no][i] = make_uint4(v, pd | CHUNK, cost, off + j * (uint32_t)split);
        else atomicOr(&c->error, (uint32_t)ERR_QCAP);
      }
    }
    todo &= ~__ballot_sync(0xffffffffu, mine);
  }
}

// Plan the item {v, pd, cost, off}: the edge range [eb, eb + n) to relax now, and at
// most one follow-up item (a continuation of a long range into the near list, or
// the rest of the list into the far list under the key of its next edge).
// wmax: heaviest edge the state may still use (the upper bound's limit).
// A head item (no CHUNK flag) relaxes the first `split` edges of its range now and
// spawns chunk items for the rest of the range, which the next step relaxes in
// parallel (hub vertices spread over many warps); only a head item defers the
// remainder of its list to the far list.  A chunk item relaxes its chunk only.
struct Plan {
  int64_t eb;
  uint32_t n;
  bool push, far;
  uint32_t off, key;
  uint32_t spawn;   // chunk items to append at offsets off + n + j * split
};
// b0, b1: v's row offsets, loaded by the caller together with the item's other
// loads (they depend only on v), so that planning adds one dependent load, the
// light-edge count.
__device__ __forceinline__ Plan plan_item(const DevGraph& G, uint32_t v, int64_t b0, int64_t b1,
                                          uint32_t cost, uint32_t off, uint32_t wmax,
                                          uint32_t bucket_end, int split, bool chunk) {
  Plan P{0, 0u, false, false, 0u, 0u, 0u};
  const int64_t deg = b1 - b0;
  const uint64_t in_bucket = bucket_end > cost ? (uint64_t)bucket_end - cost - 1u : 0u;
  const uint32_t hw = (uint32_t)min((uint64_t)wmax, in_bucket);
  const int64_t cnt = count_upto(G, v, deg, hw);
  if ((int64_t)off >= deg) return P;
  if (chunk) {  // a chunk of a range planned by its head item
    const int64_t end = min(cnt, (int64_t)off + split);
    if (end > (int64_t)off) {
      P.eb = b0 + off;
      P.n = (uint32_t)(end - off);
    }
    return P;
  }
  if (cnt <= (int64_t)off) {
    // nothing of this bucket left: defer to the bucket of the next edge, if the
    // bound still allows it
    if (!G.widx) return P;
    const uint32_t w0 = (uint32_t)__ldg(&G.wedges[b0 + off].y);
    if (w0 > wmax) return P;
    P.push = P.far = true;
    P.off = off;
    P.key = (uint32_t)min((uint64_t)cost + w0, (uint64_t)0xFFFFFFFEu);
    return P;
  }
  const int64_t end = cnt;
  const int64_t stop = min(end, (int64_t)off + split);
  P.eb = b0 + off;
  P.n = (uint32_t)(stop - off);
  if (stop < end) P.spawn = (uint32_t)((end - stop + split - 1) / split);
  if (end < deg && hw < wmax) {
    // the rest of the list waits for the bucket of its first edge
    const uint32_t w1 = (uint32_t)__ldg(&G.wedges[b0 + end].y);
    if (w1 <= wmax) {
      P.push = P.far = true;
      P.off = (uint32_t)end;
      P.key = (uint32_t)min((uint64_t)cost + max(w1, hw + 1u), (uint64_t)0xFFFFFFFEu);
    }
  }
  return P;
}

// Lane with `want` marks row u of query qi dirty; rows newly marked are appended
// to the query's row list with one atomicAdd per warp and query.
__device__ __forceinline__ void warp_mark_row(Ctx* ctxs, int qi, bool want, uint32_t u) {
  const int lane = threadIdx.x & 31;
  bool fresh = false;
  if (want) {
    Ctx* c = ctxs + qi;
    const uint32_t bit = 1u << (u & 31);
    fresh = !(atomicOr(&c->rowbits[u >> 5], bit) & bit);
  }
  uint32_t todo = __ballot_sync(0xffffffffu, fresh);
  while (todo) {
    const int leader = __ffs(todo) - 1;
    const int lq = __shfl_sync(0xffffffffu, qi, leader);
    const bool mine = fresh && qi == lq;
    const uint32_t grp = __ballot_sync(0xffffffffu, mine);
    Ctx* c = ctxs + lq;
    uint32_t base = 0;
    if (lane == leader) base = atomicAdd(&c->n_rows, (uint32_t)__popc(grp));
    base = __shfl_sync(0xffffffffu, base, leader);
    if (mine) {
      const uint32_t i = base + __popc(grp & ((1u << lane) - 1u));
      if (i < c->rowcap) c->rows[i] = u;
      else atomicOr(&c->error, (uint32_t)ERR_ROWCAP);
    }
    todo &= ~grp;
  }
}


// Per-CTA prefix of the input counts of all queries of the launch (MAXB <= 64:
// the first warp loads two contexts per lane and scans them).
// want: PH_SSSP (sssp input), PH_DP (grow input) or -1 (rows of DP-phase queries).
__device__ __forceinline__ uint32_t ctx_count(const Ctx* c, int want) {
  if (want < 0) return (c->phase == PH_DP) ? min(c->n_rows, c->rowcap) : 0u;
  return (c->phase == (uint32_t)want) ? c->in_n : 0u;
}
__device__ __forceinline__ void load_prefix(Ctx* ctxs, int nctx, uint32_t* s_pref, int want) {
  static_assert(MAXB <= 64, "load_prefix scans two contexts per lane");
  if (threadIdx.x < 32) {
    const int lane = threadIdx.x;
    const uint32_t n0 = lane < nctx ? ctx_count(ctxs + lane, want) : 0u;
    const uint32_t n1 = lane + 32 < nctx ? ctx_count(ctxs + lane + 32, want) : 0u;
    const uint32_t s0 = warp_incl_scan(n0);
    const uint32_t t0 = __shfl_sync(0xffffffffu, s0, 31);
    const uint32_t s1 = warp_incl_scan(n1) + t0;
    if (lane == 0) s_pref[0] = 0;
    if (lane < nctx) s_pref[lane + 1] = s0;
    if (lane + 32 < nctx) s_pref[lane + 33] = s1;
  }
  __syncthreads();
}
__device__ __forceinline__ int find_ctx(const uint32_t* s_pref, int nctx, uint32_t it) {
  int lo = 0, hi = nctx;  // s_pref[lo] <= it < s_pref[hi]
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (s_pref[mid] <= it) lo = mid;
    else hi = mid;
  }
  return lo;
}

// Warp-aggregated per-query counter update: lanes with `valid` add x to the
// counter of their own query.
__device__ __forceinline__ void add_stat(Ctx* ctxs, int qi, bool valid, uint32_t x,
                                         unsigned long long Ctx::*field) {
  const uint32_t act = __ballot_sync(0xffffffffu, valid && x > 0);
  if (!act) return;
  const int lane = threadIdx.x & 31;
  const uint32_t peers = __match_any_sync(0xffffffffu, valid && x > 0 ? qi : -1);
  const uint32_t tot = __reduce_add_sync(peers, valid && x > 0 ? x : 0u);
  if (valid && x > 0 && lane == __ffs(peers) - 1)
    atomicAdd(&(ctxs[qi].*field), (unsigned long long)tot);
}

// ---- group cache: distance rows of a query from cached per-group vectors ----------
struct GroupVecs {
  const uint32_t* v[KMAX];  // d_i(.) of the query's i-th group, V entries each (nullptr:
                            // not cached, left unreached for the distance search)
};
// rows: V distance rows of stride ds (the distance table, or one hop budget's table)
__global__ void k_gather_dist(uint32_t* rows, uint32_t ds, int k, GroupVecs gv, int64_t V) {
  for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < V;
       v += (int64_t)gridDim.x * blockDim.x) {
    uint32_t d[KMAX];
#pragma unroll
    for (int i = 0; i < KMAX; i++) d[i] = i < k && gv.v[i] ? __ldg(&gv.v[i][v]) : COST_INF;
    store_drow(rows, ds, (uint64_t)v, make_uint4(d[0], d[1], d[2], d[3]),
               make_uint4(d[4], d[5], d[6], d[7]));
  }
}

// ---- init: group members -> zero-cost singletons, SSSP sources, dirty rows ----
__global__ void k_init(Ctx* ctxs, int nctx, DevGraph G, const int64_t* grp_ptr,
                       const int32_t* members, int split) {
  for (int qi = blockIdx.y; qi < nctx; qi += gridDim.y) {
    Ctx* c = ctxs + qi;
    for (int i = 0; i < c->k; i++) {
      const int32_t g = c->gid[i];
      const int64_t b = grp_ptr[g], e = grp_ptr[g + 1];
      for (int64_t j = b + blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < e;
           j += (int64_t)gridDim.x * blockDim.x) {
        const uint32_t v = (uint32_t)members[j];
        if (!in_bounds(c, v < G.V && i < c->k, 1)) continue;
        const uint64_t cell0 = pack_cell(0, PEND | LEAF);
        uint64_t* row = row_take(c, v, c->rowmap ? __ldcg(&c->rowmap[v]) : 0u);
        if (!row) continue;
        atomicMin((unsigned long long*)&row[1u << i], (unsigned long long)cell0);
        mark_row(c, v);
        if (c->phase == PH_SSSP) {
          const uint32_t old = atomicMin(&c->dist[(uint64_t)v * c->ds + i], 0u);
          for (int h = 1; h <= c->nhb; h++)
            c->dist_h[((uint64_t)(h - 1) * (uint64_t)G.V + v) * c->ds + i] = 0u;
          const int64_t deg = G.beg[v + 1] - G.beg[v];
          if (old != 0u && deg > 0 && c->sssp_mask) {
            // group-mask items: one head item per vertex (hop count 0), the groups in fm
            const uint32_t sh = (v & 3u) * 8u;
            const uint32_t ow = atomicOr(&c->fm[c->no][v >> 2], (1u << i) << sh);
            if (((ow >> sh) & 0xFFu) == 0u) {
              const uint32_t n = atomicAdd(&c->n_q[c->no], 1u);
              if (n < c->qcap) c->q[c->no][n] = make_uint4(v, 0u, 0u, 0u);
              else atomicOr(&c->error, (uint32_t)ERR_QCAP);
            }
          } else if (old != 0u && deg > 0) {
            // group items: one head item per (member, group)
            const uint32_t n = atomicAdd(&c->n_q[c->no], 1u);
            if (n < c->qcap) c->q[c->no][n] = make_uint4(v, (uint32_t)i, 0u, 0u);
            else atomicOr(&c->error, (uint32_t)ERR_QCAP);
          }
        }
      }
    }
  }
}

// ---- one-label SSSP step: multi-source Bellman-Ford with near/far ordering ----
// Two item forms (code/TrimCDP-WB/include/mapper_enactor.cuh:249-366 computes the
// same distances as grow-only DP states (v, 1<<i)):
//  - group items {v, group index i [| hops << 8], dist, offset}: relax d_i(u) for the
//    edges of the item (searches in cost buckets);
//  - group-mask items (sssp_mask): a head item {v, hops << 8, 0, 0} takes the groups
//    whose d_i(v) improved in the previous step from fm[in_idx] (and clears them); a
//    chunk item {v, mask | hops << 8 | CHUNK, 0, offset} carries its groups.  Each
//    edge is read once for all of the item's groups and the target's 32-byte
//    distance row once, and a vertex improved for several groups in one step is
//    queued once.  A distance written in a step is announced in fm of that step,
//    read only by the next launch, so every write is visible to the item that its
//    bit schedules.  Unlimited distances (sssp_mask 1) relax with the distances
//    current when an item runs (a value at most the one announced).  Hop-limited
//    distances d_i^{<=D} (sssp_mask 2) run level-synchronous rounds of two steps:
//    the expand step snapshots the rows of the announced vertices and queues all
//    their chunks, the relax step extends exactly those distances by one edge
//    (rounds 1..D), so that the result is the same as one item per path.
// Lane-local item word of the search: bits 0..7 the group mask (group-mask items) or
// group index, 8..15 the round (hop-limited searches), 24..27 k, bit 30 SSSP_MASKED;
// in the worklists bit 31 is CHUNK.
constexpr uint32_t SSSP_MASKED = 0x40000000u;  // lane-local flag: a group-mask item
constexpr int SSSP_U = 2;                      // edges per lane per round of the relax loop
__global__ void __launch_bounds__(256, 4) k_sssp(Ctx* ctxs, int nctx, DevGraph G, int split) {
  __shared__ uint32_t s_pref[MAXB + 1];
  // per warp and lane: the distances of the lane's group-mask item (COST_INF for
  // groups outside its mask), read by the lanes that relax its edges
  __shared__ uint4 s_dv[256 / 32][32][2];
  load_prefix(ctxs, nctx, s_pref, PH_SSSP);
  const uint32_t total = s_pref[nctx];
  const int lane = threadIdx.x & 31;
  const int wib = threadIdx.x >> 5;
  const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
  const uint32_t wid = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  for (uint32_t base = wid * 32; base < total; base += warps * 32) {
    const uint32_t it = base + lane;
    uint32_t v = 0, gi = 0, cost = 0, ub = 0, bend = 0, e_off = 0;
    int qi = 0;
    Plan P{0, 0u, false, false, 0u, 0u, 0u};
    uint32_t dv[KMAX];
#pragma unroll
    for (int i = 0; i < KMAX; i++) dv[i] = COST_INF;
    if (it < total) {
      qi = find_ctx(s_pref, nctx, it);
      Ctx* c = ctxs + qi;
      const uint4 e = c->in_ptr[it - s_pref[qi]];
      v = e.x;
      gi = e.y;
      cost = e.z;
      e_off = e.w;
      const uint32_t g = gi & 0xFFu;
      if (c->sssp_mask) {
        if (in_bounds(c, v < G.V, 2)) {
          const int64_t b0 = G.beg[v], b1 = G.beg[v + 1];
          const bool chunk = (gi & CHUNK) != 0u;
          const uint32_t hops = (gi >> SSSP_HOP_SHIFT) & 0xFFu;
          const bool rounds = c->sssp_mask == 2u;
          uint32_t m;
          if (chunk) {
            m = g;
          } else {
            unsigned char* fb = (unsigned char*)c->fm[c->in_idx] + v;
            m = __ldcg(fb);
            *fb = 0;
          }
          // a hop-limited round relaxes from the distances its frontier had when the
          // round began (the snapshot its expand step took), so that a round extends
          // paths by exactly one edge
          const uint32_t* src = rounds && chunk ? c->snap : c->dist;
          uint4 a, b;
          load_drow(src, c->ds, v, a, b);
          const uint32_t d[8] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w};
          ub = sssp_cutoff(c);
          bend = COST_INF;
          const int k = c->k;
          uint32_t mind = COST_INF, mk = 0;
#pragma unroll
          for (int i = 0; i < KMAX; i++)
            if (i < k && ((m >> i) & 1u) && d[i] < ub) {
              dv[i] = d[i];
              mind = min(mind, d[i]);
              mk |= 1u << i;
            }
          cost = mind;
          gi = mk | (hops << SSSP_HOP_SHIFT) | SSSP_MASKED | ((uint32_t)k << 24);
          if (rounds && !chunk) {
            // expand step of a round: snapshot the row, queue every chunk of the range
            // for the next step, relax nothing (no distance changes in this step)
            store_drow(c->snap, c->ds, v, a, b);
            if (mk) {
              const int64_t cnt = count_upto(G, v, b1 - b0, ub - mind);
              P.spawn = (uint32_t)((cnt + split - 1) / split);
            }
            e_off = 0;
          } else if (mk) {
            P = plan_item(G, v, b0, b1, mind, e.w, ub - mind, bend, split, chunk);
          }
        }
      } else if (in_bounds(c, v < G.V && g < (uint32_t)c->k, 2)) {
        const int64_t b0 = G.beg[v], b1 = G.beg[v + 1];
        const uint32_t cur = __ldcg(&c->dist[(uint64_t)v * c->ds + g]);
        // ub is read once per item (a per-edge read of one word by every thread of
        // a one-query launch is an L2 hot spot); a stale, larger ub prunes less
        ub = sssp_cutoff(c);
        bend = c->bucket_end;
        // not stale, and still able to reach a vertex at distance <= ub
        if (cur >= cost && cost < ub)
          P = plan_item(G, v, b0, b1, cost, e.w, ub - cost, bend, split, (gi & CHUNK) != 0u);
      }
      gi &= ~CHUNK;
    }
    s_dv[wib][lane][0] = make_uint4(dv[0], dv[1], dv[2], dv[3]);
    s_dv[wib][lane][1] = make_uint4(dv[4], dv[5], dv[6], dv[7]);
    __syncwarp();
    warp_append(ctxs, qi, P.push, P.far, v, gi, cost, P.off, P.key);
    warp_append_chunks(ctxs, qi, P.spawn, v, (gi & SSSP_MASKED) ? (gi & 0xFFFFu) : gi, cost,
                       e_off + P.n, split);
    const uint32_t n = P.n;
    const int64_t eb = P.eb;
    add_stat(ctxs, qi, it < total, n, &Ctx::st_sssp);
    const uint32_t scan = warp_incl_scan(n);
    const uint32_t tot = __shfl_sync(0xffffffffu, scan, 31);
    // SSSP_U edges per lane per round: their loads are independent, so a warp has
    // SSSP_U edge loads, then SSSP_U distance loads, in flight at once
    for (uint32_t j0 = 0; j0 < tot; j0 += 32 * SSSP_U) {
      int2 ed[SSSP_U];
      uint32_t x_gi[SSSP_U], x_cost[SSSP_U], x_ub[SSSP_U], x_o[SSSP_U];
      uint4 ra[SSSP_U], rb[SSSP_U];  // target's distance row (ra.x alone for group items)
      int x_qi[SSSP_U];
      bool ok[SSSP_U];
#pragma unroll
      for (int x = 0; x < SSSP_U; x++) {
        const uint32_t j = j0 + (uint32_t)x * 32u + lane;
        const int o = warp_owner(scan, j < tot ? j : tot - 1);
        const uint32_t o_scan = __shfl_sync(0xffffffffu, scan, o);
        const uint32_t o_n = __shfl_sync(0xffffffffu, n, o);
        const int64_t o_eb = __shfl_sync(0xffffffffu, eb, o);
        x_o[x] = (uint32_t)o;
        x_gi[x] = __shfl_sync(0xffffffffu, gi, o);
        x_cost[x] = __shfl_sync(0xffffffffu, cost, o);
        x_ub[x] = __shfl_sync(0xffffffffu, ub, o);
        x_qi[x] = __shfl_sync(0xffffffffu, qi, o);
        const uint32_t off = j - (o_scan - o_n);
        ok[x] = j < tot && in_bounds(ctxs + x_qi[x], o_eb + off < G.E, 3);
        ed[x] = ok[x] ? G.wedges[o_eb + off] : make_int2(0, 0);
      }
#pragma unroll
      for (int x = 0; x < SSSP_U; x++) {
        const uint32_t u = (uint32_t)ed[x].x, nd = x_cost[x] + (uint32_t)ed[x].y;
        // distances above ub are never needed exactly: a state whose missing group
        // lies further than ub is pruned whatever the exact distance (for a group-mask
        // item, cost is its smallest distance)
        ok[x] = ok[x] && in_bounds(ctxs + x_qi[x], u < G.V, 4) && nd <= x_ub[x];
        const uint32_t xds = ctxs[x_qi[x]].ds;
        const uint32_t* dbase = ctxs[x_qi[x]].dist;
        ra[x] = make_uint4(0u, 0u, 0u, 0u);
        rb[x] = make_uint4(COST_INF, COST_INF, COST_INF, COST_INF);
        if (ok[x] && (x_gi[x] & SSSP_MASKED)) {
          load_drow(dbase, xds, u, ra[x], rb[x]);
        } else if (ok[x]) {
          ra[x].x = __ldcg(dbase + (uint64_t)u * xds + (x_gi[x] & 0xFFu));
        }
      }
#pragma unroll
      for (int x = 0; x < SSSP_U; x++) {
        const uint32_t u = (uint32_t)ed[x].x, w = (uint32_t)ed[x].y, nd = x_cost[x] + w;
        Ctx* c = ctxs + x_qi[x];
        bool push = false, far = false;
        uint32_t p_gi = 0, p_cost = 0;
        if (ok[x] && (x_gi[x] & SSSP_MASKED)) {
          // group-mask edge: every group of the owner's item whose distance through
          // this edge beats the target's
          const uint4 oa = s_dv[wib][x_o[x]][0], ob = s_dv[wib][x_o[x]][1];
          const uint32_t od[8] = {oa.x, oa.y, oa.z, oa.w, ob.x, ob.y, ob.z, ob.w};
          uint32_t cu[8] = {ra[x].x, ra[x].y, ra[x].z, ra[x].w, rb[x].x, rb[x].y, rb[x].z, rb[x].w};
          const int k = (int)((x_gi[x] >> 24) & 0xFu);
          const uint32_t lim = x_ub[x];
          uint32_t imp = 0, ext = 0;
#pragma unroll
          for (int i = 0; i < KMAX; i++) {
            if (i < k && od[i] < lim && w <= lim - od[i]) {
              const uint32_t ndi = od[i] + w;
              if (ndi < cu[i]) {
                const uint32_t old = atomicMin(&c->dist[(uint64_t)u * c->ds + i], ndi);
                if (ndi < old) {
                  imp |= 1u << i;
                  if (ndi < lim) ext |= 1u << i;
                  // a path of hops + 1 edges (hop-limited rounds): a candidate for every
                  // budget from hops + 1 on
                  for (int h = (int)((x_gi[x] >> SSSP_HOP_SHIFT) & 0xFFu) + 1; h <= c->nhb; h++)
                    atomicMin(&c->dist_h[((uint64_t)(h - 1) * (uint64_t)G.V + u) * c->ds + i],
                              ndi);
                }
                cu[i] = min(ndi, old);
              }
            }
          }
          if (imp) {
            // star bound (see below): the k shortest paths found so far from u
            uint64_t sum = 0;
#pragma unroll
            for (int i = 0; i < KMAX; i++)
              if (i < k) sum += cu[i];
            if (sum < (uint64_t)lim) atomicMin(&c->ub, (uint32_t)sum);
            // hop-limited rounds up to D/2: every distance of u comes from a path of at
            // most D/2 edges, so the star spans a tree of diameter <= D
            const uint32_t hr = ((x_gi[x] >> SSSP_HOP_SHIFT) & 0xFFu) + 1u;
            if (c->sssp_hops && 2u * hr <= c->sssp_hops && sum < (uint64_t)__ldcg(&c->ub_hop))
              atomicMin(&c->ub_hop, (uint32_t)sum);
          }
          // a hop-limited round: u's paths of hops + 1 edges extend only while the
          // bound allows one more edge
          const uint32_t hops = (x_gi[x] >> SSSP_HOP_SHIFT) & 0xFFu, hl = c->sssp_hops;
          if (hl && hops + 1u >= hl) ext = 0u;
          if (ext) {
            // announce the improved groups to the next step; the first announcement
            // of u in this step queues it
            const uint32_t sh = (u & 3u) * 8u;
            const uint32_t ow = atomicOr(&c->fm[c->no][u >> 2], ext << sh);
            push = ((ow >> sh) & 0xFFu) == 0u;
            p_gi = hl ? (hops + 1u) << SSSP_HOP_SHIFT : 0u;
          }
        } else if (ok[x] && nd < ra[x].x) {
          const uint32_t grp = x_gi[x] & 0xFFu;
          const uint32_t old = atomicMin(&c->dist[(uint64_t)u * c->ds + grp], nd);
          if (nd < old) {
            // star bound from tentative distances: the k paths found so far from u
            // to a member of each group form a connected subgraph covering every
            // group, so their total length is a feasible cost
            uint4 a, b;
            load_drow(c->dist, c->ds, u, a, b);
            const uint32_t d[8] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w};
            const int k = c->k;
            uint64_t sum = 0;
#pragma unroll
            for (int i = 0; i < KMAX; i++)
              if (i < k) sum += (i == (int)grp) ? nd : d[i];
            if (sum < (uint64_t)x_ub[x]) atomicMin(&c->ub, (uint32_t)sum);
            push = nd < x_ub[x];
            // an improved vertex relaxes its own edges from the lightest one, which
            // lands at nd + 1 or later: in this bucket or a later one
            far = (uint64_t)nd + 1u >= c->bucket_end;
            p_gi = grp;
            p_cost = nd;
          }
        }
        warp_append(ctxs, x_qi[x], push, far, u, p_gi, p_cost, 0u, p_cost + 1u);
      }
    }
    __syncwarp();
  }
  // Queries whose distances are final (PH_PREP): one pass over the distance rows
  // gives the star bound min_v sum_i d_i(v) (the cost of the k shortest paths from
  // the best centre v, a feasible tree, so a valid ub) and the group distances
  // vv[i][j] = min over members m of group i of d_j(m) (the host loop of
  // code/TrimCDP-WB/src/GSTnonHop.cu:341-353, done on the device).
  for (int qi = 0; qi < nctx; qi++) {
    Ctx* c = ctxs + qi;
    if (c->phase != PH_PREP) continue;
    const int k = c->k;
    uint32_t best = COST_INF, best_h = COST_INF;
    // Hop-bounded queries: a star whose k paths have at most D/2 edges each spans a tree
    // of diameter <= D (breadth-first from the centre, every vertex lies within D/2
    // edges of it), so min_v sum_i d_i^{<=D/2}(v) is a feasible cost of the query
    const int hs = c->hop && c->sssp_hops && c->D / 2 <= c->nhb ? c->D / 2 : -1;
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < G.V;
         v += (int64_t)gridDim.x * blockDim.x) {
      uint4 a, b;
      load_drow(c->dist, c->ds, (uint64_t)v, a, b);
      const uint32_t d[8] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w};
      uint64_t sum = 0;
#pragma unroll
      for (int i = 0; i < KMAX; i++)
        if (i < k) sum += d[i];
      if (sum < best) best = (uint32_t)sum;
      if (hs >= 0) {
        uint4 ha, hb;
        budget_row(c, G.V, (uint32_t)v, hs, ha, hb);
        const uint32_t e[8] = {ha.x, ha.y, ha.z, ha.w, hb.x, hb.y, hb.z, hb.w};
        uint64_t sh = 0;
#pragma unroll
        for (int i = 0; i < KMAX; i++)
          if (i < k) sh += e[i];
        if (sh < best_h) best_h = (uint32_t)sh;
      }
#pragma unroll
      for (int i = 0; i < KMAX; i++)
        if (i < k && d[i] == 0u) {
#pragma unroll
          for (int j = 0; j < KMAX; j++)
            if (j < k && d[j] < __ldcg(&c->vv[i * KMAX + j])) atomicMin(&c->vv[i * KMAX + j], d[j]);
        }
    }
    best = __reduce_min_sync(0xffffffffu, best);
    best_h = __reduce_min_sync(0xffffffffu, best_h);
    if ((threadIdx.x & 31) == 0 && best < COST_INF && best < __ldcg(&c->ub))
      atomicMin(&c->ub, best);
    // ub_cell bounds with strict tests (a state must beat a tree already found), so a
    // feasible cost that no state holds yet enters it plus one
    if ((threadIdx.x & 31) == 0 && best_h < COST_INF - 1u) atomicMin(&c->ub_cell, best_h + 1u);
  }
}

// ---- DP grow step ----------------------------------------------------------------
__global__ void __launch_bounds__(256, 3) k_grow(Ctx* ctxs, int nctx, DevGraph G, int split) {
  __shared__ uint32_t s_pref[MAXB + 1];
  load_prefix(ctxs, nctx, s_pref, PH_DP);
  const uint32_t total = s_pref[nctx];
  const int lane = threadIdx.x & 31;
  const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
  const uint32_t wid = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  for (uint32_t base = wid * 32; base < total; base += warps * 32) {
    const uint32_t it = base + lane;
    uint32_t v = 0, pd = 0, cost = 0, bound = 0, e_off = 0;
    bool chunk = false;
    int qi = 0;
    Plan P{0, 0u, false, false, 0u, 0u, 0u};
    if (it < total) {
      qi = find_ctx(s_pref, nctx, it);
      Ctx* c = ctxs + qi;
      const uint4 e = c->in_ptr[it - s_pref[qi]];
      v = e.x;
      chunk = (e.y & CHUNK) != 0u;
      pd = e.y & ~CHUNK;
      cost = e.z;
      e_off = e.w;
      const uint32_t p = pd & 0xFFFFu, d = pd >> 16;
      const bool ok = in_bounds(c, v < G.V && p < (uint32_t)c->W && d < (uint32_t)c->DD, 5);
      const int64_t b0 = ok ? G.beg[v] : 0, b1 = ok ? G.beg[v + 1] : 0;
      const uint64_t* srow = ok ? row_of(c, v) : nullptr;
      const uint64_t cell = srow ? __ldcg((const unsigned long long*)&srow[((uint64_t)d << c->k) + p])
                                 : CELL_INF;
      bound = c->hop ? __ldcg(&c->ub_cell) : __ldcg(&c->ub);
      // a work item always names a state that holds a finite cost
      const bool src_ok = !ok || in_bounds(c, cost_of(cell) != COST_INF, 12);
      if (ok && src_ok && cost_of(cell) >= cost && 2ull * cost <= (uint64_t)bound) {
        const uint32_t wmax = c->hop ? (bound > cost ? bound - cost - 1u : 0u)
                                     : (bound >= cost ? bound - cost : 0u);
        P = plan_item(G, v, b0, b1, cost, e.w, wmax, c->bucket_end, split, chunk);
      }
    }
    warp_append(ctxs, qi, P.push, P.far, v, pd, cost, P.off, P.key);
    warp_append_chunks(ctxs, qi, P.spawn, v, pd, cost, e_off + P.n, split);
    const uint32_t n = P.n;
    const int64_t eb = P.eb;
    add_stat(ctxs, qi, it < total, n, &Ctx::st_relax);
    add_stat(ctxs, qi, it < total, n > 0 ? 1u : 0u, &Ctx::st_items);
    const uint32_t scan = warp_incl_scan(n);
    const uint32_t tot = __shfl_sync(0xffffffffu, scan, 31);
    for (uint32_t j0 = 0; j0 < tot; j0 += 32 * RELAX_U) {
      int2 ed[RELAX_U];
      uint32_t x_v[RELAX_U], x_pd[RELAX_U], x_cost[RELAX_U], x_bound[RELAX_U];
      uint64_t cur[RELAX_U];
      int x_qi[RELAX_U];
      bool ok[RELAX_U];
#pragma unroll
      for (int x = 0; x < RELAX_U; x++) {
        const uint32_t j = j0 + (uint32_t)x * 32u + lane;
        const int o = warp_owner(scan, j < tot ? j : tot - 1);
        const uint32_t o_scan = __shfl_sync(0xffffffffu, scan, o);
        const uint32_t o_n = __shfl_sync(0xffffffffu, n, o);
        const int64_t o_eb = __shfl_sync(0xffffffffu, eb, o);
        x_v[x] = __shfl_sync(0xffffffffu, v, o);
        x_pd[x] = __shfl_sync(0xffffffffu, pd, o);
        x_cost[x] = __shfl_sync(0xffffffffu, cost, o);
        x_bound[x] = __shfl_sync(0xffffffffu, bound, o);
        x_qi[x] = __shfl_sync(0xffffffffu, qi, o);
        const uint32_t off = j - (o_scan - o_n);
        ok[x] = j < tot && in_bounds(ctxs + x_qi[x], o_eb + off < G.E, 6);
        ed[x] = ok[x] ? G.wedges[o_eb + off] : make_int2(0, 0);
      }
      // The bounds are tested before the target's cell is read: an improving target
      // state (u, X) that cannot be part of a tree within the bound is not written
      // at all (its cost plus the one-label bound max_{i not in X} d_i(u), or the
      // O(k) half of the tour bound, exceeds the bound; the same tests the rows
      // kernel applies before growing a state).  The distance rows of a query
      // (32 bytes per vertex) stay in L2 while its state table does not, so the
      // tests come first and only edges that pass them read a table cell.
      uint4 da[RELAX_U], db[RELAX_U];
      uint32_t rm[RELAX_U];  // the target's pool row (row pool), loaded with its distances
#pragma unroll
      for (int x = 0; x < RELAX_U; x++) {
        Ctx* c = ctxs + x_qi[x];
        const uint32_t u = (uint32_t)ed[x].x, nc = x_cost[x] + (uint32_t)ed[x].y;
        // a target costing more than ub cannot be part of an optimal tree
        const int hop = c->hop;
        const bool keep = hop ? (nc < x_bound[x]) : (nc <= x_bound[x]);
        const uint32_t d = (x_pd[x] >> 16) + (uint32_t)hop;
        ok[x] = ok[x] && in_bounds(c, u < G.V, 7) && keep && in_bounds(c, d < (uint32_t)c->DD, 11);
        rm[x] = ok[x] && c->rowmap ? __ldcg(&c->rowmap[u]) : ROW_NONE;
        da[x] = db[x] = make_uint4(0, 0, 0, 0);
        if (ok[x] && c->use_lb) {
          if (hop && c->sssp_hops) {
            // the target state has height d: its bounds are the distances within the
            // hop budget D - d
            budget_row(c, G.V, u, c->D - (int)d, da[x], db[x]);
          } else {
            load_drow(c->dist, c->ds, u, da[x], db[x]);
          }
        }
      }
#pragma unroll
      for (int x = 0; x < RELAX_U; x++) {
        Ctx* c = ctxs + x_qi[x];
        const uint32_t u = (uint32_t)ed[x].x, nc = x_cost[x] + (uint32_t)ed[x].y;
        const uint32_t p = x_pd[x] & 0xFFFFu, d = (x_pd[x] >> 16) + (uint32_t)c->hop;
        if (ok[x] && c->use_lb) {
          const uint32_t cut = c->cut;
          const uint32_t lim = cut == COST_INF ? COST_INF : cut + 1u;
          const uint32_t dd[8] = {da[x].x, da[x].y, da[x].z, da[x].w,
                                  db[x].x, db[x].y, db[x].z, db[x].w};
          const int k = c->k;
          uint32_t lb = 0;
#pragma unroll
          for (int i = 0; i < KMAX; i++)
            if (i < k && !((p >> i) & 1u)) lb = max(lb, min(dd[i], lim));
          if ((uint64_t)nc + lb > (uint64_t)x_bound[x]) ok[x] = false;
          if (ok[x] && c->use_tour && p != (uint32_t)c->full) {
            // the O(k) half of the tour bound (see the rows kernel): twice the rest
            // of any tree holding (u, p) costs at least
            // max_a d_a(u) + min_b P(a,b,Xb) + min_b d_b(u) over groups a, b not in p
            const uint32_t Xb = (uint32_t)c->full ^ p;
            const uint32_t* W2 = c->tour + (size_t)c->W * TOUR_STRIDE + (size_t)Xb * KMAX;
            uint32_t mind = COST_INF;
#pragma unroll
            for (int i = 0; i < KMAX; i++)
              if (i < k && ((Xb >> i) & 1u)) mind = min(mind, min(dd[i], lim));
            uint64_t lb2 = 0;
#pragma unroll
            for (int i = 0; i < KMAX; i++)
              if (i < k && ((Xb >> i) & 1u)) {
                const uint64_t t2 = (uint64_t)min(dd[i], lim) + __ldg(&W2[i]) + mind;
                lb2 = t2 > lb2 ? t2 : lb2;
              }
            if ((uint64_t)nc + (lb2 + 1) / 2 > (uint64_t)x_bound[x]) ok[x] = false;
          }
        }
        // the target's cell: unreached when its vertex has no pool row yet
        const bool has_row = ok[x] && (!c->rowmap || rm[x] != ROW_NONE);
        const uint64_t off = ((uint64_t)d << c->k) + p;
        cur[x] = has_row ? __ldcg((const unsigned long long*)&(c->rowmap ? c->table + (uint64_t)rm[x] * c->RW
                                                                         : c->table + (uint64_t)u * c->RW)[off])
                         : CELL_INF;
      }
#pragma unroll
      for (int x = 0; x < RELAX_U; x++) {
        Ctx* c = ctxs + x_qi[x];
        const uint32_t u = (uint32_t)ed[x].x, nc = x_cost[x] + (uint32_t)ed[x].y;
        bool dirty = false;
        if (ok[x] && pack_cell(nc, PEND | x_v[x]) < cur[x]) {
          const uint32_t p = x_pd[x] & 0xFFFFu, d = (x_pd[x] >> 16) + (uint32_t)c->hop;
          uint64_t* row = row_take(c, u, rm[x]);
          if (row) {
            unsigned long long* tp = (unsigned long long*)&row[((uint64_t)d << c->k) + p];
            const uint64_t old = atomicMin(tp, (unsigned long long)pack_cell(nc, PEND | x_v[x]));
            dirty = cost_of(old) > nc;
          }
        }
        warp_mark_row(ctxs, x_qi[x], dirty, u);
      }
    }
  }
}

// ---- DP rows step: merge closure of dirty rows in shared memory -------------------
// Per-warp shared memory: RW cells, RW/32 pending words, RW/32 processed words, three
// lists of RW cell indices (pending cells, finite cells, the cells of a round),
// 16-B aligned.
__host__ __device__ __forceinline__ size_t rows_smem_per_warp(int rw_max) {
  const size_t b = (size_t)rw_max * 8 + (size_t)((rw_max + 31) / 32) * 8 + (size_t)rw_max * 6;
  return (b + 15) & ~(size_t)15;
}

// Dynamic shared memory per warp: RWmax cells + RWmax/32 pending words + RWmax list.
__global__ void __launch_bounds__(256, 4) k_rows(Ctx* ctxs, int nctx, DevGraph G, int split,
                                              int rw_max) {
  __shared__ uint32_t s_pref[MAXB + 1];
  extern __shared__ __align__(16) unsigned char s_dyn[];
  load_prefix(ctxs, nctx, s_pref, -1);
  const uint32_t total = s_pref[nctx];
  const int lane = threadIdx.x & 31;
  const int wib = threadIdx.x >> 5;
  const size_t per_warp = rows_smem_per_warp(rw_max);
  unsigned char* wbase = s_dyn + per_warp * wib;
  unsigned long long* buf = (unsigned long long*)wbase;
  uint32_t* pend = (uint32_t*)(wbase + (size_t)rw_max * 8);
  uint32_t* done = pend + (rw_max + 31) / 32;
  uint16_t* plist = (uint16_t*)(done + (rw_max + 31) / 32);
  uint16_t* flist = plist + rw_max;
  uint16_t* clist = flist + rw_max;
  uint16_t* list = plist;  // reused for the tour-bound candidates after the closure
  const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
  const uint32_t wid = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  int st_q = -1;
  unsigned long long st_merges = 0, st_rows = 0;
  for (uint32_t it = wid; it < total; it += warps) {
    uint32_t merges = 0;
    const int qi = find_ctx(s_pref, nctx, it);
    Ctx* c = ctxs + qi;
    const uint32_t v = c->rows[it - s_pref[qi]];
    if (!in_bounds(c, v < G.V && c->RW <= rw_max, 8)) continue;
    const int RW = c->RW, W = c->W, DD = c->DD, k = c->k, D = c->D, hop = c->hop;
    (void)W;
    // cell i sits at i ^ ((i >> 4) & swz) in shared memory: the partners of a merge round
    // (submasks of one complement, cells of one popcount class) often share their low
    // index bits, and the XOR spreads them over the banks; a row whose width is not a
    // multiple of 16 cells stays unswizzled (its positions must stay below RW)
    const uint32_t swz = (RW & 15) ? 0u : 15u;
    auto B = [&](uint32_t i) -> unsigned long long& { return buf[i ^ ((i >> 4) & swz)]; };
    const uint32_t full = (uint32_t)c->full;
    unsigned long long* row = (unsigned long long*)row_of(c, v);
    if (row == nullptr) {  // never for a dirty row: a row is taken before its first write
      if (lane == 0) {
        atomicAnd(&c->rowbits[v >> 5], ~(1u << (v & 31)));
        atomicOr(&c->error, (uint32_t)ERR_BOUNDS);
      }
      continue;
    }
    // load the row; list its pending cells (plist) and its finite cells (flist)
    int np = 0, nf = 0;
    for (int i0 = 0; i0 < RW; i0 += 32) {
      const int i = i0 + lane;
      uint64_t x = CELL_INF;
      if (i < RW) {
        x = __ldcg(row + i);
        B((uint32_t)i) = x;
      }
      // an unreached cell is all ones, so its pending bit must be ignored
      const bool fin = i < RW && x != CELL_INF;
      const bool pn = fin && ((uint32_t)x & PEND);
      const bool fl = fin && ((uint32_t)i & full) != 0u;
      const uint32_t bp = __ballot_sync(0xffffffffu, pn);
      const uint32_t bf = __ballot_sync(0xffffffffu, fl);
      const uint32_t lt = (1u << lane) - 1u;
      if (pn) plist[np + __popc(bp & lt)] = (uint16_t)i;
      if (fl) flist[nf + __popc(bf & lt)] = (uint16_t)i;
      np += __popc(bp);
      nf += __popc(bf);
      if (lane == 0) {
        pend[i0 >> 5] = bp;
        done[i0 >> 5] = 0u;
      }
    }
    if (lane == 0) atomicAnd(&c->rowbits[v >> 5], ~(1u << (v & 31)));
    __syncwarp();
    const uint32_t ubm = hop ? c->ub_cell : c->ub;
    // Merge closure T(v, X|Y) <= T(v, X) + T(v, Y), by rounds of popcount class: in a
    // round the unprocessed pending cells X of the smallest class (clist) are merged
    // with every finite cell Y disjoint from them, all pairs of the round spread
    // over the lanes (partners from flist, or the submasks of ~X when flist is the
    // longer).  Merges only create cells of a larger class, so a cell is final when
    // its round comes; the cells a round creates or improves join plist (and flist).
    for (;;) {
      uint32_t mc = 0xFFFFFFFFu;
      for (int t = lane; t < np; t += 32) {
        const uint32_t cc = plist[t];
        if (!((done[cc >> 5] >> (cc & 31)) & 1u)) mc = min(mc, (uint32_t)__popc(cc & full));
      }
      mc = __reduce_min_sync(0xffffffffu, mc);
      if (mc >= (uint32_t)k) break;  // nothing left below the full set
      int nl = 0;
      for (int t0 = 0; t0 < np; t0 += 32) {
        const int t = t0 + lane;
        uint32_t cc = 0;
        bool sel = false;
        if (t < np) {
          cc = plist[t];
          sel = !((done[cc >> 5] >> (cc & 31)) & 1u) && (uint32_t)__popc(cc & full) == mc;
        }
        const uint32_t bs = __ballot_sync(0xffffffffu, sel);
        if (sel) clist[nl + __popc(bs & ((1u << lane) - 1u))] = (uint16_t)cc;
        nl += __popc(bs);
      }
      __syncwarp();
      for (int t = lane; t < nl; t += 32) {
        const uint32_t cc = clist[t];
        atomicOr(&done[cc >> 5], 1u << (cc & 31));
      }
      const uint32_t m = (1u << (k - (int)mc)) - 1u;  // non-empty submasks of ~X
      const bool scan_f = (uint32_t)nf <= m * (uint32_t)DD;
      const uint32_t per = scan_f ? (uint32_t)nf : m * (uint32_t)DD;
      const uint32_t tp = (uint32_t)nl * per;
      merges += tp;
      const float inv_per = 1.0f / (float)max(per, 1u);
      const float inv_m = 1.0f / (float)m;
      __syncwarp();
      for (uint32_t t0 = 0; t0 < tp; t0 += 32) {
        const uint32_t t = t0 + lane;
        bool newp = false, newf = false;
        uint32_t tgt = 0;
        if (t < tp) {
          const uint32_t a = udiv_small(t, per, inv_per), r = t - a * per;
          const uint32_t cell = clist[a];
          const uint32_t X = cell & full, d1 = cell >> k;
          uint32_t Y, d2;
          if (scan_f) {
            const uint32_t yc = flist[r];
            Y = yc & full;
            d2 = yc >> k;
          } else {
            // r = d2 * m + (yb - 1): partner hop d2, partner = yb-th submask of ~X
            d2 = udiv_small(r, m, inv_m);
            Y = __ldg(&SUBMASK.v[full ^ X][r - d2 * m + 1u]);
          }
          const uint32_t yi = (d2 << k) + Y;
          const uint32_t cy = (Y & X) ? COST_INF : cost_of(B(yi));
          const uint32_t S = X | Y;
          const uint32_t cand = cost_of(B(cell)) + cy;
          bool ok = cy != COST_INF && !(hop && (int)(d1 + d2) > D) &&
                    in_bounds(c, yi < (uint32_t)RW && S < (uint32_t)W, 9);
          if (ok && S != full && 3ull * cand > 2ull * ubm) ok = false;
          if (ok) {
            const uint32_t nd = d1 > d2 ? d1 : d2;
            tgt = (nd << k) + S;
            const uint64_t nv = pack_cell(cand, PEND | MERGE | Y | (d2 << 16) | (d1 << 21));
            if (nv < B(tgt)) {
              const uint64_t old = atomicMin(&B(tgt), (unsigned long long)nv);
              if (nv < old) {
                newf = old == CELL_INF;
                const uint32_t bit = 1u << (tgt & 31);
                newp = !(atomicOr(&pend[tgt >> 5], bit) & bit);
              }
            }
          }
        }
        // cells this step made pending or finite join the lists
        const uint32_t bp = __ballot_sync(0xffffffffu, newp);
        const uint32_t bf = __ballot_sync(0xffffffffu, newf);
        const uint32_t lt = (1u << lane) - 1u;
        if (newp) plist[np + __popc(bp & lt)] = (uint16_t)tgt;
        if (newf) flist[nf + __popc(bf & lt)] = (uint16_t)tgt;
        np += __popc(bp);
        nf += __popc(bf);
      }
      __syncwarp();
    }
    // one-label distances of v: dv as stored (path lengths, for the one-label upper
    // bound); hb the lower bounds of the pruning tests, clamped to cut + 1.  For a
    // hop-bounded query lane L < D + 1 holds the bounds of a state of height L, the
    // distances within the hop budget D - L; the tests take the row of their state's
    // height from that lane.
    uint32_t dv[KMAX], hb[KMAX];
    uint32_t lim = COST_INF;
#pragma unroll
    for (int i = 0; i < KMAX; i++) dv[i] = hb[i] = COST_INF;
    const bool budgets = c->use_lb && hop && c->sssp_hops;
    if (c->use_lb) {
      const uint32_t mine = lane < k ? __ldcg(&c->dist[(uint64_t)v * c->ds + lane]) : COST_INF;
      const uint32_t cut = c->cut;
      lim = cut == COST_INF ? COST_INF : cut + 1u;
#pragma unroll
      for (int i = 0; i < KMAX; i++) {
        dv[i] = __shfl_sync(0xffffffffu, mine, i);
        hb[i] = min(dv[i], lim);
      }
      if (budgets) {
        uint4 a, b;
        budget_row(c, G.V, v, D - min(lane, D), a, b);
        const uint32_t e[8] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w};
#pragma unroll
        for (int i = 0; i < KMAX; i++) hb[i] = min(e[i], lim);
      }
    }
    const int64_t deg = G.beg[v + 1] - G.beg[v];
    const int use_tour = c->use_tour;
    // settle changed states (lane-parallel): write them back, update the full-set
    // bounds, and apply the one-label and hop tests.  pend keeps the states that
    // pass; those that still need the tour bound are listed for the warp below.
    int ncand = 0;
    for (int i0 = 0; i0 < RW; i0 += 32) {
      const int i = i0 + lane;
      bool keep = false, cand = false;
      uint32_t dl[KMAX];
      if (budgets) {
        const int src = (i < RW ? i : 0) >> k;  // the lane holding this height's bounds
#pragma unroll
        for (int b = 0; b < KMAX; b++) dl[b] = __shfl_sync(0xffffffffu, hb[b], src);
      } else {
#pragma unroll
        for (int b = 0; b < KMAX; b++) dl[b] = hb[b];
      }
      if (i < RW && ((pend[i >> 5] >> (i & 31)) & 1u)) {
        const uint64_t x = B((uint32_t)i);
        row[i] = x & ~(uint64_t)PEND;
        const uint32_t cst = cost_of(x);
        const uint32_t p = (uint32_t)i & full, d = (uint32_t)i >> k;
        if (p == full) {
          atomicMin(&c->best, ((unsigned long long)cst << 32) | ((unsigned long long)d << 27) | v);
          atomicMin(&c->ub_cell, cst);
          atomicMin(&c->ub, cst);
        } else {
          uint32_t lb = 0;
          uint64_t one = cst;
          if (c->use_lb) {
#pragma unroll
            for (int b = 0; b < KMAX; b++)
              if (b < k && !((p >> b) & 1u)) {
                lb = max(lb, dl[b]);
                one += dv[b];
              }
            if (!hop && one < (uint64_t)c->ub) atomicMin(&c->ub, (uint32_t)one);
          }
          const uint32_t bound = hop ? c->ub_cell : c->ub;
          bool grow = 2ull * cst <= (uint64_t)bound && (uint64_t)cst + lb <= (uint64_t)bound;
          if (hop) grow = grow && (int)d < D && cst < bound;
          if (grow && deg > 0) {
            keep = true;
            cand = use_tour != 0;
          }
        }
      }
      const uint32_t bk = __ballot_sync(0xffffffffu, keep);
      const uint32_t bc = __ballot_sync(0xffffffffu, cand);
      if (cand) list[ncand + __popc(bc & ((1u << lane) - 1u))] = (uint16_t)i;
      ncand += __popc(bc);
      if (lane == 0) pend[i0 >> 5] = bk;
    }
    __syncwarp();
    if (ncand > 0) {
      // tour bound of PrunedDP++ (code/PrunedDP++/include/CPUNONHOP.h:433-493): the
      // rest of the tree, doubled, is a closed walk from v through every group of
      // Xb = full \ p, so twice its cost is at least
      //   lb2 = max_a d_a(v) + min_b P(a,b,Xb) + min_b d_b(v)    and
      //   lb1 = min_{a,b} d_a(v) + P(a,b,Xb) + d_b(v),
      // P = cheapest group sequence from a to b visiting each group of Xb once.
      // One candidate per lane: the O(k) bound first, the O(k^2) one for the
      // candidates it keeps (the test is cost + ceil(max(lb1, lb2) / 2) > bound).
      const uint32_t bound = hop ? __ldcg(&c->ub_cell) : __ldcg(&c->ub);
      const uint32_t* tour = c->tour;
      const uint32_t Wq = (uint32_t)c->W;
      for (int t0 = 0; t0 < ncand; t0 += 32) {
        const int t = t0 + lane;
        uint32_t dl[KMAX];
        if (budgets) {
          const int src = t < ncand ? (int)(list[t] >> k) : 0;
#pragma unroll
          for (int b = 0; b < KMAX; b++) dl[b] = __shfl_sync(0xffffffffu, hb[b], src);
        } else {
#pragma unroll
          for (int b = 0; b < KMAX; b++) dl[b] = hb[b];
        }
        if (t < ncand) {
          const uint32_t i = list[t];
          const uint32_t p = i & full, cst = cost_of(B(i));
          const uint32_t Xb = full ^ p;
          const uint32_t* W2 = tour + (size_t)Wq * TOUR_STRIDE + (size_t)Xb * KMAX;
          uint32_t mind = COST_INF;
#pragma unroll
          for (int b2 = 0; b2 < KMAX; b2++)
            if (b2 < k && ((Xb >> b2) & 1u)) mind = min(mind, dl[b2]);
          uint64_t lb2 = 0;
#pragma unroll
          for (int b2 = 0; b2 < KMAX; b2++)
            if (b2 < k && ((Xb >> b2) & 1u)) {
              const uint64_t t2 = (uint64_t)dl[b2] + __ldg(&W2[b2]) + mind;
              lb2 = t2 > lb2 ? t2 : lb2;
            }
          // both bounds saturate at COST_INF (an unreachable group)
          lb2 = lb2 < COST_INF ? lb2 : COST_INF;
          bool drop = (uint64_t)cst + (lb2 + 1) / 2 > (uint64_t)bound;
          if (!drop) {
            const uint32_t* Wt = tour + (size_t)Xb * TOUR_STRIDE;
            uint64_t lb1 = ~0ull;
#pragma unroll
            for (int a1 = 0; a1 < KMAX; a1++)
              if (a1 < k && ((Xb >> a1) & 1u)) {
#pragma unroll
                for (int b1 = 0; b1 < KMAX; b1++)
                  if (b1 < k && ((Xb >> b1) & 1u)) {
                    const uint64_t t1 =
                        (uint64_t)dl[a1] + __ldg(&Wt[a1 * KMAX + b1]) + dl[b1];
                    lb1 = t1 < lb1 ? t1 : lb1;
                  }
              }
            lb1 = lb1 < COST_INF ? lb1 : COST_INF;
            drop = (uint64_t)cst + (lb1 + 1) / 2 > (uint64_t)bound;
          }
          if (drop) atomicAnd(&pend[i >> 5], ~(1u << (i & 31)));
        }
      }
      __syncwarp();
    }
    // emit the growing states, each relaxed from its lightest edge on (which lands
    // at cst + 1 or later): one reservation per list for the whole row
    {
      const uint32_t bend = c->bucket_end;
      uint32_t cn = 0, cf = 0, kmin = COST_INF;
      for (int i0 = 0; i0 < RW; i0 += 32) {
        const int i = i0 + lane;
        if (i < RW && ((pend[i >> 5] >> (i & 31)) & 1u)) {
          const uint32_t key = cost_of(B(i)) + 1u;
          if (key >= bend) {
            cf++;
            kmin = min(kmin, key);
          } else {
            cn++;
          }
        }
      }
      const uint32_t sn = warp_incl_scan(cn), sf = warp_incl_scan(cf);
      const uint32_t tn = __shfl_sync(0xffffffffu, sn, 31), tf = __shfl_sync(0xffffffffu, sf, 31);
      kmin = __reduce_min_sync(0xffffffffu, kmin);
      if (tn + tf > 0) {
        uint32_t bn = 0, bfr = 0;
        if (lane == 0) {
          if (tn) bn = atomicAdd(&c->n_q[c->no], tn);
          if (tf) {
            bfr = atomicAdd(&c->n_far[c->f], tf);
            atomicMin(&c->far_min, kmin);
          }
        }
        bn = __shfl_sync(0xffffffffu, bn, 0) + sn - cn;
        bfr = __shfl_sync(0xffffffffu, bfr, 0) + sf - cf;
        uint4* nl = c->q[c->no];
        uint4* fl = c->far[c->f];
        for (int i0 = 0; i0 < RW; i0 += 32) {
          const int i = i0 + lane;
          if (i < RW && ((pend[i >> 5] >> (i & 31)) & 1u)) {
            const uint32_t cst = cost_of(B(i));
            const uint32_t p = (uint32_t)i & full, d = (uint32_t)i >> k;
            const uint4 item = make_uint4(v, p | (d << 16), cst, 0u);
            if (cst + 1u >= bend) {
              if (bfr < c->farcap) fl[bfr] = item;
              else atomicOr(&c->error, (uint32_t)ERR_FARCAP);
              bfr++;
            } else {
              if (bn < c->qcap) nl[bn] = item;
              else atomicOr(&c->error, (uint32_t)ERR_QCAP);
              bn++;
            }
          }
        }
      }
    }
    // statistics: one atomic per query change of the warp, not per row
    if (qi != st_q) {
      if (st_q >= 0 && lane == 0) {
        atomicAdd(&ctxs[st_q].st_merge, (unsigned long long)st_merges);
        atomicAdd(&ctxs[st_q].st_rows, (unsigned long long)st_rows);
      }
      st_q = qi;
      st_merges = 0;
      st_rows = 0;
    }
    st_merges += merges;
    st_rows += 1;
    __syncwarp();
  }
  if (st_q >= 0 && lane == 0) {
    atomicAdd(&ctxs[st_q].st_merge, (unsigned long long)st_merges);
    atomicAdd(&ctxs[st_q].st_rows, (unsigned long long)st_rows);
  }
}

// ---- control: one thread per query -------------------------------------------------
__device__ __forceinline__ void ctrl_take_far(Ctx* c) {
  // advance the cost bucket and take the far list as the next input
  const uint32_t fm = c->far_min;
  c->bucket_end = (c->delta == 0) ? 0xFFFFFFFFu
                                  : (uint32_t)min((uint64_t)fm + c->delta, (uint64_t)0xFFFFFFFFu);
  c->in_ptr = c->far[c->f];
  c->in_n = min(c->n_far[c->f], c->farcap);
  c->in_kind = 1;
  c->in_idx = c->f;
  c->f ^= 1u;
  c->n_far[c->f] = 0;
  c->far_min = 0xFFFFFFFFu;
}

// Tour table of one query (all threads of the block): P[X][i][j] = cheapest
// sequence of group-to-group hops that starts in group i, ends in group j and
// visits every group of X exactly once (Held-Karp over the vv distances), then the
// row minima P2[X][i] = min_j P[X][i][j].  The reference builds a closure of the
// same table on the host (code/TrimCDP-WB/src/GSTnonHop.cu:355-404,
// code/PrunedDP++/include/CPUNONHOP.h:266-383 and :564-586).
__device__ void build_tour(Ctx* c) {
  const int k = c->k, W = c->W;
  uint32_t* P = c->tour;
  for (int L = 1; L <= k; L++) {
    for (int idx = threadIdx.x; idx < W * k; idx += blockDim.x) {
      const uint32_t X = (uint32_t)(idx / k);
      const int i = idx - (int)X * k;
      if (__popc(X) != L || !((X >> i) & 1u)) continue;
      for (int p = 0; p < k; p++) {
        if (!((X >> p) & 1u)) continue;
        uint32_t val = COST_INF;
        if (L == 1) {
          val = 0u;  // X == {i}, p == i
        } else if (p != i) {
          const uint32_t prev = X ^ (1u << p);
          for (int j = 0; j < k; j++) {
            if (!((prev >> j) & 1u)) continue;
            const uint64_t x = (uint64_t)P[(size_t)prev * TOUR_STRIDE + i * KMAX + j] +
                               c->vv[j * KMAX + p];
            if (x < val) val = (uint32_t)x;
          }
        }
        P[(size_t)X * TOUR_STRIDE + i * KMAX + p] = val;
      }
    }
    __syncthreads();
  }
  uint32_t* P2 = P + (size_t)W * TOUR_STRIDE;
  for (int idx = threadIdx.x; idx < W * k; idx += blockDim.x) {
    const uint32_t X = (uint32_t)(idx / k);
    const int i = idx - (int)X * k;
    uint32_t m = COST_INF;
    if ((X >> i) & 1u)
      for (int p = 0; p < k; p++)
        if ((X >> p) & 1u) m = min(m, P[(size_t)X * TOUR_STRIDE + i * KMAX + p]);
    P2[(size_t)X * KMAX + i] = m;
  }
}

// DP start: the first step of the DP is the rows kernel over the seeded rows.
__device__ __forceinline__ void ctrl_start_dp(Ctx* c) {
  c->phase = PH_DP;
  c->in_n = 0;
  c->no = 0;
  c->n_q[0] = c->n_q[1] = 0;
  c->n_far[0] = c->n_far[1] = 0;
  c->far_min = 0xFFFFFFFFu;
  c->bucket_end = c->delta ? c->delta : 0xFFFFFFFFu;
}

// One block per query context; thread 0 runs the control logic, the whole block
// builds the tour table when a query leaves its distance phase.
__global__ void k_ctrl(Ctx* ctxs, int nctx, int mode) {
  const int qi = blockIdx.x;
  if (qi >= nctx) return;
  Ctx* c = ctxs + qi;
  if (mode == CTRL_SSSP && c->phase == PH_PREP && !c->error && c->dist_only) {
    // a group-cache fill: its distances are final, nothing else to build
    if (threadIdx.x == 0) {
      c->phase = PH_DONE;
      c->in_n = 0;
    }
    return;
  }
  if (mode == CTRL_SSSP && c->phase == PH_PREP && !c->error) {
    // The distances are final up to the cutoff ub: every stored distance <= ub is
    // exact, and any other is only known to be > ub.  The group distances feed a
    // lower bound, so they are clamped to ub + 1, a value never above the truth.
    const uint32_t cut = sssp_cutoff(c);
    const uint32_t lim = cut == COST_INF ? COST_INF : cut + 1u;
    for (int i = threadIdx.x; i < KMAX * KMAX; i += blockDim.x) c->vv[i] = min(c->vv[i], lim);
    __syncthreads();
    if (c->use_tour) build_tour(c);  // block-uniform branch
    if (threadIdx.x == 0) {
      c->cut = cut;
      ctrl_start_dp(c);
    }
    return;
  }
  if (threadIdx.x != 0) return;
  if (c->phase >= PH_DONE) return;
  if (c->error) {
    c->phase = PH_ERROR;
    c->in_n = 0;
    return;
  }
  if (mode == CTRL_SSSP) {
    if (c->phase != PH_SSSP) return;
    if (++c->levels > c->max_levels) {
      c->error |= ERR_TIMEOUT;
      c->phase = PH_ERROR;
      c->in_n = 0;
      return;
    }
    // the finished step read in_ptr and pushed near items into q[no]
    if (c->in_kind == 0) c->n_q[c->in_idx] = 0;
    else c->n_far[c->in_idx] = 0;
    const uint32_t s = c->no;
    c->st_qmax = max(c->st_qmax, max(c->n_q[s], c->n_far[c->f]));
    if (c->n_q[s] > 0) {
      c->in_ptr = c->q[s];
      c->in_n = min(c->n_q[s], c->qcap);
      c->in_kind = 0;
      c->in_idx = s;
      c->no = s ^ 1u;
    } else if (c->n_far[c->f] > 0) {
      ctrl_take_far(c);
      c->no = s;
    } else {
      // distances final: the next k_sssp launch builds the bounds (PH_PREP), the
      // control step after it the tour table, then the DP starts
      c->phase = PH_PREP;
      c->in_n = 0;
    }
  } else if (mode == CTRL_DP_ROWS) {
    // the rows kernel appended the grow items of the states it settled to q[no]
    // (after the continuations the last grow step appended there)
    if (c->phase != PH_DP) return;
    c->n_rows = 0;  // consumed by the rows kernel
    const uint32_t s = c->no;
    c->st_qmax = max(c->st_qmax, max(c->n_q[s], c->n_far[c->f]));
    if (c->n_q[s] > 0) {
      c->in_ptr = c->q[s];
      c->in_n = min(c->n_q[s], c->qcap);
      c->in_kind = 0;
      c->in_idx = s;
      c->no = s ^ 1u;
    } else if (c->n_far[c->f] > 0) {
      ctrl_take_far(c);
    } else {
      c->phase = PH_DONE;
      c->in_n = 0;
    }
  } else {  // CTRL_DP_GROW
    if (c->phase != PH_DP) return;
    if (++c->levels > c->max_levels) {
      c->error |= ERR_TIMEOUT;
      c->phase = PH_ERROR;
      c->in_n = 0;
      return;
    }
    if (c->in_kind == 0) c->n_q[c->in_idx] = 0;
    else c->n_far[c->in_idx] = 0;
    c->in_n = 0;
  }
}

// ---- device-side loop control of the level graph -----------------------------------
// Last node of the level body of the CUDA graph's WHILE loop: go on while no
// resident query has finished, some query is resident and iterations are left.
// loop[0] = iterations left (host-set before the launch), loop[1] = a query finished.
__global__ void k_loop_cond(const Ctx* ctxs, int nctx, uint32_t* loop,
                            cudaGraphConditionalHandle h) {
  const int i = threadIdx.x;  // blockDim.x >= MAXB
  bool fin = false, act = false;
  if (i < nctx) {
    const Ctx* c = ctxs + i;
    if (!c->idle) {
      act = true;
      fin = c->phase >= PH_DONE;
    }
  }
  const int any_fin = __syncthreads_or(fin);
  const int any_act = __syncthreads_or(act);
  if (i == 0) {
    const uint32_t left = loop[0] > 0 ? loop[0] - 1u : 0u;
    loop[0] = left;
    loop[1] = any_fin ? 1u : 0u;
    cudaGraphSetConditional(h, (!any_fin && any_act && left > 0) ? 1u : 0u);
  }
}

// ---- tree extraction: parent walk from the best full-set state --------------------
__device__ int32_t edge_weight_dev(const DevGraph& G, uint32_t v, uint32_t u) {
  int64_t lo = G.beg[v], hi = G.beg[v + 1];
  while (lo < hi) {
    const int64_t mid = (lo + hi) >> 1;
    if ((uint32_t)G.edges[mid].x < u) lo = mid + 1;
    else hi = mid;
  }
  int32_t w = -1;
  for (int64_t i = lo; i < G.beg[v + 1] && (uint32_t)G.edges[i].x == u; i++)
    if (w < 0 || G.edges[i].y < w) w = G.edges[i].y;
  return w;
}

__global__ void k_extract(Ctx* ctxs, int nctx, DevGraph G) {
  const int qi = blockIdx.x * blockDim.x + threadIdx.x;
  if (qi >= nctx) return;
  Ctx* c = ctxs + qi;
  c->n_out = 0;
  if (c->phase != PH_DONE || c->best == ~0ull) return;
  const uint32_t v0 = (uint32_t)(c->best & 0x7FFFFFFull);
  const uint32_t d0 = (uint32_t)((c->best >> 27) & 31u);
  const uint64_t RW = (uint64_t)c->RW;
  const uint32_t DD = (uint32_t)c->DD;
  const int k = c->k;
  uint32_t sp = 0, nout = 0, steps = 0;
  c->stack[sp++] = (uint64_t)v0 * RW + ((uint64_t)d0 << k) + (uint64_t)c->full;
  while (sp > 0) {
    if (++steps > 4u * c->stackcap) {
      c->error |= ERR_EXTRACT;
      break;
    }
    const uint64_t idx = c->stack[--sp];
    if (!in_bounds(c, idx < (uint64_t)G.V * RW, 10)) break;
    const uint32_t v = (uint32_t)(idx / RW);
    const uint32_t r = (uint32_t)(idx - (uint64_t)v * RW);
    const uint32_t p = r & (uint32_t)c->full, d = r >> k;
    const uint64_t* vrow = row_of(c, v);
    const uint64_t cell = vrow ? vrow[r] : CELL_INF;
    const uint32_t par = (uint32_t)cell & ~PEND;
    if (cost_of(cell) == COST_INF) {  // a parent pointer never leads to an unreached state
      c->error |= ERR_EXTRACT;
      break;
    }
    if (par == LEAF) continue;
    if (!(par & MERGE)) {
      const uint32_t u = par;
      if (u >= G.V || (c->hop && d == 0)) {
        c->error |= ERR_EXTRACT;
        break;
      }
      if (nout < c->outcap) {
        c->out[3 * nout + 0] = (int32_t)u;
        c->out[3 * nout + 1] = (int32_t)v;
        c->out[3 * nout + 2] = edge_weight_dev(G, v, u);
      }
      nout++;
      if (sp + 1 > c->stackcap) {
        c->error |= ERR_EXTRACT;
        break;
      }
      c->stack[sp++] = (uint64_t)u * RW + ((uint64_t)(d - (uint32_t)c->hop) << k) + p;
    } else {
      const uint32_t Y = par & 0xFFFFu, d2 = (par >> 16) & 31u, d1 = (par >> 21) & 31u;
      const uint32_t X = p ^ Y;
      if (Y == 0 || (Y & ~p) != 0 || X == 0 || d1 >= DD || d2 >= DD) {
        c->error |= ERR_EXTRACT;
        break;
      }
      if (sp + 2 > c->stackcap) {
        c->error |= ERR_EXTRACT;
        break;
      }
      c->stack[sp++] = (uint64_t)v * RW + ((uint64_t)d1 << k) + X;
      c->stack[sp++] = (uint64_t)v * RW + ((uint64_t)d2 << k) + Y;
    }
  }
  if (nout > c->outcap) c->error |= ERR_EXTRACT;
  c->n_out = nout;
}

}  // namespace gst
