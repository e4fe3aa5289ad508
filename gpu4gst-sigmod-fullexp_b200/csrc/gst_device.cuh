// Device side of the GST engine: state layout, worklists and the level kernels.
//
// State table.  One query owns a slab of V rows; row v holds the 2^k x (D+1)
// states (v, p, d) of that vertex (d only for hop-bounded queries) as packed
// 64-bit cells
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
// Pruning (all safe with ub >= optimum; see the engine's design notes):
//   grow a state only if 2c <= ub (code/TrimCDP-WB/include/mapper_enactor.cuh /
//   reducer.cuh:317-433 use c-1 <= best/2); keep a merged non-full state only if
//   3c <= 2ub (PrunedDP++ CPUNONHOP.h:913 uses 0.667*best+2); drop a state if
//   c + max_{i not in X} dist_i(v) > ub (one-label bound, get_lb mapper.cuh:163-191).
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
constexpr int DIST_STRIDE = 8;    // int32 one-label distances per vertex row

// PH_PREP: distances final; the star bound, group distances and tour table are
// being built (one k_sssp pass over the distance rows, then the control block).
enum Phase : uint32_t { PH_SSSP = 0, PH_PREP = 1, PH_DP = 2, PH_DONE = 3, PH_ERROR = 4 };
enum ErrBits : uint32_t { ERR_QCAP = 1, ERR_FARCAP = 2, ERR_ROWCAP = 4, ERR_TIMEOUT = 8,
                          ERR_EXTRACT = 16, ERR_BOUNDS = 32 };
enum CtrlMode : int { CTRL_SSSP = 0, CTRL_DP_ROWS = 1, CTRL_DP_GROW = 2 };

constexpr int WIDX = 8;            // light-edge index: counts of edges with w <= 2^j, j < 8
constexpr int TOUR_STRIDE = KMAX * KMAX;

struct DevGraph {
  int64_t V;
  int64_t E;
  const int64_t* beg;     // V+1
  const int2* edges;      // E x {neighbour, weight}, sorted by neighbour per vertex
  const int2* wedges;     // the same edges sorted by (weight, neighbour) per vertex
  const uint32_t* widx;   // V x WIDX: edges of v with weight <= 2^j (NULL: no index,
                          // wedges then need not be weight-sorted)
};

// Number of leading entries of v's weight-sorted edge list that can hold an edge
// of weight <= lim (an over-count by at most the edges in (lim, 2^j]).
__device__ __forceinline__ int64_t light_count(const DevGraph& G, uint32_t v, int64_t deg,
                                               uint32_t lim) {
  if (lim == 0u) return 0;
  if (!G.widx || lim > (1u << (WIDX - 1))) return deg;
  const int j = 32 - __clz(lim - 1u);  // smallest j with 2^j >= lim
  return (int64_t)__ldg(&G.widx[(uint64_t)v * WIDX + j]);
}

// Per-query context.  Fields above `in_ptr` are written by the host before the
// query starts; the rest are updated by the control kernel between launches and
// by atomics inside the level kernels.
struct Ctx {
  uint64_t* table;
  uint32_t* dist;
  uint32_t* rowbits;
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
  uint32_t ub_cell;     // best full-state cell
  unsigned long long best;  // cost<<32 | d<<27 | v of the best full-state cell
  uint32_t phase;
  uint32_t error;
  uint32_t levels;
  uint32_t n_out;
  uint32_t bad_site;    // checked builds: first failed bounds check (site id)
  unsigned long long st_items, st_relax, st_merge, st_rows, st_sssp;
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

__device__ __forceinline__ uint32_t cost_of(uint64_t c) { return (uint32_t)(c >> 32); }
__device__ __forceinline__ uint64_t pack_cell(uint32_t cost, uint32_t low) {
  return ((uint64_t)cost << 32) | low;
}

// b-th (1-based) non-empty submask of `mask`, bits of b deposited into mask's bits.
__device__ __forceinline__ uint32_t deposit(uint32_t b, uint32_t mask) {
  uint32_t r = 0;
  while (mask) {
    const uint32_t low = mask & (0u - mask);
    if (b & 1u) r |= low;
    b >>= 1;
    mask ^= low;
  }
  return r;
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

// ---- worklist pushes ---------------------------------------------------------
__device__ __forceinline__ void push_near(Ctx* c, const uint4& e) {
  const uint32_t i = atomicAdd(&c->n_q[c->no], 1u);
  if (i < c->qcap) c->q[c->no][i] = e;
  else atomicOr(&c->error, (uint32_t)ERR_QCAP);
}
__device__ __forceinline__ void push_far(Ctx* c, const uint4& e) {
  const uint32_t i = atomicAdd(&c->n_far[c->f], 1u);
  if (i < c->farcap) c->far[c->f][i] = e;
  else atomicOr(&c->error, (uint32_t)ERR_FARCAP);
  atomicMin(&c->far_min, e.z);
}
// Emit the work items of state (v, pd) with cost `cost`: one per `split` edges of
// the first `cnt` entries of v's edge list.
__device__ __forceinline__ void push_state(Ctx* c, uint32_t v, uint32_t pd, uint32_t cost,
                                           int64_t cnt, int split, uint32_t bucket_end) {
  const uint32_t nch = (uint32_t)((cnt + split - 1) / split);
  const bool near = cost < bucket_end;
  for (uint32_t ch = 0; ch < nch; ch++) {
    const uint4 e = make_uint4(v, pd, cost, ch);
    if (near) push_near(c, e);
    else push_far(c, e);
  }
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

// Per-CTA prefix of the input counts of all queries of the launch.
// want: PH_SSSP (sssp input), PH_DP (grow input) or -1 (rows of DP-phase queries).
__device__ __forceinline__ void load_prefix(Ctx* ctxs, int nctx, uint32_t* s_pref, int want) {
  if (threadIdx.x == 0) {
    uint32_t acc = 0;
    s_pref[0] = 0;
    for (int i = 0; i < nctx; i++) {
      const Ctx* c = ctxs + i;
      uint32_t n = 0;
      if (want < 0) n = (c->phase == PH_DP) ? min(c->n_rows, c->rowcap) : 0u;
      else n = (c->phase == (uint32_t)want) ? c->in_n : 0u;
      acc += n;
      s_pref[i + 1] = acc;
    }
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
        atomicMin((unsigned long long*)&c->table[(uint64_t)v * c->RW + (uint64_t)(1u << i) * c->DD],
                  (unsigned long long)cell0);
        mark_row(c, v);
        if (c->phase == PH_SSSP) {
          const uint32_t old = atomicMin(&c->dist[(uint64_t)v * DIST_STRIDE + i], 0u);
          if (old != 0u) {
            const int64_t deg = G.beg[v + 1] - G.beg[v];
            push_state(c, v, (uint32_t)i, 0u, deg, split, 0xFFFFFFFFu);
          }
        }
      }
    }
  }
}

// ---- one-label SSSP step: multi-source Bellman-Ford with near/far ordering ----
// Work item {v, group index i, dist, chunk}: relax dist_i(u) for u in the chunk.
// (code/TrimCDP-WB/include/mapper_enactor.cuh:249-366 computes the same
// distances as grow-only DP states (v, 1<<i).)
__global__ void __launch_bounds__(256) k_sssp(Ctx* ctxs, int nctx, DevGraph G, int split) {
  __shared__ uint32_t s_pref[MAXB + 1];
  load_prefix(ctxs, nctx, s_pref, PH_SSSP);
  const uint32_t total = s_pref[nctx];
  const int lane = threadIdx.x & 31;
  const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
  const uint32_t wid = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  for (uint32_t base = wid * 32; base < total; base += warps * 32) {
    const uint32_t it = base + lane;
    uint32_t n = 0, v = 0, gi = 0, cost = 0;
    int64_t eb = 0;
    int qi = 0;
    if (it < total) {
      qi = find_ctx(s_pref, nctx, it);
      Ctx* c = ctxs + qi;
      const uint4 e = c->in_ptr[it - s_pref[qi]];
      v = e.x;
      gi = e.y;
      cost = e.z;
      if (!in_bounds(c, v < G.V && gi < (uint32_t)c->k, 2)) { v = 0; gi = 0; cost = 0xFFFFFFFFu; }
      const uint32_t cur = __ldcg(&c->dist[(uint64_t)v * DIST_STRIDE + gi]);
      if (cur >= cost) {  // not stale
        if (cost >= c->bucket_end) {
          push_far(c, e);
        } else {
          const int64_t b0 = G.beg[v], b1 = G.beg[v + 1];
          eb = b0 + (int64_t)e.w * split;
          const int64_t ee = min(b1, eb + (int64_t)split);
          n = ee > eb ? (uint32_t)(ee - eb) : 0u;
        }
      }
    }
    add_stat(ctxs, qi, it < total, n, &Ctx::st_sssp);
    const uint32_t scan = warp_incl_scan(n);
    const uint32_t tot = __shfl_sync(0xffffffffu, scan, 31);
    for (uint32_t j0 = 0; j0 < tot; j0 += 32) {
      const uint32_t j = j0 + lane;
      const int o = warp_owner(scan, j < tot ? j : tot - 1);
      const uint32_t o_scan = __shfl_sync(0xffffffffu, scan, o);
      const uint32_t o_n = __shfl_sync(0xffffffffu, n, o);
      const int64_t o_eb = __shfl_sync(0xffffffffu, eb, o);
      const uint32_t o_gi = __shfl_sync(0xffffffffu, gi, o);
      const uint32_t o_cost = __shfl_sync(0xffffffffu, cost, o);
      const int o_qi = __shfl_sync(0xffffffffu, qi, o);
      if (j < tot) {
        const uint32_t off = j - (o_scan - o_n);
        Ctx* c = ctxs + o_qi;
        if (!in_bounds(c, o_eb + off < G.E, 3)) continue;
        const int2 ed = G.wedges[o_eb + off];
        const uint32_t u = (uint32_t)ed.x;
        const uint32_t nd = o_cost + (uint32_t)ed.y;
        if (!in_bounds(c, u < G.V, 4)) continue;
        uint32_t* dp = &c->dist[(uint64_t)u * DIST_STRIDE + o_gi];
        if (nd < __ldcg(dp)) {
          const uint32_t old = atomicMin(dp, nd);
          if (nd < old) {
            const int64_t deg = G.beg[u + 1] - G.beg[u];
            push_state(c, u, o_gi, nd, deg, split, c->bucket_end);
          }
        }
      }
    }
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
    uint32_t best = COST_INF;
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < G.V;
         v += (int64_t)gridDim.x * blockDim.x) {
      const uint4* row = (const uint4*)&c->dist[(uint64_t)v * DIST_STRIDE];
      const uint4 a = __ldcg(row), b = __ldcg(row + 1);
      const uint32_t d[8] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w};
      uint64_t sum = 0;
#pragma unroll
      for (int i = 0; i < KMAX; i++)
        if (i < k) sum += d[i];
      if (sum < best) best = (uint32_t)sum;
#pragma unroll
      for (int i = 0; i < KMAX; i++)
        if (i < k && d[i] == 0u) {
#pragma unroll
          for (int j = 0; j < KMAX; j++)
            if (j < k && d[j] < __ldcg(&c->vv[i * KMAX + j])) atomicMin(&c->vv[i * KMAX + j], d[j]);
        }
    }
    best = __reduce_min_sync(0xffffffffu, best);
    if ((threadIdx.x & 31) == 0 && best < COST_INF && !c->hop && best < __ldcg(&c->ub))
      atomicMin(&c->ub, best);
  }
}

// ---- DP grow step ----------------------------------------------------------------
__global__ void __launch_bounds__(256) k_grow(Ctx* ctxs, int nctx, DevGraph G, int split) {
  __shared__ uint32_t s_pref[MAXB + 1];
  load_prefix(ctxs, nctx, s_pref, PH_DP);
  const uint32_t total = s_pref[nctx];
  const int lane = threadIdx.x & 31;
  const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
  const uint32_t wid = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  for (uint32_t base = wid * 32; base < total; base += warps * 32) {
    const uint32_t it = base + lane;
    uint32_t n = 0, v = 0, pd = 0, cost = 0;
    int64_t eb = 0;
    int qi = 0;
    if (it < total) {
      qi = find_ctx(s_pref, nctx, it);
      Ctx* c = ctxs + qi;
      const uint4 e = c->in_ptr[it - s_pref[qi]];
      v = e.x;
      pd = e.y;
      cost = e.z;
      const uint32_t p = pd & 0xFFFFu, d = pd >> 16;
      const bool ok = in_bounds(c, v < G.V && p < (uint32_t)c->W && d < (uint32_t)c->DD, 5);
      const uint64_t cell = ok ? __ldcg((const unsigned long long*)&c->table[(uint64_t)v * c->RW +
                                                                           (uint64_t)p * c->DD + d])
                               : 0ull;
      const uint32_t bound = c->hop ? c->ub_cell : c->ub;
      // a work item always names a state that holds a finite cost
      const bool src_ok = !ok || in_bounds(c, cost_of(cell) != COST_INF, 12);
      if (ok && src_ok && cost_of(cell) >= cost && 2ull * cost <= (uint64_t)bound) {
        if (cost >= c->bucket_end) {
          push_far(c, e);
        } else {
          const int64_t b0 = G.beg[v], b1 = G.beg[v + 1];
          const int64_t lc = light_count(G, v, b1 - b0, grow_limit(c, cost));
          eb = b0 + (int64_t)e.w * split;
          const int64_t ee = min(b0 + lc, eb + (int64_t)split);
          n = ee > eb ? (uint32_t)(ee - eb) : 0u;
        }
      }
    }
    add_stat(ctxs, qi, it < total, n, &Ctx::st_relax);
    add_stat(ctxs, qi, it < total, n > 0 ? 1u : 0u, &Ctx::st_items);
    const uint32_t scan = warp_incl_scan(n);
    const uint32_t tot = __shfl_sync(0xffffffffu, scan, 31);
    for (uint32_t j0 = 0; j0 < tot; j0 += 32) {
      const uint32_t j = j0 + lane;
      const int o = warp_owner(scan, j < tot ? j : tot - 1);
      const uint32_t o_scan = __shfl_sync(0xffffffffu, scan, o);
      const uint32_t o_n = __shfl_sync(0xffffffffu, n, o);
      const int64_t o_eb = __shfl_sync(0xffffffffu, eb, o);
      const uint32_t o_v = __shfl_sync(0xffffffffu, v, o);
      const uint32_t o_pd = __shfl_sync(0xffffffffu, pd, o);
      const uint32_t o_cost = __shfl_sync(0xffffffffu, cost, o);
      const int o_qi = __shfl_sync(0xffffffffu, qi, o);
      if (j < tot) {
        Ctx* c = ctxs + o_qi;
        const uint32_t off = j - (o_scan - o_n);
        if (!in_bounds(c, o_eb + off < G.E, 6)) continue;
        const int2 ed = G.wedges[o_eb + off];
        const uint32_t u = (uint32_t)ed.x;
        const uint32_t nc = o_cost + (uint32_t)ed.y;
        if (!in_bounds(c, u < G.V, 7)) continue;
        // a target costing more than ub cannot be part of an optimal tree
        const bool keep = c->hop ? (nc < c->ub_cell) : (nc <= c->ub);
        if (keep) {
          const uint32_t p = o_pd & 0xFFFFu, d = (o_pd >> 16) + (uint32_t)c->hop;
          if (!in_bounds(c, d < (uint32_t)c->DD, 11)) continue;
          unsigned long long* tp =
              (unsigned long long*)&c->table[(uint64_t)u * c->RW + (uint64_t)p * c->DD + d];
          const uint64_t nv = pack_cell(nc, PEND | o_v);
          if (nv < __ldcg(tp)) {
            const uint64_t old = atomicMin(tp, (unsigned long long)nv);
            if (cost_of(old) > nc) mark_row(c, u);
          }
        }
      }
    }
  }
}

// ---- DP rows step: merge closure of dirty rows in shared memory -------------------
// Per-warp shared memory: RW cells, RW/32 pending words, RW list slots (16-B aligned).
__host__ __device__ __forceinline__ size_t rows_smem_per_warp(int rw_max) {
  const size_t b = (size_t)rw_max * 8 + (size_t)((rw_max + 31) / 32) * 4 + (size_t)rw_max * 2;
  return (b + 15) & ~(size_t)15;
}

// Dynamic shared memory per warp: RWmax cells + RWmax/32 pending words + RWmax list.
__global__ void __launch_bounds__(256) k_rows(Ctx* ctxs, int nctx, DevGraph G, int split,
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
  uint16_t* list = (uint16_t*)(wbase + (size_t)rw_max * 8 + (size_t)((rw_max + 31) / 32) * 4);
  const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
  const uint32_t wid = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  for (uint32_t it = wid; it < total; it += warps) {
    uint32_t merges = 0;
    const int qi = find_ctx(s_pref, nctx, it);
    Ctx* c = ctxs + qi;
    const uint32_t v = c->rows[it - s_pref[qi]];
    if (!in_bounds(c, v < G.V && c->RW <= rw_max, 8)) continue;
    const int RW = c->RW, DD = c->DD, k = c->k, D = c->D, hop = c->hop;
    const uint32_t full = (uint32_t)c->full;
    unsigned long long* row = (unsigned long long*)&c->table[(uint64_t)v * RW];
    // load row, collect pending bits
    for (int i0 = 0; i0 < RW; i0 += 32) {
      const int i = i0 + lane;
      uint64_t x = CELL_INF;
      if (i < RW) {
        x = __ldcg(row + i);
        buf[i] = x;
      }
      // an unreached cell is all ones, so its pending bit must be ignored
      const uint32_t bal =
          __ballot_sync(0xffffffffu, i < RW && x != CELL_INF && ((uint32_t)x & PEND));
      if (lane == 0) pend[i0 >> 5] = bal;
    }
    if (lane == 0) atomicAnd(&c->rowbits[v >> 5], ~(1u << (v & 31)));
    __syncwarp();
    const uint32_t ubm = hop ? c->ub_cell : c->ub;
    // merge closure, by popcount class of the pending operand
    for (int j = 1; j < k; j++) {
      int nl = 0;
      for (int i0 = 0; i0 < RW; i0 += 32) {
        const int i = i0 + lane;
        const bool sel = i < RW && ((pend[i >> 5] >> (i & 31)) & 1u) && __popc(i / DD) == j;
        const uint32_t bal = __ballot_sync(0xffffffffu, sel);
        if (sel) list[nl + __popc(bal & ((1u << lane) - 1u))] = (uint16_t)i;
        nl += __popc(bal);
      }
      __syncwarp();
      if (nl == 0) continue;
      const uint32_t m = (1u << (k - j)) - 1u;  // non-empty submasks of the complement
      const uint32_t per = m * (uint32_t)DD;
      const uint32_t tp = (uint32_t)nl * per;
      merges += tp;
      for (uint32_t t = lane; t < tp; t += 32) {
        const uint32_t a = t / per, r = t - a * per;
        const uint32_t yb = r / DD + 1u, d2 = r - (yb - 1u) * DD;
        const uint32_t cell = list[a];
        const uint32_t X = cell / DD, d1 = cell - X * DD;
        if (hop && (int)(d1 + d2) > D) continue;
        const uint32_t Y = deposit(yb, full ^ X);
        if (!in_bounds(c, Y * DD + d2 < (uint32_t)RW && (X | Y) * DD < (uint32_t)RW, 9)) continue;
        const uint32_t cy = cost_of(buf[Y * DD + d2]);
        if (cy == COST_INF) continue;
        const uint32_t cand = cost_of(buf[cell]) + cy;
        const uint32_t S = X | Y;
        if (S != full && 3ull * cand > 2ull * ubm) continue;
        const uint32_t nd = d1 > d2 ? d1 : d2;
        const uint32_t tgt = S * DD + nd;
        const uint64_t nv = pack_cell(cand, PEND | MERGE | Y | (d2 << 16) | (d1 << 21));
        if (nv < buf[tgt]) {
          const uint64_t old = atomicMin(&buf[tgt], (unsigned long long)nv);
          if (nv < old) atomicOr(&pend[tgt >> 5], 1u << (tgt & 31));
        }
      }
      __syncwarp();
    }
    // one-label distances of v (non-hop, or hop with use_lb)
    uint32_t dv[KMAX];
#pragma unroll
    for (int i = 0; i < KMAX; i++) dv[i] = COST_INF;
    if (c->use_lb) {
      const uint32_t mine = lane < k ? __ldcg(&c->dist[(uint64_t)v * DIST_STRIDE + lane]) : COST_INF;
#pragma unroll
      for (int i = 0; i < KMAX; i++) dv[i] = __shfl_sync(0xffffffffu, mine, i);
    }
    const int64_t deg = G.beg[v + 1] - G.beg[v];
    // settle changed states; emit growable ones
    for (int i0 = 0; i0 < RW; i0 += 32) {
      const int i = i0 + lane;
      if (i < RW && ((pend[i >> 5] >> (i & 31)) & 1u)) {
        const uint64_t x = buf[i];
        row[i] = x & ~(uint64_t)PEND;
        const uint32_t cst = cost_of(x);
        const uint32_t p = (uint32_t)i / DD, d = (uint32_t)i - p * DD;
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
                lb = max(lb, dv[b]);
                one += dv[b];
              }
            if (!hop && one < (uint64_t)c->ub) atomicMin(&c->ub, (uint32_t)one);
          }
          const uint32_t bound = hop ? c->ub_cell : c->ub;
          bool grow = 2ull * cst <= (uint64_t)bound && (uint64_t)cst + lb <= (uint64_t)bound;
          if (hop) grow = grow && (int)d < D && cst < bound;
          if (grow && c->use_tour) {
            // tour bound of PrunedDP++ (code/PrunedDP++/include/CPUNONHOP.h:433-493):
            // the rest of the tree, doubled, is a closed walk from v through every
            // group of Xb = full \ p, so twice its cost is at least
            //   min_{i,j} d_i(v) + P(i,j,Xb) + d_j(v)            and, for every i,
            //   d_i(v) + min_j P(i,j,Xb) + min_j d_j(v),
            // P = cheapest group sequence from i to j visiting each group of Xb once.
            const uint32_t Xb = full ^ p;
            const uint32_t* Wt = c->tour + (size_t)Xb * TOUR_STRIDE;
            const uint32_t* W2 = c->tour + (size_t)c->W * TOUR_STRIDE + (size_t)Xb * KMAX;
            uint64_t mind = COST_INF;
#pragma unroll
            for (int b = 0; b < KMAX; b++)
              if (b < k && ((Xb >> b) & 1u) && dv[b] < mind) mind = dv[b];
            uint64_t lb1 = ~0ull, lb2 = 0;
#pragma unroll
            for (int a = 0; a < KMAX; a++) {
              if (a >= k || !((Xb >> a) & 1u)) continue;
              const uint64_t t2 = (uint64_t)dv[a] + __ldg(&W2[a]) + mind;
              if (t2 > lb2) lb2 = t2;
#pragma unroll
              for (int b = 0; b < KMAX; b++) {
                if (b >= k || !((Xb >> b) & 1u)) continue;
                const uint64_t t1 = (uint64_t)dv[a] + __ldg(&Wt[a * KMAX + b]) + dv[b];
                if (t1 < lb1) lb1 = t1;
              }
            }
            const uint64_t t = lb1 > lb2 ? lb1 : lb2;
            grow = (uint64_t)cst + (t + 1) / 2 <= (uint64_t)bound;
          }
          if (grow && deg > 0)
            push_state(c, v, p | (d << 16), cst, light_count(G, v, deg, grow_limit(c, cst)), split,
                       c->bucket_end);
        }
      }
    }
    if (lane == 0) {
      atomicAdd(&c->st_merge, (unsigned long long)merges);
      atomicAdd(&c->st_rows, 1ull);
    }
    __syncwarp();
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
  if (mode == CTRL_SSSP && c->phase == PH_PREP && !c->error) {
    if (c->use_tour) build_tour(c);  // block-uniform branch
    if (threadIdx.x == 0) ctrl_start_dp(c);
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
    if (c->phase != PH_DP) return;
    c->n_rows = 0;  // consumed by the rows kernel
    if (c->n_q[0] > 0) {
      c->in_ptr = c->q[0];
      c->in_n = min(c->n_q[0], c->qcap);
      c->in_kind = 0;
      c->in_idx = 0;
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
    if (c->in_kind == 0) c->n_q[0] = 0;
    else c->n_far[c->in_idx] = 0;
    c->in_n = 0;
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
  uint32_t sp = 0, nout = 0, steps = 0;
  c->stack[sp++] = (uint64_t)v0 * RW + (uint64_t)c->full * DD + d0;
  while (sp > 0) {
    if (++steps > 4u * c->stackcap) {
      c->error |= ERR_EXTRACT;
      break;
    }
    const uint64_t idx = c->stack[--sp];
    if (!in_bounds(c, idx < (uint64_t)G.V * RW, 10)) break;
    const uint32_t v = (uint32_t)(idx / RW);
    const uint32_t r = (uint32_t)(idx - (uint64_t)v * RW);
    const uint32_t p = r / DD, d = r - p * DD;
    const uint64_t cell = c->table[idx];
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
      c->stack[sp++] = (uint64_t)u * RW + (uint64_t)p * DD + (d - (uint32_t)c->hop);
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
      c->stack[sp++] = (uint64_t)v * RW + (uint64_t)X * DD + d1;
      c->stack[sp++] = (uint64_t)v * RW + (uint64_t)Y * DD + d2;
    }
  }
  if (nout > c->outcap) c->error |= ERR_EXTRACT;
  c->n_out = nout;
}

}  // namespace gst
