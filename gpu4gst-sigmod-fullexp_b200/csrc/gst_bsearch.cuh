// Batch-shared one-label distance search.
//
// The unbounded queries of one batch call need the distances from each of their groups
// to every vertex (below a cutoff).  Searching query by query reads the graph's edges and
// one random 32-byte distance row per relaxation, once per query; the relaxation rate is
// then bound by the device's random-access rate.  Here the distinct groups of all the
// batch's unbounded queries (up to BS_COLS of them) are searched together: one distance
// table of V rows x Gp columns (column c = the c-th group), one announcement bit per
// (vertex, column), and a relaxation of edge (v, u) serves every column whose distance
// at v improved in the previous step, reading u's row as one contiguous span (lanes of a
// warp take its 32-byte sectors) instead of one random row per query.
//
// Cutoffs: a query's distances are needed exactly only up to its search cutoff (its star
// bound x cut_pm / 1000).  Column c keeps the largest cutoff of the queries that use it;
// stars are found while the search runs (before each relax step, k_bs_star sums each
// query's columns at every announced vertex) and the cutoffs only decrease, so every distance at
// most a column's final cutoff is exact (every prefix of its shortest path stayed below
// it) and every other one is only known to exceed it.  A query then takes the smallest
// final cutoff of its columns as its own `cut` (distances above it are clamped to cut + 1
// by every bound), at least as strong as its own search would have reached.
//
// Hop-bounded queries of one bound D (1 <= D <= KMAX) share a search the same way over
// D tables: table h holds d^{<=h}, the cheapest paths of at most h edges (table D is the
// distance table, 1..D-1 the hop budgets).  One step is one round: round r (r >= 1)
// first copies table r into table r+1 (a coalesced pass, so that table r+1 starts from
// the paths of at most r edges), then relaxes the edges of the vertices whose table r
// row improved in round r-1 (round 0: the members, distance 0) from table r into table
// r+1 alone.  Table r is final while round r reads it, so no snapshot is needed, and
// the result is the per-query rounds'.  Stars come from tables r with 2r <= D (trees of
// diameter <= D), as in the per-query search; after the last round the tables above
// it are filled from it.
//
// Per step: k_bs_scan turns the announcement bits of the previous step into relax items
// of at most BS_CHUNK edges (a hub's range spread over many warps), k_bs_star finds the
// stars at the announced vertices and k_bs_ctrl lowers the cutoffs, k_bs_relax relaxes
// the items, and k_bs_ctrl updates the cutoffs again and ends the search when nothing
// was announced.
#pragma once
#include "gst_device.cuh"

namespace gst {

constexpr int BS_COLS = 256;   // columns (distinct groups) of one shared search, at most
constexpr int BS_CHUNK = 128;  // edges per relax item
constexpr int BS_MAXQ = MAXB;  // queries of one shared search, at most

struct BsCtx {
  uint32_t* dist;       // V x Gp distances, row v at dist + v * Gp
  uint32_t* fm[2];      // V x Wm announcement words (bit c: column c improved at v)
  uint32_t* am;         // V x Wm: v's active columns in the current step (scan -> relax)
  uint2* items;         // relax items of the current step: {v, chunk}
  uint32_t item_cap;
  uint32_t n_items;     // items of the current step (appended by the scan)
  uint32_t Gp, Wm;      // columns (a multiple of 8), mask words per vertex
  uint32_t in;          // fm[in] is scanned this step; fm[in ^ 1] takes its announcements
  uint32_t ann;         // the relax step announced something
  uint32_t done, steps, max_steps, error;
  uint32_t cut_pm;      // query cutoff: star x cut_pm / 1000
  uint32_t D;           // 0: unbounded distances; else the hop bound (rounds 0..D-1)
  uint32_t round;       // hop-bounded: the current round
  uint32_t* tab[KMAX + 1];  // hop-bounded: tab[h] = d^{<=h} (V x Gp), tab[D] = dist
  uint32_t nq;          // queries
  uint32_t qk[BS_MAXQ];
  uint16_t qcol[BS_MAXQ][KMAX];  // columns of each query's groups
  uint32_t star[BS_MAXQ];        // best star found per query (a feasible cost)
  uint32_t cutc[BS_COLS];        // per column: its distance cutoff
  unsigned long long st_relax;   // target-row sectors read (edges x active lanes)
};
constexpr uint32_t BS_ERR_ITEMS = 1, BS_ERR_STEPS = 2;

// Seeds: column c's members at distance 0, announced (blockIdx.y = column).
__global__ void k_bs_seed(BsCtx* b, DevGraph G, const int64_t* grp_ptr, const int32_t* members,
                          const int32_t* col_gid, int ncols) {
  const int c = blockIdx.y;
  if (c >= ncols) return;
  const int32_t g = col_gid[c];
  const uint32_t Gp = b->Gp, Wm = b->Wm;
  for (int64_t j = grp_ptr[g] + blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < grp_ptr[g + 1];
       j += (int64_t)gridDim.x * blockDim.x) {
    const uint32_t v = (uint32_t)members[j];
    if (v >= G.V) continue;
    atomicMin(&(b->D ? b->tab[1] : b->dist)[(uint64_t)v * Gp + c], 0u);
    if (G.beg[v + 1] > G.beg[v]) atomicOr(&b->fm[b->in][(uint64_t)v * Wm + (c >> 5)], 1u << (c & 31));
  }
}

// Scan: every vertex announced in the previous step gets its active columns (moved from
// fm[in] to am) and one relax item per BS_CHUNK edges of its list.
__global__ void k_bs_scan(BsCtx* b, DevGraph G) {
  if (b->done) return;
  const uint32_t Wm = b->Wm;
  uint32_t* fi = b->fm[b->in];
  const int lane = threadIdx.x & 31;
  for (int64_t base = (int64_t)blockIdx.x * blockDim.x; base < G.V;
       base += (int64_t)gridDim.x * blockDim.x) {
    const int64_t v = base + threadIdx.x;
    uint32_t nchunks = 0;
    if (v < G.V) {
      uint32_t x[BS_COLS / 32];
      uint32_t any = 0;
#pragma unroll
      for (uint32_t w = 0; w < BS_COLS / 32; w++) {
        x[w] = w < Wm ? __ldcg(&fi[(uint64_t)v * Wm + w]) : 0u;
        any |= x[w];
      }
      if (any) {
        // the announcements become this step's active columns; the words are cleared
        // for the step after next
#pragma unroll
        for (uint32_t w = 0; w < BS_COLS / 32; w++)
          if (w < Wm) {
            b->am[(uint64_t)v * Wm + w] = x[w];
            fi[(uint64_t)v * Wm + w] = 0u;
          }
        const int64_t deg = G.beg[v + 1] - G.beg[v];
        nchunks = (uint32_t)((deg + BS_CHUNK - 1) / BS_CHUNK);
      }
    }
    // warp-aggregated reservation of the items
    const uint32_t scan = warp_incl_scan(nchunks);
    const uint32_t tot = __shfl_sync(0xffffffffu, scan, 31);
    uint32_t basei = 0;
    if (lane == 31 && tot) basei = atomicAdd(&b->n_items, tot);
    basei = __shfl_sync(0xffffffffu, basei, 31);
    for (uint32_t j = 0; j < nchunks; j++) {
      const uint32_t i = basei + scan - nchunks + j;
      if (i < b->item_cap) b->items[i] = make_uint2((uint32_t)v, j);
      else atomicOr(&b->error, BS_ERR_ITEMS);
    }
  }
}

// Relax: one item per warp iteration, in two phases.  First lane s holds sector s
// (columns 8s..8s+7) of the item's vertex: its distances, active bits and, per active
// column, the heaviest edge it may still take (`lim`).  Then the work is the
// item's edges times its nA sectors with an active column, spread over all 32 lanes:
// lane t takes active sector t mod nA and the edges t / nA, t / nA + R, ... (R = 32 /
// nA), reading that sector of each target's row, relaxing and announcing the improved
// columns.  The kernel is bound by instruction issue, not memory (a row is one
// contiguous span), and an item rarely has more than a few active sectors, so the
// edge loop is what the compaction keeps busy.
__global__ void __launch_bounds__(256, 4) k_bs_relax(BsCtx* b, DevGraph G) {
  __shared__ uint32_t s_cut[BS_COLS];
  __shared__ uint16_t s_split[33][32];           // [nA][t]: t mod nA | (t / nA) << 8
  __shared__ unsigned char s_map[256 / 32][32];  // per warp: active index -> sector
  if (b->done) return;
  const uint32_t Gp = b->Gp, Wm = b->Wm, nsec = Gp / 8u;
  for (uint32_t c = threadIdx.x; c < BS_COLS; c += blockDim.x) s_cut[c] = c < Gp ? b->cutc[c] : 0u;
  for (uint32_t x = threadIdx.x; x < 33u * 32u; x += blockDim.x) {
    const uint32_t na = x >> 5, t = x & 31u;
    s_split[na][t] = na ? (uint16_t)((t % na) | ((t / na) << 8)) : 0;
  }
  __syncthreads();
  // hop-bounded round r: sources in table r (the members at 0 for r = 0), targets in
  // table r + 1; a round's paths extend only while they have fewer than D edges
  const uint32_t D = b->D, r = b->round;
  if (D && r >= D) return;
  const uint32_t* src_tab = D ? (r ? b->tab[r] : nullptr) : b->dist;
  uint32_t* dst_tab = D ? b->tab[r + 1] : b->dist;
  const bool extend = D == 0u || r + 1u < D;
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const uint32_t n = min(b->n_items, b->item_cap);
  const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
  uint32_t* fo = b->fm[b->in ^ 1u];
  const bool mine = (uint32_t)lane < nsec;
  const uint32_t s = (uint32_t)lane;
  unsigned long long relaxed = 0;
  uint32_t any = 0;
  for (uint32_t it = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; it < n; it += warps) {
    const uint2 item = b->items[it];
    const uint32_t v = item.x, chunk = item.y;
    uint32_t m = 0;
    if (mine) m = (__ldcg(&b->am[(uint64_t)v * Wm + (s >> 2)]) >> ((s & 3u) * 8u)) & 0xFFu;
    uint32_t dv[8];
#pragma unroll
    for (int i = 0; i < 8; i++) dv[i] = COST_INF;
    if (mine && !src_tab) {
#pragma unroll
      for (int i = 0; i < 8; i++)
        if ((m >> i) & 1u) dv[i] = 0u;  // round 0: the members themselves
    } else if (mine && m) {
      const uint4* src = (const uint4*)&src_tab[(uint64_t)v * Gp + s * 8];
      const uint4 a = __ldcg(src), c4 = __ldcg(src + 1);
      dv[0] = a.x;
      dv[1] = a.y;
      dv[2] = a.z;
      dv[3] = a.w;
      dv[4] = c4.x;
      dv[5] = c4.y;
      dv[6] = c4.z;
      dv[7] = c4.w;
    }
    // per active column: the heaviest edge it may still take from v (0: none; edge
    // weights are at least 1), and for the warp the heaviest of them all
    uint32_t lim[8], wl = 0;
#pragma unroll
    for (int i = 0; i < 8; i++) {
      const uint32_t cut = mine ? s_cut[s * 8 + i] : 0u;
      lim[i] = (((m >> i) & 1u) && dv[i] < cut) ? cut - dv[i] : 0u;
      wl = max(wl, lim[i]);
    }
    const uint32_t amask = __ballot_sync(0xffffffffu, wl != 0u);
    wl = __reduce_max_sync(0xffffffffu, wl);
    if (!amask) continue;
    const int64_t b0 = G.beg[v], b1 = G.beg[v + 1];
    const int64_t cnt = count_upto(G, v, b1 - b0, wl);
    const int64_t e0 = (int64_t)chunk * BS_CHUNK, e1 = min(cnt, e0 + BS_CHUNK);
    if (e1 <= e0) continue;
    // work: the target-row sectors this item reads, one per active sector and edge
    const uint32_t nA = (uint32_t)__popc(amask);
    relaxed += (unsigned long long)(e1 - e0) * nA;
    // compaction: active index -> sector, then each lane takes its sector's values
    if ((amask >> lane) & 1u) s_map[wib][__popc(amask & ((1u << lane) - 1u))] = (unsigned char)lane;
    __syncwarp();
    const uint32_t sp = s_split[nA][lane];
    const uint32_t R = 32u / nA;  // edges per round (warp-uniform)
    const uint32_t sec = s_map[wib][sp & 0xFFu];
    const int64_t joff = (int64_t)(sp >> 8);
    uint32_t dx[8], lx[8];
#pragma unroll
    for (int i = 0; i < 8; i++) {
      dx[i] = __shfl_sync(0xffffffffu, dv[i], (int)sec);
      lx[i] = __shfl_sync(0xffffffffu, lim[i], (int)sec);
    }
    if (joff >= (int64_t)R) continue;  // lanes beyond R x nA
    int64_t e = e0 + joff;
    // the edges are sorted by weight: a lane stops at the first one heavier than every
    // limit of its sector; two edges per lane in flight
    uint32_t lmax = 0;
#pragma unroll
    for (int i = 0; i < 8; i++) lmax = max(lmax, lx[i]);
    const int64_t R2 = 2 * (int64_t)R;
    int2 ea = e < e1 ? G.wedges[b0 + e] : make_int2(0, 0);
    int2 eb = e + R < e1 ? G.wedges[b0 + e + R] : make_int2(0, 0);
    for (; e < e1; e += R2) {
      const bool hb = e + R < e1;
      const uint32_t ua = (uint32_t)ea.x, wa = (uint32_t)ea.y;
      const uint32_t ub = (uint32_t)eb.x, wb = (uint32_t)eb.y;
      if (wa > lmax) break;
      const bool ga = ua < G.V, gb = hb && wb <= lmax && ub < G.V;
      uint4 ra0 = make_uint4(0, 0, 0, 0), ra1 = ra0, rb0 = ra0, rb1 = ra0;
      if (ga) {
        const uint4* dst = (const uint4*)&dst_tab[(uint64_t)ua * Gp + sec * 8];
        ra0 = __ldcg(dst);
        ra1 = __ldcg(dst + 1);
      }
      if (gb) {
        const uint4* dst = (const uint4*)&dst_tab[(uint64_t)ub * Gp + sec * 8];
        rb0 = __ldcg(dst);
        rb1 = __ldcg(dst + 1);
      }
      if (e + R2 < e1) ea = G.wedges[b0 + e + R2];
      if (e + R2 + R < e1) eb = G.wedges[b0 + e + R2 + R];
#pragma unroll
      for (int x = 0; x < 2; x++) {
        const bool g = x ? gb : ga;
        const uint32_t u = x ? ub : ua, w = x ? wb : wa;
        const uint4 r0 = x ? rb0 : ra0, r1 = x ? rb1 : ra1;
        if (!g) continue;
        const uint32_t du[8] = {r0.x, r0.y, r0.z, r0.w, r1.x, r1.y, r1.z, r1.w};
        uint32_t imp = 0;
#pragma unroll
        for (int i = 0; i < 8; i++) {
          if (w <= lx[i]) {
            const uint32_t nd = dx[i] + w;
            if (nd < du[i]) {
              atomicMin(&dst_tab[(uint64_t)u * Gp + sec * 8 + i], nd);
              if (w < lx[i] && extend) imp |= 1u << i;
            }
          }
        }
        if (imp) {
          atomicOr(&fo[(uint64_t)u * Wm + (sec >> 2)], imp << ((sec & 3u) * 8u));
          any = 1u;
        }
      }
    }
  }
  any = __reduce_or_sync(0xffffffffu, any);
  if (lane == 0 && any) b->ann = 1u;
  if (lane == 0 && relaxed) atomicAdd(&b->st_relax, relaxed);  // the same in every lane
}

// Hop-bounded tables (n4 = V x Gp / 4 uint4 per table).  Before round r >= 1:
// table r + 1 := table r.  With `finish`, after the search: every table above the last
// round's target := that target (the search ended early; no path has more edges).
__global__ void k_bs_copy(BsCtx* b, int64_t n4, int finish) {
  const uint32_t D = b->D;
  if (!D) return;
  uint32_t from, h1;  // tables from + 1..h1 := table from
  if (!finish) {
    if (b->done || b->round == 0u || b->round >= D) return;
    from = b->round;
    h1 = from + 1u;
  } else {
    if (b->error) return;
    from = b->round + 1u;
    h1 = D;
  }
  if (from >= h1) return;
  const uint4* src = (const uint4*)b->tab[from];
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n4;
       i += (int64_t)gridDim.x * blockDim.x) {
    const uint4 x = __ldcs(src + i);
    for (uint32_t h = from + 1u; h <= h1; h++) __stcs((uint4*)b->tab[h] + i, x);
  }
}

// Stars, before the relax step: at every vertex announced for this step (the first
// chunk of its items), each query's columns summed (the query's k shortest paths from v
// form a connected subgraph covering every group, a feasible cost).  Hop-bounded: from
// table r with 2r <= D only (a tree of diameter <= D).  Found before the relax step, a
// star lowers the cutoffs that this very step relaxes against.
__global__ void __launch_bounds__(256) k_bs_star(BsCtx* b) {
  __shared__ __align__(16) uint32_t s_row[256 / 32][BS_COLS];  // per warp: the vertex's row
  __shared__ uint32_t s_star[BS_MAXQ];
  if (b->done) return;
  const uint32_t D = b->D, r = b->round;
  if (D && !(r >= 1u && 2u * r <= D)) return;
  const uint32_t* src_tab = D ? b->tab[r] : b->dist;
  const uint32_t Gp = b->Gp, nsec = Gp / 8u, nq = b->nq;
  for (uint32_t q = threadIdx.x; q < BS_MAXQ; q += blockDim.x) s_star[q] = COST_INF;
  __syncthreads();
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const uint32_t n = min(b->n_items, b->item_cap);
  const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
  const uint32_t wid = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  for (uint32_t base = wid * 32u; base < n; base += warps * 32u) {
    // lane i looks at item base + i; the warp then takes the first chunks one by one
    uint32_t v = 0;
    bool first = false;
    if (base + lane < n) {
      const uint2 item = b->items[base + lane];
      v = item.x;
      first = item.y == 0u;
    }
    uint32_t todo = __ballot_sync(0xffffffffu, first);
    while (todo) {
      const int src = __ffs(todo) - 1;
      todo &= todo - 1u;
      const uint32_t x = __shfl_sync(0xffffffffu, v, src);
      if ((uint32_t)lane < nsec) {
        const uint4* p = (const uint4*)&src_tab[(uint64_t)x * Gp + lane * 8];
        const uint4 a = __ldcg(p), c4 = __ldcg(p + 1);
        uint4* o = (uint4*)&s_row[wib][lane * 8];
        o[0] = a;
        o[1] = c4;
      }
      __syncwarp();
      for (uint32_t q = (uint32_t)lane; q < nq; q += 32) {
        uint64_t sum = 0;
        for (uint32_t i = 0; i < b->qk[q]; i++) sum += s_row[wib][b->qcol[q][i]];
        if (sum < (uint64_t)s_star[q]) atomicMin(&s_star[q], (uint32_t)sum);
      }
      __syncwarp();
    }
  }
  __syncthreads();
  for (uint32_t q = threadIdx.x; q < nq; q += blockDim.x)
    if (s_star[q] < COST_INF) atomicMin(&b->star[q], s_star[q]);
}

// Control (one block): column cutoffs from the query stars; with `advance`, after the
// relax step, the next step's buffers and the end of the search.
__global__ void k_bs_ctrl(BsCtx* b, int advance) {
  if (b->done) return;
  const uint32_t nq = b->nq, Gp = b->Gp;
  for (uint32_t c = threadIdx.x; c < Gp; c += blockDim.x) {
    uint32_t mx = 0;
    bool used = false;
    for (uint32_t q = 0; q < nq; q++)
      for (uint32_t i = 0; i < b->qk[q]; i++)
        if (b->qcol[q][i] == c) {
          used = true;
          const uint32_t st = b->star[q];
          const uint64_t x = st == COST_INF ? COST_INF : (uint64_t)st * b->cut_pm / 1000u;
          mx = max(mx, x >= COST_INF ? COST_INF : (uint32_t)x);
        }
    if (used) b->cutc[c] = min(b->cutc[c], mx);
  }
  if (!advance) return;
  __syncthreads();
  if (threadIdx.x == 0) {
    if (b->error || !b->ann) {
      b->done = 1u;
    } else if (++b->steps > b->max_steps) {
      b->error |= BS_ERR_STEPS;
      b->done = 1u;
    } else {
      b->ann = 0u;
      b->in ^= 1u;
      b->n_items = 0u;
      b->round++;
    }
  }
}

// A query's distance rows (stride ds) from a shared table (V x Gp): column cols[i] for
// group i.
__global__ void k_bs_gather(uint32_t* rows, uint32_t ds, int k, const uint32_t* table, uint32_t Gp,
                            ushort4 c0, ushort4 c1, int64_t V) {
  const uint16_t cols[8] = {c0.x, c0.y, c0.z, c0.w, c1.x, c1.y, c1.z, c1.w};
  for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < V;
       v += (int64_t)gridDim.x * blockDim.x) {
    uint32_t d[8];
#pragma unroll
    for (int i = 0; i < 8; i++) d[i] = i < k ? __ldcg(&table[(uint64_t)v * Gp + cols[i]]) : COST_INF;
    store_drow(rows, ds, (uint64_t)v, make_uint4(d[0], d[1], d[2], d[3]), make_uint4(d[4], d[5], d[6], d[7]));
  }
}

}  // namespace gst
