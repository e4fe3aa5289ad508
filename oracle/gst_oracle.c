/*
 * gst_oracle.c — CPU restatement of the reference's exact GST dynamic program.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker for the CUDA engine: only
 * tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg may load it.
 * The engine never calls it and has no CPU fallback.
 *
 * What it restates (rucdatascience/GPU4GST-sigmod-fullEXP):
 *   oracle_sssp_groups  multi-source Dijkstra from a vertex group, as
 *                       graph_v_of_v_idealID_PrunedDPPlusPlus_find_SPs_to_g
 *                       (code/PrunedDP++/include/CPUNONHOP.h:21-67): a dummy
 *                       source joined to every member by a 0-weight edge.
 *   oracle_gst_nonhop   the best-first DPBF recurrence that PrunedDP++ prunes
 *                       (code/PrunedDP++/include/CPUNONHOP.h:496-957): states
 *                       (v,p), T(v,p)=0 for every non-empty p inside v's group
 *                       mask (:593-621), grow along each edge (:797-866), merge
 *                       T(v,p1)+T(v,p2) with already-popped disjoint p2
 *                       (:870-955), stop at the first popped full-set state
 *                       (:655-675); tree rebuilt by the parent walk of
 *                       graph_v_of_v_idealID_PrunedDPPlusPlus_build_tree
 *                       (:387-429).  The cost is the same optimum PrunedDP++
 *                       returns (its pruning only skips states that cannot be on
 *                       an optimal tree); the returned tree may differ on ties.
 *   oracle_gst_hop      HOP_cpu (code/D-PrunedDP++/include/CPUHOP.h:107-283):
 *                       states (v,p,d), singletons (v,{i},0) (:153-168), grow to
 *                       d+1 while d<D (:190-204), merge with any current
 *                       (v,p2,d2), d2<=D-d, into max(d,d2) (:205-225), stop at
 *                       the first popped full-set state at any d<=D (:184-188),
 *                       parent walk (:231-257).
 *   oracle_hop_bound_check, oracle_nonhop_bound_check  not reference algorithms:
 *                       the DPs above pruned with the engine's rules, so that tests
 *                       can check that those rules never remove an optimal tree.
 *
 * Parity pin: tests/golden/ holds costs produced by the reference's own CPU
 * solvers (compiled unmodified under oracle/_ref by oracle/Makefile) on seeded
 * inputs; tests check this file against them.
 *
 * Costs are int64 here; "infeasible" is reported as -1 (the reference prints its
 * sentinel 100000, code/PrunedDP++/include/exp_CPU_nonHop.h:120-126).
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define ORACLE_INF ((int64_t)1 << 60)

/* ---- binary min-heap of (key, a, b, c) with lazy deletion ----------------- */
typedef struct {
  int64_t key;
  int32_t v;
  int32_t p;
  int32_t d;
} hitem;

typedef struct {
  hitem* a;
  int64_t n, cap;
} heap_t;

static int hless(const hitem* x, const hitem* y) {
  if (x->key != y->key) return x->key < y->key;
  if (x->v != y->v) return x->v < y->v;
  if (x->p != y->p) return x->p < y->p;
  return x->d < y->d;
}

static int heap_push(heap_t* h, hitem it) {
  if (h->n == h->cap) {
    int64_t nc = h->cap ? h->cap * 2 : 1024;
    hitem* na = (hitem*)realloc(h->a, sizeof(hitem) * nc);
    if (!na) return -1;
    h->a = na;
    h->cap = nc;
  }
  int64_t i = h->n++;
  h->a[i] = it;
  while (i > 0) {
    int64_t p = (i - 1) / 2;
    if (!hless(&h->a[i], &h->a[p])) break;
    hitem t = h->a[i];
    h->a[i] = h->a[p];
    h->a[p] = t;
    i = p;
  }
  return 0;
}

static hitem heap_pop(heap_t* h) {
  hitem top = h->a[0];
  h->a[0] = h->a[--h->n];
  int64_t i = 0;
  for (;;) {
    int64_t l = 2 * i + 1, r = l + 1, m = i;
    if (l < h->n && hless(&h->a[l], &h->a[m])) m = l;
    if (r < h->n && hless(&h->a[r], &h->a[m])) m = r;
    if (m == i) break;
    hitem t = h->a[i];
    h->a[i] = h->a[m];
    h->a[m] = t;
    i = m;
  }
  return top;
}

/* ---- helpers -------------------------------------------------------------- */
static int32_t edge_weight(const int64_t* beg, const int32_t* adj, const int32_t* w, int32_t a,
                           int32_t b) {
  for (int64_t i = beg[a]; i < beg[a + 1]; i++)
    if (adj[i] == b) return w[i];
  return -1;
}

/* group-membership mask of each vertex for the k query groups (bit i = i-th id) */
static uint32_t* query_masks(int64_t V, const int64_t* grp_ptr, const int32_t* members,
                             int32_t k, const int32_t* group_ids) {
  uint32_t* m = (uint32_t*)calloc((size_t)V, sizeof(uint32_t));
  if (!m) return NULL;
  for (int32_t i = 0; i < k; i++) {
    int32_t g = group_ids[i];
    for (int64_t j = grp_ptr[g]; j < grp_ptr[g + 1]; j++) m[members[j]] |= 1u << i;
  }
  return m;
}

typedef struct {
  int32_t a, b, w;
} tedge;

static int cmp_tedge(const void* x, const void* y) {
  const tedge* p = (const tedge*)x;
  const tedge* q = (const tedge*)y;
  if (p->a != q->a) return p->a < q->a ? -1 : 1;
  if (p->b != q->b) return p->b < q->b ? -1 : 1;
  return 0;
}

/* sort + unique the collected edges (the reference collects them in a hash
 * graph, so duplicates collapse), copy out, return the distinct count */
static int64_t emit_edges(tedge* e, int64_t n, int64_t cap, int32_t* eu, int32_t* ev,
                          int32_t* ew, int64_t* wsum) {
  qsort(e, (size_t)n, sizeof(tedge), cmp_tedge);
  int64_t m = 0;
  *wsum = 0;
  for (int64_t i = 0; i < n; i++) {
    if (i > 0 && e[i].a == e[i - 1].a && e[i].b == e[i - 1].b) continue;
    if (m < cap) {
      eu[m] = e[i].a;
      ev[m] = e[i].b;
      ew[m] = e[i].w;
    }
    *wsum += e[i].w;
    m++;
  }
  return m;
}

/* ---- multi-source Dijkstra ------------------------------------------------ */
int oracle_sssp_groups(int64_t V, const int64_t* beg, const int32_t* adj, const int32_t* w,
                       int64_t n_src, const int32_t* src, int64_t* dist) {
  heap_t h = {0};
  for (int64_t v = 0; v < V; v++) dist[v] = ORACLE_INF;
  for (int64_t i = 0; i < n_src; i++) {
    dist[src[i]] = 0;
    hitem it = {0, src[i], 0, 0};
    if (heap_push(&h, it)) return 1;
  }
  while (h.n) {
    hitem it = heap_pop(&h);
    if (it.key != dist[it.v]) continue;
    for (int64_t e = beg[it.v]; e < beg[it.v + 1]; e++) {
      int64_t nd = it.key + w[e];
      if (nd < dist[adj[e]]) {
        dist[adj[e]] = nd;
        hitem ni = {nd, adj[e], 0, 0};
        if (heap_push(&h, ni)) return 1;
      }
    }
  }
  free(h.a);
  return 0;
}

/* ---- non-hop exact DP ----------------------------------------------------- */
/* Returns 0 on success.  *cost = optimum (-1 if the groups cannot be connected),
 * *root = vertex of the popped full-set state, *n_edges = distinct tree edges
 * (written up to edge_cap), *edge_sum = their weight sum, *pops = states popped. */
int oracle_gst_nonhop(int64_t V, const int64_t* beg, const int32_t* adj, const int32_t* w,
                      const int64_t* grp_ptr, const int32_t* members, int32_t k,
                      const int32_t* group_ids, int64_t* cost, int32_t* root, int64_t* n_edges,
                      int64_t edge_cap, int32_t* eu, int32_t* ev, int32_t* ew, int64_t* edge_sum,
                      int64_t* pops) {
  if (k < 1 || k > 16) return 1;
  const int32_t W = 1 << k, FULL = W - 1;
  uint32_t* mask = query_masks(V, grp_ptr, members, k, group_ids);
  int64_t* c = (int64_t*)malloc(sizeof(int64_t) * (size_t)V * W);
  int32_t* par = (int32_t*)malloc(sizeof(int32_t) * (size_t)V * W); /* grow: -1-u ; merge: p1 */
  uint8_t* done = (uint8_t*)calloc((size_t)V * W, 1);
  if (!mask || !c || !par || !done) return 2;
  for (int64_t i = 0; i < V * W; i++) c[i] = ORACLE_INF;
  heap_t h = {0};
  for (int64_t v = 0; v < V; v++) {
    uint32_t m = mask[v];
    for (uint32_t p = m; p; p = (p - 1) & m) {
      c[v * W + p] = 0;
      par[v * W + p] = 0; /* leaf */
      hitem it = {0, (int32_t)v, (int32_t)p, 0};
      heap_push(&h, it);
    }
  }
  int64_t npop = 0;
  int32_t rv = -1;
  while (h.n) {
    hitem it = heap_pop(&h);
    const int64_t s = (int64_t)it.v * W + it.p;
    if (done[s] || it.key != c[s]) continue;
    done[s] = 1;
    npop++;
    if (it.p == FULL) {
      rv = it.v;
      break;
    }
    const int64_t cv = it.key;
    for (int64_t e = beg[it.v]; e < beg[it.v + 1]; e++) {
      const int64_t t = (int64_t)adj[e] * W + it.p;
      if (!done[t] && cv + w[e] < c[t]) {
        c[t] = cv + w[e];
        par[t] = -1 - it.v;
        hitem ni = {c[t], adj[e], it.p, 0};
        heap_push(&h, ni);
      }
    }
    const uint32_t comp = (uint32_t)FULL & ~(uint32_t)it.p;
    for (uint32_t q = comp; q; q = (q - 1) & comp) {
      const int64_t sq = (int64_t)it.v * W + q;
      if (!done[sq]) continue;
      const int64_t t = (int64_t)it.v * W + (it.p | q);
      const int64_t nc = cv + c[sq];
      if (!done[t] && nc < c[t]) {
        c[t] = nc;
        par[t] = it.p; /* p1; p2 = (p|q) ^ p1 */
        hitem ni = {nc, it.v, (int32_t)(it.p | q), 0};
        heap_push(&h, ni);
      }
    }
  }
  *pops = npop;
  *root = rv;
  *n_edges = 0;
  *edge_sum = 0;
  if (rv < 0) {
    *cost = -1;
  } else {
    *cost = c[(int64_t)rv * W + FULL];
    /* parent walk: queue of (v,p) */
    int64_t qcap = 1024, qh = 0, qt = 0, ecap = 1024, ne = 0;
    int64_t* qs = (int64_t*)malloc(sizeof(int64_t) * qcap);
    tedge* es = (tedge*)malloc(sizeof(tedge) * ecap);
    qs[qt++] = (int64_t)rv * W + FULL;
    while (qh < qt) {
      const int64_t s = qs[qh++];
      const int32_t v = (int32_t)(s / W), p = (int32_t)(s % W);
      int64_t add[2];
      int na = 0;
      if (c[s] == 0 && ((uint32_t)p & ~mask[v]) == 0) {
        /* leaf: v covers p */
      } else if (par[s] < 0) {
        const int32_t u = -1 - par[s];
        if (ne == ecap) es = (tedge*)realloc(es, sizeof(tedge) * (ecap *= 2));
        es[ne].a = u < v ? u : v;
        es[ne].b = u < v ? v : u;
        es[ne].w = edge_weight(beg, adj, w, u, v);
        ne++;
        add[na++] = (int64_t)u * W + p;
      } else {
        const int32_t p1 = par[s], p2 = p ^ p1;
        add[na++] = (int64_t)v * W + p1;
        add[na++] = (int64_t)v * W + p2;
      }
      for (int i = 0; i < na; i++) {
        if (qt == qcap) qs = (int64_t*)realloc(qs, sizeof(int64_t) * (qcap *= 2));
        qs[qt++] = add[i];
      }
    }
    *n_edges = emit_edges(es, ne, edge_cap, eu, ev, ew, edge_sum);
    free(qs);
    free(es);
  }
  free(h.a);
  free(mask);
  free(c);
  free(par);
  free(done);
  return 0;
}

/* ---- hop-bounded DP (HOP_cpu) --------------------------------------------- */
int oracle_gst_hop(int64_t V, const int64_t* beg, const int32_t* adj, const int32_t* w,
                   const int64_t* grp_ptr, const int32_t* members, int32_t k,
                   const int32_t* group_ids, int32_t D, int64_t* cost, int32_t* root,
                   int32_t* root_d, int64_t* n_edges, int64_t edge_cap, int32_t* eu, int32_t* ev,
                   int32_t* ew, int64_t* edge_sum, int64_t* pops) {
  if (k < 1 || k > 16 || D < 0 || D > 64) return 1;
  const int32_t W = 1 << k, FULL = W - 1, DD = D + 1;
  const int64_t S = V * W * DD;
  uint32_t* mask = query_masks(V, grp_ptr, members, k, group_ids);
  int64_t* c = (int64_t*)malloc(sizeof(int64_t) * (size_t)S);
  /* parent: type(2 bits) | payload: grow -> u ; merge -> p1, d1, d2 */
  uint8_t* typ = (uint8_t*)calloc((size_t)S, 1);
  int32_t* pa = (int32_t*)malloc(sizeof(int32_t) * (size_t)S);
  int32_t* pb = (int32_t*)malloc(sizeof(int32_t) * (size_t)S);
  if (!mask || !c || !typ || !pa || !pb) return 2;
  for (int64_t i = 0; i < S; i++) c[i] = ORACLE_INF;
  heap_t h = {0};
#define IDX(v, p, d) (((int64_t)(v) * W + (p)) * DD + (d))
  for (int64_t v = 0; v < V; v++) {
    for (int32_t i = 0; i < k; i++)
      if (mask[v] >> i & 1) {
        c[IDX(v, 1 << i, 0)] = 0;
        hitem it = {0, (int32_t)v, 1 << i, 0};
        heap_push(&h, it);
      }
  }
  int64_t npop = 0;
  int32_t rv = -1, rp = 0, rd = 0;
  while (h.n) {
    hitem it = heap_pop(&h);
    const int32_t v = it.v, p = it.p, d = it.d;
    const int64_t cv = it.key;
    if (cv != c[IDX(v, p, d)]) continue;
    npop++;
    if (p == FULL) {
      rv = v;
      rp = p;
      rd = d;
      break;
    }
    if (d < D) {
      for (int64_t e = beg[v]; e < beg[v + 1]; e++) {
        const int64_t t = IDX(adj[e], p, d + 1);
        if (c[t] > cv + w[e]) {
          c[t] = cv + w[e];
          typ[t] = 1;
          pa[t] = v;
          hitem ni = {c[t], adj[e], p, d + 1};
          heap_push(&h, ni);
        }
      }
    }
    for (int32_t p2 = 1; p2 <= FULL; p2++) {
      if (p2 & p) continue;
      for (int32_t d2 = 0; d2 <= D - d; d2++) {
        const int64_t c2 = c[IDX(v, p2, d2)];
        if (c2 >= ORACLE_INF) continue;
        const int32_t nd = d > d2 ? d : d2;
        const int64_t t = IDX(v, p | p2, nd);
        if (c[t] > cv + c2) {
          c[t] = cv + c2;
          typ[t] = 2;
          pa[t] = p;
          pb[t] = (d << 8) | d2;
          hitem ni = {c[t], v, p | p2, nd};
          heap_push(&h, ni);
        }
      }
    }
  }
  *pops = npop;
  *root = rv;
  *root_d = rd;
  *n_edges = 0;
  *edge_sum = 0;
  if (rv < 0) {
    *cost = -1;
  } else {
    *cost = c[IDX(rv, rp, rd)];
    int64_t qcap = 1024, qh = 0, qt = 0, ecap = 1024, ne = 0;
    int64_t* qs = (int64_t*)malloc(sizeof(int64_t) * qcap);
    tedge* es = (tedge*)malloc(sizeof(tedge) * ecap);
    qs[qt++] = IDX(rv, rp, rd);
    while (qh < qt) {
      const int64_t s = qs[qh++];
      const int32_t d = (int32_t)(s % DD);
      const int32_t p = (int32_t)((s / DD) % W);
      const int32_t v = (int32_t)(s / DD / W);
      int64_t add[2];
      int na = 0;
      if (typ[s] == 1) {
        const int32_t u = pa[s];
        if (ne == ecap) es = (tedge*)realloc(es, sizeof(tedge) * (ecap *= 2));
        es[ne].a = u < v ? u : v;
        es[ne].b = u < v ? v : u;
        es[ne].w = edge_weight(beg, adj, w, u, v);
        ne++;
        add[na++] = IDX(u, p, d - 1);
      } else if (typ[s] == 2) {
        const int32_t p1 = pa[s], d1 = pb[s] >> 8, d2 = pb[s] & 0xff;
        add[na++] = IDX(v, p1, d1);
        add[na++] = IDX(v, p ^ p1, d2);
      }
      for (int i = 0; i < na; i++) {
        if (qt == qcap) qs = (int64_t*)realloc(qs, sizeof(int64_t) * (qcap *= 2));
        qs[qt++] = add[i];
      }
    }
    *n_edges = emit_edges(es, ne, edge_cap, eu, ev, ew, edge_sum);
    free(qs);
    free(es);
  }
#undef IDX
  free(h.a);
  free(mask);
  free(c);
  free(typ);
  free(pa);
  free(pb);
  return 0;
}

/* ---- check of the engine's hop-bounded pruning (not a reference algorithm) ----
 * oracle_hop_bound_check runs the cost-ordered hop DP of oracle_gst_hop with the rules
 * the engine prunes hop-bounded queries with, against ub = the cheapest star of paths
 * of at most D/2 edges (a tree of diameter <= D), or no bound when none exists.  With
 * d^{<=h} the cheapest paths of at most h edges (h synchronous rounds here), a state
 * (v, p, d) of cost c, Xb the missing groups and dl_i = d_i^{<=D-d}(v):
 *   it grows (to height d + 1 < = D) only if 2c <= ub, c + max_{i in Xb} dl_i <= ub and
 *   c + ceil(max(lb1, lb2) / 2) <= ub, lb1 and lb2 the tour bounds below on dl;
 *   a grown target (u, p, d + 1) is written only if its cost c' keeps c' < ub + 1,
 *   c' + max dl_i(u) <= ub and c' + ceil(lb2(u) / 2) <= ub;
 *   a merged state other than the full set is kept only if 3c <= 2ub.
 * The tour bounds use group distances vv[i][j] = min over members m of group i of
 * d_j^{<=D}(m) (the tree paths between groups have at most D edges):
 *   lb1 = min_{a,b in Xb} dl_a + P(Xb, a, b) + dl_b,
 *   lb2 = max_{a in Xb} (dl_a + min_b P(Xb, a, b)) + min_{b in Xb} dl_b.
 * The engine keeps c + lb <= ub + 1 (its bound is the star plus one), a looser test.
 * Equal costs to oracle_gst_hop on random instances check that the rules never remove
 * an optimal tree.  Outputs: cost (-1 infeasible), star (-1 none), pops. */
int oracle_hop_bound_check(int64_t V, const int64_t* beg, const int32_t* adj, const int32_t* w,
                           const int64_t* grp_ptr, const int32_t* members, int32_t k,
                           const int32_t* group_ids, int32_t D, int64_t* cost, int64_t* star,
                           int64_t* pops) {
  if (k < 1 || k > 8 || D < 0 || D > 64) return 1;
  const int32_t W = 1 << k, FULL = W - 1, DD = D + 1;
  const int64_t S = V * W * DD;
  uint32_t* mask = query_masks(V, grp_ptr, members, k, group_ids);
  int64_t* dh = (int64_t*)malloc(sizeof(int64_t) * (size_t)(V * k * DD));
  int64_t* c = (int64_t*)malloc(sizeof(int64_t) * (size_t)S);
  int64_t* P = (int64_t*)malloc(sizeof(int64_t) * (size_t)W * 64);  /* P[X][a][b] */
  if (!mask || !dh || !c || !P) return 2;
  /* d^{<=h}: round h extends the paths of round h - 1 by one edge */
  for (int64_t v = 0; v < V; v++)
    for (int32_t i = 0; i < k; i++) dh[v * k + i] = (mask[v] >> i & 1) ? 0 : ORACLE_INF;
  for (int32_t h = 1; h <= D; h++) {
    const int64_t* prev = dh + (int64_t)(h - 1) * V * k;
    int64_t* cur = dh + (int64_t)h * V * k;
    memcpy(cur, prev, sizeof(int64_t) * (size_t)(V * k));
    for (int64_t v = 0; v < V; v++)
      for (int64_t e = beg[v]; e < beg[v + 1]; e++)
        for (int32_t i = 0; i < k; i++) {
          const int64_t x = prev[v * k + i] + w[e];
          if (prev[v * k + i] < ORACLE_INF && x < cur[(int64_t)adj[e] * k + i])
            cur[(int64_t)adj[e] * k + i] = x;
        }
  }
#define DH(h, v, i) (dh[((int64_t)(h) * V + (v)) * k + (i)])
  int64_t vv[8][8];
  for (int32_t i = 0; i < k; i++)
    for (int32_t j = 0; j < k; j++) {
      vv[i][j] = ORACLE_INF;
      const int32_t g = group_ids[i];
      for (int64_t m = grp_ptr[g]; m < grp_ptr[g + 1]; m++)
        if (DH(D, members[m], j) < vv[i][j]) vv[i][j] = DH(D, members[m], j);
    }
  for (int64_t x = 0; x < (int64_t)W * 64; x++) P[x] = ORACLE_INF;
  for (int32_t X = 1; X <= FULL; X++)
    for (int32_t a = 0; a < k; a++) {
      if (!(X >> a & 1)) continue;
      for (int32_t b = 0; b < k; b++) {
        if (!(X >> b & 1)) continue;
        int64_t val = ORACLE_INF;
        if (X == (1 << a)) {
          val = 0;
        } else if (b != a) {
          const int32_t prev = X ^ (1 << b);
          for (int32_t j = 0; j < k; j++)
            if ((prev >> j & 1) && P[(int64_t)prev * 64 + a * 8 + j] < ORACLE_INF &&
                vv[j][b] < ORACLE_INF && P[(int64_t)prev * 64 + a * 8 + j] + vv[j][b] < val)
              val = P[(int64_t)prev * 64 + a * 8 + j] + vv[j][b];
        }
        P[(int64_t)X * 64 + a * 8 + b] = val;
      }
    }
  int64_t ub = ORACLE_INF;
  for (int64_t v = 0; v < V; v++) {
    int64_t sum = 0;
    for (int32_t i = 0; i < k && sum < ORACLE_INF; i++)
      sum = DH(D / 2, v, i) >= ORACLE_INF ? ORACLE_INF : sum + DH(D / 2, v, i);
    if (sum < ub) ub = sum;
  }
  *star = ub < ORACLE_INF ? ub : -1;
  /* the one-label bound, lb2 and (with `both`) lb1 of state (v, p) at height d */
  int64_t one, lb1, lb2;
#define BOUNDS(v, p, d, both)                                                          \
  do {                                                                                 \
    const int32_t xb_ = FULL ^ (p), h_ = D - (d);                                      \
    int64_t mind_ = ORACLE_INF;                                                        \
    one = 0;                                                                           \
    lb1 = ORACLE_INF;                                                                  \
    lb2 = 0;                                                                           \
    for (int32_t i_ = 0; i_ < k; i_++)                                                 \
      if (xb_ >> i_ & 1) {                                                             \
        if (DH(h_, v, i_) > one) one = DH(h_, v, i_);                                  \
        if (DH(h_, v, i_) < mind_) mind_ = DH(h_, v, i_);                              \
      }                                                                                \
    for (int32_t a_ = 0; a_ < k; a_++) {                                               \
      if (!(xb_ >> a_ & 1)) continue;                                                  \
      int64_t w2_ = ORACLE_INF;                                                        \
      for (int32_t b_ = 0; b_ < k; b_++)                                               \
        if (xb_ >> b_ & 1) {                                                           \
          const int64_t pab_ = P[(int64_t)xb_ * 64 + a_ * 8 + b_];                     \
          if (pab_ < w2_) w2_ = pab_;                                                  \
          if (both && DH(h_, v, a_) + pab_ + DH(h_, v, b_) < lb1)                      \
            lb1 = DH(h_, v, a_) + pab_ + DH(h_, v, b_);                                \
        }                                                                              \
      if (DH(h_, v, a_) + w2_ + mind_ > lb2) lb2 = DH(h_, v, a_) + w2_ + mind_;        \
    }                                                                                  \
  } while (0)
  for (int64_t i = 0; i < S; i++) c[i] = ORACLE_INF;
  heap_t h = {0};
#define IDX(v, p, d) (((int64_t)(v) * W + (p)) * DD + (d))
  for (int64_t v = 0; v < V; v++)
    for (int32_t i = 0; i < k; i++)
      if (mask[v] >> i & 1) {
        c[IDX(v, 1 << i, 0)] = 0;
        hitem it = {0, (int32_t)v, 1 << i, 0};
        heap_push(&h, it);
      }
  int64_t npop = 0, best = -1;
  while (h.n) {
    hitem it = heap_pop(&h);
    const int32_t v = it.v, p = it.p, d = it.d;
    const int64_t cv = it.key;
    if (cv != c[IDX(v, p, d)]) continue;
    npop++;
    if (p == FULL) {
      best = cv;
      break;
    }
    BOUNDS(v, p, d, 1);
    const int64_t tb = lb1 > lb2 ? lb1 : lb2;
    if (d < D && 2 * cv <= ub && cv + one <= ub && cv + (tb + 1) / 2 <= ub)
      for (int64_t e = beg[v]; e < beg[v + 1]; e++) {
        const int64_t t = IDX(adj[e], p, d + 1), nc = cv + w[e];
        if (nc > ub || c[t] <= nc) continue;
        BOUNDS(adj[e], p, d + 1, 0);
        if (nc + one > ub || nc + (lb2 + 1) / 2 > ub) continue;
        c[t] = nc;
        hitem ni = {nc, adj[e], p, d + 1};
        heap_push(&h, ni);
      }
    for (int32_t p2 = 1; p2 <= FULL; p2++) {
      if (p2 & p) continue;
      for (int32_t d2 = 0; d2 <= D - d; d2++) {
        const int64_t c2 = c[IDX(v, p2, d2)];
        if (c2 >= ORACLE_INF) continue;
        const int32_t nd = d > d2 ? d : d2, q = p | p2;
        const int64_t t = IDX(v, q, nd), nc = cv + c2;
        if (q != FULL && 3 * nc > 2 * ub) continue;
        if (c[t] > nc) {
          c[t] = nc;
          hitem ni = {nc, v, q, nd};
          heap_push(&h, ni);
        }
      }
    }
  }
#undef IDX
#undef BOUNDS
#undef DH
  *cost = best;
  *pops = npop;
  free(h.a);
  free(mask);
  free(dh);
  free(c);
  free(P);
  return 0;
}

/* ---- check of the engine's unbounded pruning (not a reference algorithm) -----
 * oracle_nonhop_bound_check runs the cost-ordered DP of oracle_gst_nonhop with the
 * engine's rules against ub = the star bound min_v sum_i d_i(v) (a feasible cost):
 *   a popped state (v, p, c) grows only if 2c <= ub, c + max_{i not in p} d_i(v) <= ub
 *   and c + ceil(max(lb1, lb2) / 2) <= ub (tour bound, below);
 *   a grown target (u, p, c') is written only if c' <= ub, c' + max_{i not in p} d_i(u)
 *   <= ub and c' + ceil(lb2 / 2) <= ub (the O(k) half of the tour bound);
 *   a merged state other than the full set is kept only if 3c <= 2ub;
 * with Xb the missing groups, vv[i][j] = min over members m of group i of d_j(m),
 * P(X, a, b) the cheapest group sequence from a to b visiting each group of X once
 * (P(X, a, a) unbounded once X has two groups), W2(X, a) = min_b P(X, a, b),
 *   lb1 = min_{a,b in Xb} d_a(v) + P(Xb, a, b) + d_b(v),
 *   lb2 = max_{a in Xb} (d_a(v) + W2(Xb, a)) + min_{b in Xb} d_b(v).
 * Equal costs to oracle_gst_nonhop on random instances check that these rules never
 * remove an optimal tree.  Outputs: cost (-1 infeasible), star (-1 none), pops. */
int oracle_nonhop_bound_check(int64_t V, const int64_t* beg, const int32_t* adj,
                              const int32_t* w, const int64_t* grp_ptr, const int32_t* members,
                              int32_t k, const int32_t* group_ids, int64_t* cost, int64_t* star,
                              int64_t* pops) {
  if (k < 1 || k > 8) return 1;
  const int32_t W = 1 << k, FULL = W - 1;
  uint32_t* mask = query_masks(V, grp_ptr, members, k, group_ids);
  int64_t* d = (int64_t*)malloc(sizeof(int64_t) * (size_t)(V * k));  /* d[i * V + v] */
  int64_t* c = (int64_t*)malloc(sizeof(int64_t) * (size_t)(V * W));
  int64_t* P = (int64_t*)malloc(sizeof(int64_t) * (size_t)W * 64);   /* P[X][a][b] */
  if (!mask || !d || !c || !P) return 2;
  for (int32_t i = 0; i < k; i++) {
    const int32_t g = group_ids[i];
    oracle_sssp_groups(V, beg, adj, w, grp_ptr[g + 1] - grp_ptr[g], members + grp_ptr[g],
                       d + (int64_t)i * V);
  }
  int64_t vv[8][8];
  for (int32_t i = 0; i < k; i++)
    for (int32_t j = 0; j < k; j++) {
      vv[i][j] = ORACLE_INF;
      const int32_t g = group_ids[i];
      for (int64_t m = grp_ptr[g]; m < grp_ptr[g + 1]; m++)
        if (d[(int64_t)j * V + members[m]] < vv[i][j]) vv[i][j] = d[(int64_t)j * V + members[m]];
    }
  for (int64_t x = 0; x < (int64_t)W * 64; x++) P[x] = ORACLE_INF;
  for (int32_t X = 1; X <= FULL; X++)
    for (int32_t a = 0; a < k; a++) {
      if (!(X >> a & 1)) continue;
      for (int32_t b = 0; b < k; b++) {
        if (!(X >> b & 1)) continue;
        int64_t val = ORACLE_INF;
        if (X == (1 << a)) {
          val = 0;
        } else if (b != a) {
          const int32_t prev = X ^ (1 << b);
          for (int32_t j = 0; j < k; j++)
            if ((prev >> j & 1) && P[(int64_t)prev * 64 + a * 8 + j] < ORACLE_INF &&
                vv[j][b] < ORACLE_INF && P[(int64_t)prev * 64 + a * 8 + j] + vv[j][b] < val)
              val = P[(int64_t)prev * 64 + a * 8 + j] + vv[j][b];
        }
        P[(int64_t)X * 64 + a * 8 + b] = val;
      }
    }
  int64_t ub = ORACLE_INF;
  for (int64_t v = 0; v < V; v++) {
    int64_t s = 0;
    for (int32_t i = 0; i < k && s < ORACLE_INF; i++)
      s = d[(int64_t)i * V + v] >= ORACLE_INF ? ORACLE_INF : s + d[(int64_t)i * V + v];
    if (s < ub) ub = s;
  }
  *star = ub < ORACLE_INF ? ub : -1;
#define DV(i, v) (d[(int64_t)(i) * V + (v)])
  for (int64_t i = 0; i < V * W; i++) c[i] = ORACLE_INF;
  heap_t h = {0};
  for (int64_t v = 0; v < V; v++)
    for (int32_t i = 0; i < k; i++)
      if (mask[v] >> i & 1) {
        c[v * W + (1 << i)] = 0;
        hitem it = {0, (int32_t)v, 1 << i, 0};
        heap_push(&h, it);
      }
  int64_t npop = 0, best = -1;
  while (h.n) {
    hitem it = heap_pop(&h);
    const int32_t v = it.v, p = it.p;
    const int64_t cv = it.key;
    if (cv != c[(int64_t)v * W + p]) continue;
    npop++;
    if (p == FULL) {
      best = cv;
      break;
    }
    const int32_t Xb = FULL ^ p;
    /* bounds at the source */
    int64_t one = 0, mind = ORACLE_INF, lb1 = ORACLE_INF, lb2 = 0;
    for (int32_t i = 0; i < k; i++)
      if (Xb >> i & 1) {
        if (DV(i, v) > one) one = DV(i, v);
        if (DV(i, v) < mind) mind = DV(i, v);
      }
    for (int32_t a = 0; a < k; a++) {
      if (!(Xb >> a & 1)) continue;
      int64_t w2 = ORACLE_INF;
      for (int32_t b = 0; b < k; b++)
        if ((Xb >> b & 1) && P[(int64_t)Xb * 64 + a * 8 + b] < w2) w2 = P[(int64_t)Xb * 64 + a * 8 + b];
      const int64_t t2 = DV(a, v) + w2 + mind;
      if (t2 > lb2) lb2 = t2;
      for (int32_t b = 0; b < k; b++)
        if (Xb >> b & 1) {
          const int64_t t1 = DV(a, v) + P[(int64_t)Xb * 64 + a * 8 + b] + DV(b, v);
          if (t1 < lb1) lb1 = t1;
        }
    }
    const int64_t tb = lb1 > lb2 ? lb1 : lb2;
    const int grow = 2 * cv <= ub && cv + one <= ub && cv + (tb + 1) / 2 <= ub;
    if (grow)
      for (int64_t e = beg[v]; e < beg[v + 1]; e++) {
        const int32_t u = adj[e];
        const int64_t nc = cv + w[e];
        if (nc > ub || c[(int64_t)u * W + p] <= nc) continue;
        /* the grow-time test on the target */
        int64_t oneu = 0, mindu = ORACLE_INF, lb2u = 0;
        for (int32_t i = 0; i < k; i++)
          if (Xb >> i & 1) {
            if (DV(i, u) > oneu) oneu = DV(i, u);
            if (DV(i, u) < mindu) mindu = DV(i, u);
          }
        for (int32_t a = 0; a < k; a++) {
          if (!(Xb >> a & 1)) continue;
          int64_t w2 = ORACLE_INF;
          for (int32_t b = 0; b < k; b++)
            if ((Xb >> b & 1) && P[(int64_t)Xb * 64 + a * 8 + b] < w2) w2 = P[(int64_t)Xb * 64 + a * 8 + b];
          const int64_t t2 = DV(a, u) + w2 + mindu;
          if (t2 > lb2u) lb2u = t2;
        }
        if (nc + oneu > ub || nc + (lb2u + 1) / 2 > ub) continue;
        c[(int64_t)u * W + p] = nc;
        hitem ni = {nc, u, p, 0};
        heap_push(&h, ni);
      }
    for (int32_t p2 = 1; p2 <= FULL; p2++) {
      if (p2 & p) continue;
      const int64_t c2 = c[(int64_t)v * W + p2];
      if (c2 >= ORACLE_INF) continue;
      const int32_t q = p | p2;
      const int64_t nc = cv + c2;
      if (q != FULL && 3 * nc > 2 * ub) continue;
      if (c[(int64_t)v * W + q] > nc) {
        c[(int64_t)v * W + q] = nc;
        hitem ni = {nc, v, q, 0};
        heap_push(&h, ni);
      }
    }
  }
#undef DV
  *cost = best;
  *pops = npop;
  free(h.a);
  free(mask);
  free(d);
  free(c);
  free(P);
  return 0;
}
