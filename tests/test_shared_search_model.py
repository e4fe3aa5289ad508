"""The batch-shared distance search's algorithm, restated step by step on the CPU (numpy),
against exact distances: the properties the DP relies on (CPU only; the kernels
themselves are checked on the GPU through the optimal costs).

- Unbounded: with per-column cutoffs that only decrease (the largest star x cut_pm /
  1000 among the queries of a column, stars found at the announced vertices before each
  relax step), every distance at most its column's final cutoff is exact and every
  other stored value is at least the exact one and above the cutoff.
- Hop-bounded (bound D): round r copies table r into table r + 1, then relaxes the
  vertices whose table-r row improved in round r - 1, from table r into table r + 1;
  table h then holds d^{<=h} exactly up to the cutoff, and the stars (from tables r with
  2r <= D) are costs of trees of diameter <= D.
"""
import numpy as np
import pytest

import gst_b200 as G

INF = np.uint64(1 << 40)


def exact_hop(beg, adj, w, src_sets, H):
    """d^{<=h} for h = 0..H per column (Bellman-Ford by edge count), shape (H+1, C, V)."""
    V = len(beg) - 1
    C = len(src_sets)
    out = np.full((H + 1, C, V), INF, dtype=np.uint64)
    for c, s in enumerate(src_sets):
        out[0, c, s] = 0
    tail = np.repeat(np.arange(V), np.diff(beg))
    for h in range(1, H + 1):
        cur = out[h - 1].copy()
        cand = out[h - 1][:, tail] + w[None, :].astype(np.uint64)
        for c in range(C):
            np.minimum.at(cur[c], adj, cand[c])
        out[h] = cur
    return out


def _bf(beg, adj, w, src_sets):
    V = len(beg) - 1
    C = len(src_sets)
    d = np.full((C, V), INF, dtype=np.uint64)
    for c, s in enumerate(src_sets):
        d[c, s] = 0
    tail = np.repeat(np.arange(V), np.diff(beg))
    while True:
        cand = d[:, tail] + w[None, :].astype(np.uint64)
        nd = d.copy()
        for c in range(C):
            np.minimum.at(nd[c], adj, cand[c])
        if np.array_equal(nd, d):
            return d
        d = nd


def model_search(beg, adj, w, src_sets, queries, D, cut_pm):
    """The shared search as the kernels run it (sequential within a step).  Returns the
    tables (one for D = 0, else tables 1..D), the final column cutoffs and the stars."""
    V = len(beg) - 1
    C = len(src_sets)
    ntab = max(D, 1)
    tab = np.full((ntab + 1, C, V), INF, dtype=np.uint64)  # tab[1..D] (tab[1] when D = 0)
    ann = np.zeros((C, V), dtype=bool)
    for c, s in enumerate(src_sets):
        tab[1, c, s] = 0
        ann[c, s] = True
    cutc = np.full(C, INF, dtype=np.uint64)
    star = np.full(len(queries), INF, dtype=np.uint64)

    def cut_update():
        for c in range(C):
            users = [star[q] for q, cols in enumerate(queries) if c in cols]
            if users:
                mx = max(u * np.uint64(cut_pm) // np.uint64(1000) if u < INF else INF for u in users)
                cutc[c] = min(cutc[c], mx)

    r = 0
    while ann.any():
        src = None if (D and r == 0) else (tab[r] if D else tab[1])
        if D and r >= 1:
            tab[r + 1] = tab[r].copy()
        dst = tab[r + 1] if D else tab[1]
        stars_ok = D == 0 or (r >= 1 and 2 * r <= D)
        verts = np.nonzero(ann.any(axis=0))[0]
        if stars_ok:
            for v in verts:
                for q, cols in enumerate(queries):
                    s = sum(int(src[c, v]) for c in cols)
                    if s < star[q]:
                        star[q] = s
            cut_update()
        act = ann.copy()
        ann[:] = False
        extend = D == 0 or r + 1 < D
        for v in verts:
            for c in np.nonzero(act[:, v])[0]:
                dv = np.uint64(0) if src is None else src[c, v]
                if dv >= cutc[c]:
                    continue
                for e in range(beg[v], beg[v + 1]):
                    nd = dv + np.uint64(w[e])
                    if nd <= cutc[c] and nd < dst[c, adj[e]]:
                        dst[c, adj[e]] = nd
                        if nd < cutc[c] and extend:
                            ann[c, adj[e]] = True
        cut_update()
        r += 1
        if D and r >= D:
            break
    if D:
        for h in range(r + 1, D + 1):
            tab[h] = tab[r].copy()
    return tab, cutc, star


@pytest.fixture(scope="module")
def small_graph():
    g = G.synth_rmat(400, 1600, 71)
    grp = G.synth_groups_zipf(g.V, 40, 1.5, 1, 12, 72)
    return g, grp


def _columns(grp, n):
    return [grp.members[grp.grp_ptr[i]:grp.grp_ptr[i + 1]] for i in range(n)]


@pytest.mark.parametrize("cut_pm", [1000, 750])
def test_unbounded_distances_exact_up_to_cutoff(small_graph, cut_pm):
    g, grp = small_graph
    cols = _columns(grp, 10)
    queries = [[0, 1, 2], [2, 3, 4, 5], [6, 7], [1, 8, 9, 4, 0]]
    beg, adj, w = g.beg_pos, g.adj, g.weight
    tab, cutc, star = model_search(beg, adj, w, cols, queries, 0, cut_pm)
    ex = _bf(beg, adj, w, cols)
    got = tab[1]
    assert (got >= ex).all()
    for c in range(len(cols)):
        inside = ex[c] <= cutc[c]
        assert np.array_equal(got[c][inside], ex[c][inside]), c
        assert (got[c][~inside] > cutc[c]).all(), c
    # every star is a feasible cost: at least the best star over exact distances
    for q, qc in enumerate(queries):
        best = min(sum(int(ex[c, v]) for c in qc) for v in range(g.V))
        assert star[q] >= best


@pytest.mark.parametrize("D", [1, 2, 3, 4])
def test_hop_tables_exact_up_to_cutoff(small_graph, D):
    g, grp = small_graph
    cols = _columns(grp, 8)
    queries = [[0, 1, 2], [3, 4], [5, 6, 7, 0]]
    beg, adj, w = g.beg_pos, g.adj, g.weight
    tab, cutc, star = model_search(beg, adj, w, cols, queries, D, 1000)
    ex = exact_hop(beg, adj, w, cols, D)
    for h in range(1, D + 1):
        assert (tab[h] >= ex[h]).all(), h
        for c in range(len(cols)):
            inside = ex[h][c] <= cutc[c]
            assert np.array_equal(tab[h][c][inside], ex[h][c][inside]), (h, c)
    # stars only from paths of at most D/2 edges: at least the best such star
    for q, qc in enumerate(queries):
        if star[q] < INF:
            half = ex[D // 2]
            best = min(sum(int(half[c, v]) for c in qc) for v in range(g.V))
            assert star[q] >= best
