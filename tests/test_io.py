"""Reference file formats, synthetic inputs and the tree verifier (CPU)."""
import os

import numpy as np
import pytest

import gst_b200 as G
import oracle as O


def test_synth_deterministic():
    a = G.synth_rmat(5000, 20000, 123)
    b = G.synth_rmat(5000, 20000, 123)
    assert (a.beg_pos == b.beg_pos).all() and (a.adj == b.adj).all() and (a.weight == b.weight).all()
    c = G.synth_rmat(5000, 20000, 124)
    assert a.E != c.E or (a.adj != c.adj).any()


def test_synth_graph_properties():
    g = G.synth_rmat(5000, 20000, 5)
    deg = np.diff(g.beg_pos)
    assert g.E == 2 * 20000 or g.E < 2 * 20000  # largest component kept
    # simple, symmetric, sorted, weights in range
    for v in range(0, g.V, 97):
        nb = g.adj[g.beg_pos[v]:g.beg_pos[v + 1]]
        assert (np.diff(nb) > 0).all() and (nb != v).all()
    assert g.weight.min() >= 1 and g.weight.max() <= 100
    src = np.repeat(np.arange(g.V), deg)
    fwd = set(zip(src.tolist(), g.adj.tolist(), g.weight.tolist()))
    assert all((v, u, w) in fwd for (u, v, w) in list(fwd)[:5000])
    ba = G.synth_ba(2000, 4, 9)
    assert ba.E == 2 * (10 + 4 * (2000 - 5))


def test_groups_and_queries():
    grp = G.synth_groups_zipf(10000, 500, 1.5, 2, 200, 3)
    sizes = np.diff(grp.grp_ptr)
    assert sizes.min() >= 2 and sizes.max() <= 200
    assert (sizes == 2).mean() > 0.3  # Zipf(1.5) clamped: heavy mass at 2
    for gi in range(grp.n_groups):
        m = grp.members[grp.grp_ptr[gi]:grp.grp_ptr[gi + 1]]
        assert (np.diff(m) > 0).all()
    q = G.synth_queries(grp.n_groups, 50, 7, 4)
    assert q.shape == (50, 7)
    assert all(len(set(r)) == 7 for r in q.tolist())


def test_reference_format_roundtrip(tmp_path):
    g = G.synth_ba(300, 3, 11)
    grp = G.synth_groups_uniform(g.V, 20, 2, 9, 12)
    q = G.synth_queries(grp.n_groups, 5, 3, 13)
    d = str(tmp_path)
    G.write_reference_files(d, "t", g, grp, q)
    for suf in (".in", "_beg_pos.bin", "_csr.bin", "_weight.bin", ".g", "3.csv"):
        assert os.path.exists(os.path.join(d, "t" + suf))
    g2 = G.read_reference_bin(d, "t")
    g3 = G.read_reference_in(os.path.join(d, "t.in"))
    for x in (g2, g3):
        assert (x.beg_pos == g.beg_pos).all() and (x.adj == g.adj).all() and (x.weight == g.weight).all()
    grp2 = G.read_reference_groups(os.path.join(d, "t.g"))
    assert (grp2.grp_ptr == grp.grp_ptr).all() and (grp2.members == grp.members).all()
    q2 = G.read_reference_queries(os.path.join(d, "t3.csv"))
    assert (q2 == q).all()


def test_reader_accepts_reference_quirks(tmp_path):
    # trailing spaces (stripped by read_group.hpp:21-24) and 1-based ids
    p = tmp_path / "x.g"
    p.write_text("g1:5 3 \ng2:7\n")
    grp = G.read_reference_groups(str(p))
    assert grp.n_groups == 2 and grp.members.tolist() == [3, 5, 7]
    p = tmp_path / "x3.csv"
    p.write_text("0 1 \n1 0 \n")
    assert G.read_reference_queries(str(p)).tolist() == [[0, 1], [1, 0]]


def test_verifier_catches_planted_mistakes():
    g = G.synth_rmat(2000, 8000, 21)
    grp = G.synth_groups_zipf(g.V, 100, 1.5, 2, 50, 22)
    q = G.synth_queries(grp.n_groups, 5, 4, 23)
    for qi in range(5):
        o = O.gst_nonhop(g, grp, q[qi])
        if o["cost"] <= 0 or len(o["edges"]) < 2:
            continue
        e = o["edges"]
        assert G.verify_tree(g, grp, q[qi], -1, o["cost"], e, o["root"]) == 0
        assert G.verify_tree(g, grp, q[qi], -1, o["cost"] + 1, e, o["root"]) == 4
        bad = e.copy()
        bad[0, 2] += 1
        assert G.verify_tree(g, grp, q[qi], -1, o["cost"], bad, o["root"]) == 1
        assert G.verify_tree(g, grp, q[qi], -1, o["cost"] - e[0, 2], e[1:], o["root"]) in (2, 3)
        dup = np.concatenate([e, e[:1]])
        assert G.verify_tree(g, grp, q[qi], -1, o["cost"] + e[0, 2], dup, o["root"]) == 6
        assert G.verify_tree(g, grp, q[qi], 0, o["cost"], e, o["root"]) == 5
