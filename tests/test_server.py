"""Serving and batching on the GPU: continuous batching gives every query the same
answer as solving it alone; admission by state-table memory holds queries back
until memory frees up and refuses a query that can never fit; the CUDA-graph level
loop and the host-driven loop agree."""
import time

import numpy as np
import pytest

import gst_b200 as G
from conftest import golden_inputs, load_golden

pytestmark = pytest.mark.gpu


def _mixed_queries(grp, n, seed):
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        k = int(rng.integers(2, 7))
        q = rng.choice(grp.n_groups, size=k, replace=False).astype(np.int32)
        hop = None if rng.random() < 0.6 else int(rng.integers(2, 5))
        out.append((q, hop))
    return out


def _same(a, b):
    return a.status == b.status and (not a.ok or a.cost == b.cost)


def _verified(g, grp, q, hop, a):
    return G.verify_tree(g, grp, q, -1 if hop is None else hop, a.cost, a.edges, a.root) == 0


def test_server_results_equal_alone():
    g = G.synth_rmat(6000, 40000, 11)
    grp = G.synth_groups_zipf(g.V, 200, 1.5, 2, 80, 12)
    qs = _mixed_queries(grp, 40, 13)
    eng = G.Engine(0, max_batch=8)
    dg = eng.graph(g, grp)
    alone = [dg.solve(q, h) for q, h in qs]
    sv = dg.server()
    tickets = []
    # arrivals spread over time: later queries join while earlier ones run
    for i, (q, h) in enumerate(qs):
        tickets.append(sv.submit(q, h, tag=i))
        if i % 5 == 4:
            time.sleep(0.002)
    got = [sv.wait(t) for t in tickets]
    sv.close()
    for (q, h), a, b in zip(qs, alone, got):
        assert _same(a, b), (q, h, G.STATUS[a.status], G.STATUS[b.status], a.cost, b.cost)
        if b.ok:
            assert _verified(g, grp, q, h, b)
    assert [b.user_tag for b in got] == list(range(len(qs)))
    dg.close()
    eng.close()


def test_server_poll_and_bad_query():
    g = G.synth_ba(3000, 3, 21)
    grp = G.synth_groups_uniform(g.V, 50, 3, 10, 22)
    eng = G.Engine(0, max_batch=4)
    dg = eng.graph(g, grp)
    sv = dg.server()
    t_bad = sv.submit([1, 1])            # duplicate group id
    t_ok = sv.submit([0, 1, 2])
    assert sv.wait(t_bad).status == G.BAD_INPUT
    a = None
    for _ in range(20000):
        a = sv.poll(t_ok)
        if a is not None:
            break
        time.sleep(0.0005)
    assert a is not None and a.ok
    assert a.cost == dg.solve([0, 1, 2]).cost
    with pytest.raises(G.GstError):
        sv.poll(t_ok)                    # a ticket is forgotten once taken
    sv.close()
    dg.close()
    eng.close()


@pytest.mark.timeout(300)
def test_admission_by_memory():
    """A budget below one k=8 state table (2^8 x V x 8 bytes), which holds about
    three k=5 slots: queries wait for memory, all finish with the answers they get
    alone, and the k=8 query, which can never fit, is refused."""
    g = G.synth_rmat(20000, 120000, 31)
    grp = G.synth_groups_zipf(g.V, 300, 1.5, 2, 100, 32)
    budget = g.V * 256 * 8 - 1
    eng = G.Engine(0, max_batch=16, mem_budget_bytes=budget)
    dg = eng.graph(g, grp)
    qs = [q for q in G.synth_queries(grp.n_groups, 10, 5, 33)]
    alone = [dg.solve(q) for q in qs]
    big = G.synth_queries(grp.n_groups, 1, 8, 34)[0]
    sv = dg.server()
    ts = [sv.submit(q) for q in qs]
    tb = sv.submit(big)
    got = [sv.wait(t) for t in ts]
    assert sv.wait(tb).status == G.OOM_ADMISSION
    sv.close()
    for q, a, b in zip(qs, alone, got):
        assert _same(a, b), (q, a.cost, b.cost)
    dg.close()
    eng.close()


def test_graph_loop_matches_host_loop():
    fx = load_golden("rmat3k_k4_k5")
    g, grp = golden_inputs(fx)
    qs, hops = [], []
    for case in fx["cases"]:
        for q in case["queries"][:6]:
            qs.append(q)
            hops.append(case["hop"])
    res = {}
    for ug in (0, 1):
        eng = G.Engine(0, max_batch=8, use_graphs=ug)
        dg = eng.graph(g, grp)
        res[ug] = dg.solve_batch(qs, hops) + [dg.solve(q, h) for q, h in zip(qs[:4], hops[:4])]
        dg.close()
        eng.close()
    for a, b in zip(res[0], res[1]):
        assert _same(a, b)
