"""The one-label distance cache (gst_groups_cache_warm): queries whose groups are all
cached skip the distance search and still return the reference's optimal costs; partly
cached queries search for their other groups only; hop-bounded queries take the normal
path; replacement keeps the cache consistent; batches and the server use it too."""
import numpy as np
import pytest

import gst_b200 as G
from conftest import golden_inputs, load_golden

pytestmark = pytest.mark.gpu
REF_INF = 100000


def _ref(c):
    return -1 if c >= REF_INF else c


def _check(g, grp, q, hop, a, expect):
    got = a.cost if a.ok else (-1 if a.status == G.INFEASIBLE else None)
    assert got == expect, (q, hop, G.STATUS[a.status], a.cost, expect)
    if a.ok:
        rc = G.verify_tree(g, grp, q, -1 if hop is None else hop, a.cost, a.edges, a.root)
        assert rc == 0, (q, hop, G.VERIFY_CODES[rc])


def _cases(fx):
    out = []
    for case in fx["cases"]:
        costs = next(iter(case["ref"].values()))
        for q, c in zip(case["queries"], costs):
            out.append((q, case["hop"], _ref(c)))
    return out


def test_cached_groups_match_reference(engine):
    fx = load_golden("rmat3k_k4_k5")
    g, grp = golden_inputs(fx)
    dg = engine.graph(g, grp)
    try:
        cases = _cases(fx)
        unb = [(q, h, c) for q, h, c in cases if h is None][:30]
        gids = sorted({x for q, _, _ in unb for x in q})
        vb = 4 * g.V
        assert dg.cache_warm(gids, vb * len(gids)) == len(gids)
        for q, h, c in unb:
            a = dg.solve(q, h)
            _check(g, grp, q, h, a, c)
            assert a.stats["sssp_relaxations"] == 0  # no distance search ran
        # hop-bounded queries over the same groups take the normal path
        for q, h, c in [x for x in cases if x[1] is not None][:12]:
            a = dg.solve(q, h)
            _check(g, grp, q, h, a, c)
        # batched: every query's result equals the reference's
        qs = [q for q, _, _ in cases[:40]]
        hs = [h for _, h, _ in cases[:40]]
        for (q, h, c), a in zip(cases[:40], dg.solve_batch(qs, hs)):
            _check(g, grp, q, h, a, c)
        # the server takes cached queries as well
        sv = dg.server()
        ts = [sv.submit(q, h) for q, h, _ in unb[:10]]
        for (q, h, c), t in zip(unb[:10], ts):
            _check(g, grp, q, h, sv.wait(t), c)
        sv.close()
        assert dg.cache_warm([], 0) == 0  # frees the cache
        a = dg.solve(unb[0][0], None)
        _check(g, grp, unb[0][0], None, a, unb[0][2])
        # a distance search ran (a lone query's runs on the shared-search kernels)
        assert a.stats["sssp_relaxations"] + a.stats["shared_sectors"] > 0
    finally:
        dg.close()


def test_cache_replacement_and_partial_hits():
    """Replacement and partial hits with the per-query group-mask search (the shared
    search off), whose search covers only the groups not cached."""
    fx = load_golden("rmat20k_k6")
    g, grp = golden_inputs(fx)
    own = G.Engine(0, batch_search=0)
    dg = own.graph(g, grp)
    try:
        cases = [x for x in _cases(fx) if x[1] is None][:8]
        vb = 4 * g.V
        cap = 4
        q0 = cases[0][0]
        base = dg.solve(q0, None)
        _check(g, grp, q0, None, base, cases[0][2])
        # more groups listed than fit: the first `cap` stay
        assert dg.cache_warm(q0, vb * cap) == cap
        # k = 6 > cap: the search runs for the two groups not cached only
        a = dg.solve(q0, None)
        _check(g, grp, q0, None, a, cases[0][2])
        assert 0 < a.stats["sssp_relaxations"] <= base.stats["sssp_relaxations"]
        # every query warmed in turn, replacing the previous groups
        for q, h, c in cases[1:]:
            small = list(q[:cap])
            assert dg.cache_warm(small, vb * cap) == cap
            a = dg.solve(q, None)
            _check(g, grp, q, None, a, c)
        # a query of four cached groups skips the search
        q = list(cases[-1][0][:cap])
        want = dg.solve(q, None)
        dg.cache_warm([], 0)
        assert dg.cache_warm(q, vb * cap) == cap
        a = dg.solve(q, None)
        assert a.stats["sssp_relaxations"] == 0
        assert a.status == want.status and a.cost == want.cost
    finally:
        dg.close()
        own.close()


def test_hop_cache_matches_reference(engine):
    """Hop-bounded queries whose groups are all cached for their bound skip the distance
    search (every hop budget's table gathered) and return the reference's costs; other
    bounds, and queries with a group not cached, take the normal path."""
    for name in ("rmat3k_k4_k5", "rmat50k_hop"):
        fx = load_golden(name)
        g, grp = golden_inputs(fx)
        dg = engine.graph(g, grp)
        try:
            cases = [x for x in _cases(fx) if x[1] is not None and x[1] > 0]
            for D in sorted({h for _, h, _ in cases}):
                mine = [x for x in cases if x[1] == D][:10]
                gids = sorted({x for q, _, _ in mine for x in q})
                per = 4 * g.V * (min(D - 1, 7) + 1)
                assert dg.cache_warm_hop(gids, D, per * len(gids)) == len(gids)
                for q, h, c in mine:
                    a = dg.solve(q, h)
                    _check(g, grp, q, h, a, c)
                    assert a.stats["sssp_relaxations"] == 0
                qs = [q for q, _, _ in mine]
                for (q, h, c), a in zip(mine, dg.solve_batch(qs, [D] * len(qs))):
                    _check(g, grp, q, h, a, c)
                # a query with some groups cached runs a distance search (the shared
                # kernels, over all its groups)
                q, h, c = mine[0]
                dg.cache_warm_hop([], D, 0)
                assert dg.cache_warm_hop(list(q[:2]), D, per * len(gids)) == 2
                a = dg.solve(q, h)
                _check(g, grp, q, h, a, c)
                assert len(q) > 2 and a.stats["sssp_relaxations"] + a.stats["shared_sectors"] > 0
                # another bound is not served from this cache
                other = [x for x in cases if x[1] != D][:2]
                for q, h, c in other:
                    a = dg.solve(q, h)
                    _check(g, grp, q, h, a, c)
            dg.cache_warm_hop([], 1, 0)
        finally:
            dg.close()
