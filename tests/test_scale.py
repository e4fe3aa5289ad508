"""Parity at the diameter-bounded configuration's full size (R-MAT 1M vertices, ~15M
undirected edges, 10,000 Zipf groups clipped to 2..1,000, k = 5, hop bounds 3, 4, 5),
where no reference run is affordable, through properties that do not depend on size:
every tree verifies (cost = weight of a connected tree covering the groups, diameter
within the bound); a larger bound never costs more (D = 3 >= D = 4 >= D = 5 >=
unbounded); batched and cached runs return the costs of single runs."""
import numpy as np
import pytest

import gst_b200 as G

pytestmark = pytest.mark.gpu


def _verified(g, grp, q, hop, a):
    return G.verify_tree(g, grp, q, -1 if hop is None else hop, a.cost, a.edges, a.root) == 0


@pytest.mark.timeout(900)
def test_diameter_bounded_full_size_properties(engine):
    g = G.synth_rmat(1_000_000, 15_000_000, 0x6057 + 3)
    grp = G.synth_groups_zipf(g.V, 10_000, 1.5, 2, 1000, 0x6057 + 1003)
    qs = G.synth_queries(grp.n_groups, 6, 5, 0x6057 + 2033)
    dg = engine.graph(g, grp)
    try:
        bounds = (3, 4, 5, None)
        single = {}
        for q in qs:
            for h in bounds:
                a = dg.solve(q, h)
                assert a.status in (G.OK, G.INFEASIBLE), (q, h, G.STATUS[a.status])
                if a.ok:
                    assert _verified(g, grp, q, h, a), (q, h)
                single[(tuple(q), h)] = a.cost if a.ok else None
            costs = [single[(tuple(q), h)] for h in bounds]
            # a looser bound admits every tree of a tighter one
            for tight, loose in zip(costs, costs[1:]):
                if tight is not None:
                    assert loose is not None and loose <= tight, (q, costs)
        allq = [q for q in qs for _ in bounds]
        allh = [h for _ in qs for h in bounds]
        for q, h, a in zip(allq, allh, dg.solve_batch(allq, allh)):
            assert (a.cost if a.ok else None) == single[(tuple(q), h)], (q, h)
        gids = sorted({int(x) for q in qs for x in q})
        assert dg.cache_warm(gids, 4 * g.V * len(gids)) == len(gids)
        for q in qs:
            a = dg.solve(q, None)
            assert a.stats["sssp_relaxations"] == 0
            assert (a.cost if a.ok else None) == single[(tuple(q), None)]
        dg.cache_warm([], 0)
    finally:
        dg.close()
