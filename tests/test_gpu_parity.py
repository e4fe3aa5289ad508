"""Engine parity on the GPU: optimal costs bit-exact against the reference's own
CPU solvers (golden fixtures) and the oracle, every returned tree verified
(connected, covers the queried groups, hop-feasible, weight sum == cost)."""
import numpy as np
import pytest

import gst_b200 as G
import oracle as O
from conftest import golden_inputs, known_answer_graphs, load_golden

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


def consensus(case):
    """Per query of a fixture case, the cost every solver that answered it printed
    (None when none did); solvers that disagree fail the test."""
    out = []
    for i in range(len(case["queries"])):
        vals = {s: c[i] for s, c in case["ref"].items() if i < len(c) and c[i] is not None}
        assert len(set(vals.values())) <= 1, (case["k"], case["hop"], i, vals)
        out.append(next(iter(vals.values())) if vals else None)
    return out


SMALL_FIXTURES = ["c1_ba20k_k3", "rmat3k_k4_k5", "rmat20k_k6", "rmat50k_hop", "rmat4k_k7_k8",
                  "rmat4k_k8_D4"]
# the benchmark configurations themselves (mid-scale plain path, diameter-bounded path,
# batched configuration), a sample of their queries each
BENCH_FIXTURES = ["c2_rmat170k_k5k7", "c3_rmat1M_k5_D345", "c4_rmat4M_k357"]


@pytest.mark.parametrize("name", SMALL_FIXTURES + BENCH_FIXTURES)
def test_engine_matches_reference_golden(engine, name):
    """Every query a fixture's reference solvers answered, one at a time and in one
    batch (each solver's cost is the same, checked by consensus())."""
    fx = load_golden(name)
    g, grp = golden_inputs(fx)
    dg = engine.graph(g, grp)
    try:
        qs, hops, want = [], [], []
        for case in fx["cases"]:
            for q, c in zip(case["queries"], consensus(case)):
                if c is not None:
                    qs.append(q)
                    hops.append(case["hop"])
                    want.append(_ref(c))
        assert qs
        single = name in SMALL_FIXTURES or len(qs) <= 32
        if single:
            for q, h, c in zip(qs, hops, want):
                _check(g, grp, q, h, dg.solve(q, h), c)
        for i in range(0, len(qs), 32):
            for q, h, a, c in zip(qs[i:i + 32], hops[i:i + 32],
                                  dg.solve_batch(qs[i:i + 32], hops[i:i + 32]), want[i:i + 32]):
                _check(g, grp, q, h, a, c)
    finally:
        dg.close()


def test_engine_known_answers(engine):
    for g, grp, cases in known_answer_graphs():
        dg = engine.graph(g, grp)
        for c in cases:
            _check(g, grp, c["q"], c["hop"], dg.solve(c["q"], c["hop"]), c["cost"])
        dg.close()


def test_engine_matches_oracle_random(engine):
    rng = np.random.default_rng(5)
    for trial in range(4):
        g = G.synth_rmat(1500 + 500 * trial, 6000 + 3000 * trial, 100 + trial)
        grp = G.synth_groups_zipf(g.V, 120, 1.5, 2, 60, 200 + trial)
        dg = engine.graph(g, grp)
        for k in (1, 2, 3, 5, 6):
            qs = G.synth_queries(grp.n_groups, 4, k, 300 + trial * 10 + k)
            for q in qs:
                hop = None if rng.random() < 0.5 else int(rng.integers(1, 5))
                o = O.gst_nonhop(g, grp, q) if hop is None else O.gst_hop(g, grp, q, hop)
                _check(g, grp, q, hop, dg.solve(q, hop), o["cost"])
        dg.close()


def test_batch_equals_single(engine):
    """Each result is the same alone and in the mix (continuous batching refills
    slots at level boundaries while other queries are in flight)."""
    fx = load_golden("rmat3k_k4_k5")
    g, grp = golden_inputs(fx)
    dg = engine.graph(g, grp)
    qs, hops = [], []
    for case in fx["cases"]:
        for q in case["queries"][:12]:
            qs.append(q)
            hops.append(case["hop"])
    single = [dg.solve(q, h) for q, h in zip(qs, hops)]
    mixed = dg.solve_batch(qs, hops)
    for q, h, a, b in zip(qs, hops, single, mixed):
        assert a.status == b.status and (not a.ok or a.cost == b.cost), (q, h)
        if b.ok:
            assert G.verify_tree(g, grp, q, -1 if h is None else h, b.cost, b.edges, b.root) == 0
    dg.close()


def test_bad_input_is_reported(engine):
    g = G.synth_ba(200, 2, 1)
    grp = G.synth_groups_uniform(g.V, 10, 2, 5, 2)
    dg = engine.graph(g, grp)
    assert dg.solve([0, 0]).status == G.BAD_INPUT        # duplicate group
    assert dg.solve([0, 99]).status == G.BAD_INPUT       # unknown group
    assert dg.solve(list(range(9))).status == G.BAD_INPUT  # k > 8
    res = dg.solve_batch([[0, 1], [0, 0], [2, 3]])
    assert res[1].status == G.BAD_INPUT and res[0].ok and res[2].ok
    dg.close()


@pytest.mark.parametrize("delta", [1, 3, 16])
def test_cost_buckets_match_reference(delta):
    """Cost-ordered frontiers (edges relaxed lazily, bucket by bucket) give the same
    optimum as the unordered frontier and the reference's solvers."""
    eng = G.Engine(0, bucket_delta=delta, max_batch=8)
    try:
        fx = load_golden("rmat3k_k4_k5")
        g, grp = golden_inputs(fx)
        dg = eng.graph(g, grp)
        qs, hops, want = [], [], []
        for case in fx["cases"]:
            costs = next(iter(case["ref"].values()))
            for q, c in zip(case["queries"], costs):
                qs.append(q)
                hops.append(case["hop"])
                want.append(_ref(c))
        for q, h, a, w in zip(qs, hops, dg.solve_batch(qs, hops), want):
            _check(g, grp, q, h, a, w)
        for q, h, w in list(zip(qs, hops, want))[::7]:
            _check(g, grp, q, h, dg.solve(q, h), w)
        dg.close()
        g = G.synth_rmat(2500, 12000, 77)
        grp = G.synth_groups_zipf(g.V, 100, 1.5, 2, 50, 78)
        dg = eng.graph(g, grp)
        for k in (3, 6):
            for q in G.synth_queries(grp.n_groups, 3, k, 79 + k):
                _check(g, grp, q, None, dg.solve(q), O.gst_nonhop(g, grp, q)["cost"])
        dg.close()
    finally:
        eng.close()


def test_overlapping_groups_match_oracle(engine):
    """Groups that share member vertices: a vertex that starts the distance search
    for several queried groups at once (several frontier bits set by one launch),
    and groups nested in others.  Unbounded queries (group-mask distance items),
    D = 0 (a single-vertex tree or none) and hop-bounded ones (group items) in one
    batch, against the oracle and against each query solved alone."""
    rng = np.random.default_rng(41)
    g = G.synth_rmat(2500, 12000, 42)
    base = [rng.choice(g.V, size=int(rng.integers(2, 30)), replace=False) for _ in range(12)]
    lists = []
    for i, m in enumerate(base):
        lists.append(sorted(set(m.tolist())))
        # a group sharing half of its members with the previous one, and a subset
        other = base[i - 1]
        lists.append(sorted(set(m[: len(m) // 2].tolist()) | set(other[: len(other) // 2].tolist())))
        lists.append(sorted(set(m[:1].tolist())))
    grp = G.Groups.from_lists(lists)
    dg = engine.graph(g, grp)
    qs, hops, want = [], [], []
    for t in range(24):
        k = int(rng.integers(1, 7))
        q = rng.choice(len(lists), size=k, replace=False).astype(np.int32)
        hop = [None, None, 0, 2, 3][t % 5]
        if t % 10 == 2:
            # three groups sharing one vertex: a zero-cost tree, for D = 0 and unbounded
            i = int(rng.integers(0, len(base)))
            q = np.array([3 * i, 3 * i + 1, 3 * i + 2], dtype=np.int32)
            hop = 0 if t % 20 == 2 else None
        o = O.gst_nonhop(g, grp, q) if hop is None else O.gst_hop(g, grp, q, hop)
        qs.append(q)
        hops.append(hop)
        want.append(o["cost"])
    alone = [dg.solve(q, h) for q, h in zip(qs, hops)]
    mixed = dg.solve_batch(qs, hops)
    try:
        for q, h, a, b, c in zip(qs, hops, alone, mixed, want):
            _check(g, grp, q, h, a, c)
            _check(g, grp, q, h, b, c)
    finally:
        dg.close()


def test_hop_budgets_match_oracle(engine):
    """Hop-bounded queries over the whole range of bounds: the per-height distance
    budgets (D - 1 of them up to 7 kept, the rest falling back to the full hop
    bound), the star of D/2-edge paths as the first bound, D = 1 (budget 0, the
    members themselves) and D = 0."""
    rng = np.random.default_rng(77)
    for trial in range(3):
        if trial == 1:
            g = G.synth_ba(1200, 2, 500 + trial)
        else:
            g = G.synth_rmat(1500, 7000, 500 + trial)
        grp = G.synth_groups_zipf(g.V, 80, 1.5, 1, 40, 600 + trial)
        dg = engine.graph(g, grp)
        qs, hops, want = [], [], []
        for D in (0, 1, 2, 3, 5, 6, 9):
            for k in (2, 4, 6):
                q = G.synth_queries(grp.n_groups, 1, k, int(rng.integers(1, 1 << 30)))[0]
                qs.append(q)
                hops.append(D)
                want.append(O.gst_hop(g, grp, q, D)["cost"])
        try:
            for q, h, c in zip(qs, hops, want):
                _check(g, grp, q, h, dg.solve(q, h), c)
            for q, h, a, c in zip(qs, hops, dg.solve_batch(qs, hops), want):
                _check(g, grp, q, h, a, c)
        finally:
            dg.close()


def test_wide_rows_match_oracle(engine):
    """Rows of 2^k x (D+1) cells wider than eight warps' shared memory in the rows kernel
    (k = 8 at D = 7: 2,048 cells; k = 7 at D = 14: 1,920 cells): the kernel runs fewer
    warps per CTA.  Alone, and mixed into one batch with narrow queries, against the
    oracle."""
    rng = np.random.default_rng(907)
    g = G.synth_rmat(500, 2500, 901)
    grp = G.synth_groups_zipf(g.V, 60, 1.5, 1, 12, 902)
    dg = engine.graph(g, grp)
    qs, hops, want = [], [], []
    for k, D in ((8, 7), (7, 14), (3, None), (4, 2), (8, 7)):
        q = rng.choice(grp.n_groups, size=k, replace=False).astype(np.int32)
        qs.append(q)
        hops.append(D)
        want.append(O.gst_nonhop(g, grp, q)["cost"] if D is None else O.gst_hop(g, grp, q, D)["cost"])
    try:
        for q, h, c in zip(qs, hops, want):
            _check(g, grp, q, h, dg.solve(q, h), c)
        for q, h, a, c in zip(qs, hops, dg.solve_batch(qs, hops), want):
            _check(g, grp, q, h, a, c)
    finally:
        dg.close()


@pytest.mark.parametrize("permille", [250, 500])
def test_search_cutoff_keeps_optima(permille):
    """A distance search stopped below the star bound (search_cut_permille < 1000) leaves
    distances above its cutoff clamped to cutoff + 1, weaker but still valid bounds: the
    optima stay the reference's, alone and in a batch."""
    eng = G.Engine(0, search_cut_permille=permille, hop_cut_permille=permille, max_batch=16)
    try:
        for name in ("rmat3k_k4_k5", "rmat4k_k7_k8", "c1_ba20k_k3", "rmat50k_hop", "rmat4k_k8_D4"):
            fx = load_golden(name)
            g, grp = golden_inputs(fx)
            dg = eng.graph(g, grp)
            qs, hops, want = [], [], []
            for case in fx["cases"]:
                for q, c in list(zip(case["queries"], consensus(case)))[:12]:
                    if c is not None:
                        qs.append(q)
                        hops.append(case["hop"])
                        want.append(_ref(c))
            for q, h, a, c in zip(qs, hops, dg.solve_batch(qs, hops), want):
                _check(g, grp, q, h, a, c)
            for q, h, c in list(zip(qs, hops, want))[::5]:
                _check(g, grp, q, h, dg.solve(q, h), c)
            dg.close()
    finally:
        eng.close()


def test_shared_search_matches_alone(engine):
    """The queries of a batch search their groups' distances together, one search per
    kind (unbounded, or one hop bound D: D tables of paths of at most 1..D edges), at most
    256 groups and 64 queries per search, and a lone query runs the same kernels: every
    optimum equals the query solved alone with its own group-mask search and the
    oracle's, and the trees verify."""
    rng = np.random.default_rng(61)
    g = G.synth_rmat(3000, 14000, 62)
    grp = G.synth_groups_zipf(g.V, 400, 1.5, 1, 60, 63)
    kinds = [None, None, None, 3, 2, 4, 1]
    qs, hops = [], []
    for t in range(100):
        k = int(rng.integers(2, 7))
        qs.append(rng.choice(grp.n_groups, size=k, replace=False).astype(np.int32))
        hops.append(kinds[t % len(kinds)])
    # alone: every query with its own group-mask search (the shared search off)
    own = G.Engine(0, batch_search=0)
    dgo = own.graph(g, grp)
    try:
        alone = [dgo.solve(q, h) for q, h in zip(qs, hops)]
        assert all(a.stats["shared_launches"] == 0 for a in alone)
    finally:
        dgo.close()
        own.close()
    dg = engine.graph(g, grp)
    try:
        # a lone query runs the shared kernels too, with its own cutoff
        lone = [dg.solve(q, h) for q, h in list(zip(qs, hops))[:21]]
        assert all(a.stats["shared_launches"] > 0 for a in lone)
        for a, b in zip(alone, lone):
            assert a.status == b.status and (not a.ok or a.cost == b.cost), (a.cost, b.cost)
        mixed = dg.solve_batch(qs, hops)
        assert mixed[0].stats["shared_launches"] > 0
        for q, h, a, b in zip(qs, hops, alone, mixed):
            assert a.status == b.status and (not a.ok or a.cost == b.cost), (q, h, a.cost, b.cost)
            if b.ok:
                assert G.verify_tree(g, grp, q, -1 if h is None else h, b.cost, b.edges, b.root) == 0
        for q, h, b in list(zip(qs, hops, mixed))[:14]:
            o = O.gst_nonhop(g, grp, q) if h is None else O.gst_hop(g, grp, q, h)
            assert (b.cost if b.ok else -1) == o["cost"], (q, h)
        # a batch of one hop bound alone: its search is shared
        hq = [q for q, h in zip(qs, hops) if h == 3]
        hb = dg.solve_batch(hq, [3] * len(hq))
        assert hb[0].stats["shared_launches"] > 0
        for q, a, b in zip(hq, [a for a, h in zip(alone, hops) if h == 3], hb):
            assert a.status == b.status and (not a.ok or a.cost == b.cost), (q, a.cost, b.cost)
    finally:
        dg.close()
