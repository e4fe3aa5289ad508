"""Host logic of bench.py on CPU: the workloads' hop mixing and the byte model of the
roofline figure."""
import os
import sys
from types import SimpleNamespace

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
import bench  # noqa: E402


def test_mix_queries_is_seeded_and_keeps_large_k_unbounded():
    rng = np.random.default_rng(1)
    pools = [[rng.choice(100, k, replace=False) for _ in range(200)] for k in (3, 5, 8)]
    q1, h1 = bench.mix_queries(pools, (4, 0.3, 99), kmax=7)
    q2, h2 = bench.mix_queries(pools, (4, 0.3, 99), kmax=7)
    assert [list(a) for a in q1] == [list(b) for b in q2] and h1 == h2
    assert sorted(len(q) for q in q1) == sorted(len(q) for p in pools for q in p)
    assert all(h is None for q, h in zip(q1, h1) if len(q) == 8)
    small = [h for q, h in zip(q1, h1) if len(q) <= 7]
    frac = sum(h == 4 for h in small) / len(small)
    assert 0.2 < frac < 0.4
    # without a size cap the same draws bound the same share of every k
    _, h3 = bench.mix_queries(pools, (4, 0.3, 99))
    assert sum(h == 4 for h in h3) >= sum(h == 4 for h in h1)


def test_level_bytes_follows_the_item_form():
    def ans(**st):
        return SimpleNamespace(stats=st)
    a = ans(sssp_relaxations=1000, states_expanded=10, edge_relaxations=100, rows_merged=5)
    q5 = [0, 1, 2, 3, 4]
    # unbounded, one cost bucket: group-mask items, 8 B edge + 4k B distances
    b = bench.level_bytes([a], [q5], [None], 0)
    assert b["k_sssp"] == (8 + 4 * 5) * 1000
    assert b["k_grow"] == 24 * 10 + 16 * 100
    assert b["k_rows"] == 16 * (1 << 5) * 5
    # cost buckets: one item per (vertex, group), 16 B per relaxation
    assert bench.level_bytes([a], [q5], [None], 3)["k_sssp"] == 16 * 1000
    # hop-bounded: group-mask rounds whatever the bucket width; rows of 2^k (D+1) cells
    b = bench.level_bytes([a], [q5], [4], 3)
    assert b["k_sssp"] == (8 + 4 * 5) * 1000
    assert b["k_rows"] == 16 * (1 << 5) * 5 * 5


def test_solver_stream_timing_and_budget(tmp_path):
    """The reference solvers are timed per query from their own output lines and stopped
    at the budget: a stand-in solver prints the reference drivers' lines."""
    exe = tmp_path / "solver.sh"
    exe.write_text("#!/bin/sh\nsleep 0.3\n"
                   "for i in 0 1 2 3 4 5 6 7; do echo \"w iteration $i\"; sleep 0.2; "
                   "echo \"cpu_cost $((10 + i))\"; echo '------'; done\n")
    exe.chmod(0o755)
    recs, load, window = bench.run_solver_streaming(str(exe), str(tmp_path), "w", 5, 8, None, 0.9)
    assert 0.25 < load < 2.0
    assert 0.85 < window < 1.5, window
    assert 2 <= len(recs) <= 5, recs
    assert [r[0] for r in recs] == list(range(len(recs)))
    assert [r[1] for r in recs] == [10 + i for i in range(len(recs))]
    assert all(0.15 < r[2] < 1.0 for r in recs)


def test_workload_stream_is_the_same_from_pools_and_arms():
    """Both arms build the query stream from the same pools: mixing, D cycling, k
    interleaving; the config object names the workload only."""
    rng = np.random.default_rng(3)
    pools = [rng.integers(0, 50, size=(20, k)).astype(np.int32) for k in (3, 5)]
    w4 = dict(bench.WORKLOADS["c4"])
    q1, h1 = bench.workload_queries(w4, pools)
    q2, h2 = bench.workload_queries(w4, [p.copy() for p in pools])
    assert [list(a) for a in q1] == [list(b) for b in q2] and h1 == h2
    w3 = dict(bench.WORKLOADS["c3"])
    q3, h3 = bench.workload_queries(w3, pools)
    assert h3[:4] == [3, 4, 5, 3] and [len(q) for q in q3[:4]] == [3, 5, 3, 5]
    cfg = bench.workload_config(w4, 100, 400, q1, h1, 32, 1)
    assert cfg["parallelism"] == "replicas1" and cfg["global_batch"] == 32
    assert "tuning" not in cfg and "autotuned" not in cfg
    order = bench.timed_order(40, 2, 3, 8, 0, 1)
    assert order == [(24 + i) % 40 for i in range(8)] + [(32 + i) % 40 for i in range(8)]


def test_gen_args_match_the_library_generator(tmp_path):
    """gst_gen (standalone, no engine library) writes the workload the engine arm builds
    through the library: same CSR, groups and query pools."""
    import subprocess
    import gst_b200 as G
    gen = os.path.join(bench.PKG, "gst_gen")
    if not os.path.exists(gen):
        subprocess.check_call([sys.executable, os.path.join(bench.PKG, "build.py")])
    w = {"graph": ("rmat", 3000, 12000, 77), "groups": ("zipf", 200, 1.5, 2, 100, 78),
         "queries": [(4, 10, 83), (5, 6, 84)]}
    subprocess.check_call([gen, str(tmp_path), "w"] + bench.gen_args(w), stdout=subprocess.DEVNULL)
    g = G.synth_rmat(3000, 12000, 77)
    h = G.read_reference_bin(str(tmp_path), "w")
    assert np.array_equal(g.beg_pos, h.beg_pos) and np.array_equal(g.adj, h.adj)
    assert np.array_equal(g.weight, h.weight)
    grp = G.synth_groups_zipf(g.V, 200, 1.5, 2, 100, 78)
    rg = G.read_reference_groups(str(tmp_path / "w.g"))
    assert np.array_equal(grp.grp_ptr, rg.grp_ptr) and np.array_equal(grp.members, rg.members)
    for k, n, s in w["queries"]:
        pool = np.loadtxt(tmp_path / f"w_pool{k}.txt", dtype=np.int32, ndmin=2)
        assert np.array_equal(pool, G.synth_queries(grp.n_groups, n, k, s))
