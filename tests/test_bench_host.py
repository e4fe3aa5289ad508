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
