"""Shared test setup.

Markers:
  gpu  — needs a CUDA device (runs the engine); everything else runs on the CPU.

The engine library and the oracle are built on first use (nvcc cross-compiles for
sm_100a without a GPU).  GPU tests fail loudly if the engine cannot start: there
is no CPU fallback to pass silently on.
"""
import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "gpu4gst-sigmod-fullexp_b200")
ORACLE = os.path.join(ROOT, "oracle")
GOLDEN = os.path.join(ROOT, "tests", "golden")
for p in (PKG, ORACLE, ROOT):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def _ensure_built():
    import subprocess
    if not os.path.exists(os.path.join(PKG, "libgst_b200.so")):
        subprocess.check_call([sys.executable, os.path.join(PKG, "build.py")])
    if not os.path.exists(os.path.join(ORACLE, "liboracle.so")):
        subprocess.check_call(["make", "-s", "-C", ORACLE, "liboracle.so"])


_ensure_built()


def load_golden(name):
    with open(os.path.join(GOLDEN, name + ".json")) as f:
        return json.load(f)


def golden_inputs(fx):
    """Regenerate the graph and groups of a golden fixture (and check the fingerprint)."""
    sys.path.insert(0, GOLDEN)
    import make_golden
    g, grp = make_golden.make_inputs(fx)
    assert make_golden.fingerprint(g, grp) == fx["fingerprint"], \
        f"generator output drifted for fixture {fx['name']}"
    return g, grp


def known_answer_graphs():
    import gst_b200 as G
    with open(os.path.join(GOLDEN, "known_answer.json")) as f:
        ka = json.load(f)
    out = []
    for gd in ka["graphs"]:
        V = gd["V"]
        adj = [[] for _ in range(V)]
        for u, v, w in gd["edges"]:
            adj[u].append((v, w))
            adj[v].append((u, w))
        beg = np.zeros(V + 1, dtype=np.int64)
        a, wt = [], []
        for u in range(V):
            for v, w in sorted(adj[u]):
                a.append(v)
                wt.append(w)
            beg[u + 1] = len(a)
        g = G.Graph(beg, np.array(a, dtype=np.int32), np.array(wt, dtype=np.int32))
        grp = G.Groups.from_lists(gd["groups"])
        out.append((g, grp, gd["cases"]))
    return out


@pytest.fixture(scope="session")
def engine():
    import gst_b200 as G
    eng = G.Engine(0)
    yield eng
    eng.close()
