"""Generate the golden fixtures in this directory by running the REFERENCE's own
CPU solvers (PrunedDP++, TrimCDP-multi-core-CPU, D-PrunedDP++ from
rucdatascience/GPU4GST-sigmod-fullEXP, compiled unmodified by oracle/Makefile into
oracle/_ref/) on seeded synthetic inputs written in the reference's file formats.

    make -C oracle ref && python tests/golden/make_golden.py

Each fixture records how to regenerate its inputs (generator + seeds), a
fingerprint of the generated arrays (so generator drift is caught), the queries,
and the costs the reference printed in its result CSVs (100000 = no solution).
Only this script and the oracle's build need the reference checkout (its code/
directory: GST_REFERENCE_CODE, else "reference" beside this repository); the
committed JSON is all the tests read.
"""
from __future__ import annotations

import hashlib
import json
import os
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "gpu4gst-sigmod-fullexp_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import numpy as np  # noqa: E402

import gst_b200 as G  # noqa: E402
import oracle as O  # noqa: E402


def fingerprint(g, grp) -> str:
    h = hashlib.sha256()
    for a in (g.beg_pos, g.adj, g.weight, grp.grp_ptr, grp.members):
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()[:16]


def make_inputs(spec):
    gs = spec["graph"]
    if gs["kind"] == "ba":
        g = G.synth_ba(gs["V"], gs["m"], gs["seed"])
    elif gs["kind"] == "rmat":
        g = G.synth_rmat(gs["V"], gs["E"], gs["seed"])
    else:
        raise ValueError(gs["kind"])
    gr = spec["groups"]
    if gr["kind"] == "uniform":
        grp = G.synth_groups_uniform(g.V, gr["n"], gr["smin"], gr["smax"], gr["seed"])
    else:
        grp = G.synth_groups_zipf(g.V, gr["n"], gr["s"], gr["smin"], gr["smax"], gr["seed"])
    return g, grp


SPECS = [
    {"name": "c1_ba20k_k3",
     "graph": {"kind": "ba", "V": 20000, "m": 4, "seed": 0x6057 + 1},
     "groups": {"kind": "uniform", "n": 500, "smin": 5, "smax": 50, "seed": 0x6057 + 1001},
     "queries": [{"k": 3, "n": 100, "seed": 0x6057 + 2001, "hop": [None]}],
     "solvers": ["PrunedDP++", "TrimCDP-multi-core-CPU"]},
    {"name": "rmat3k_k4_k5",
     "graph": {"kind": "rmat", "V": 3000, "E": 12000, "seed": 77},
     "groups": {"kind": "zipf", "n": 200, "s": 1.5, "smin": 2, "smax": 100, "seed": 78},
     "queries": [{"k": 4, "n": 40, "seed": 83, "hop": [None, 2, 3, 4]},
                 {"k": 5, "n": 40, "seed": 84, "hop": [None, 3, 4]}],
     "solvers": ["PrunedDP++", "TrimCDP-multi-core-CPU", "D-PrunedDP++"]},
    {"name": "rmat20k_k6",
     "graph": {"kind": "rmat", "V": 20000, "E": 150000, "seed": 91},
     "groups": {"kind": "zipf", "n": 1000, "s": 1.5, "smin": 2, "smax": 200, "seed": 92},
     "queries": [{"k": 6, "n": 20, "seed": 93, "hop": [None, 3]}],
     "solvers": ["PrunedDP++", "D-PrunedDP++"]},
    # the largest query sizes (k = 7 runs in the default bench; 8 is the maximum)
    {"name": "rmat4k_k7_k8",
     "graph": {"kind": "rmat", "V": 4000, "E": 16000, "seed": 111},
     "groups": {"kind": "zipf", "n": 300, "s": 1.5, "smin": 2, "smax": 120, "seed": 112},
     "queries": [{"k": 7, "n": 16, "seed": 113, "hop": [None, 3]},
                 {"k": 8, "n": 10, "seed": 114, "hop": [None, 3]}],
     "solvers": ["PrunedDP++", "TrimCDP-multi-core-CPU", "D-PrunedDP++"]},
    # the widest hop-bounded rows of the serving configuration's mix: k = 8 at D = 4
    {"name": "rmat4k_k8_D4",
     "graph": {"kind": "rmat", "V": 4000, "E": 16000, "seed": 121},
     "groups": {"kind": "zipf", "n": 300, "s": 1.5, "smin": 2, "smax": 120, "seed": 122},
     "queries": [{"k": 8, "n": 12, "seed": 123, "hop": [4]}],
     "solvers": ["D-PrunedDP++", "D-TrimCDP-multi-core-CPU"]},
    # hop-bounded queries at a larger scale (the hop-limited lower bounds prune hard)
    {"name": "rmat50k_hop",
     "graph": {"kind": "rmat", "V": 50000, "E": 400000, "seed": 101},
     "groups": {"kind": "zipf", "n": 2000, "s": 1.5, "smin": 2, "smax": 300, "seed": 102},
     "queries": [{"k": 4, "n": 16, "seed": 103, "hop": [2, 4, 5]},
                 {"k": 5, "n": 12, "seed": 104, "hop": [None, 3, 4]}],
     "solvers": ["PrunedDP++", "D-PrunedDP++"]},
]

# The benchmark configurations themselves (bench.py WORKLOADS, same generator calls and
# seeds): the first queries of each query pool, solved by the reference's multi-core
# CPU solvers, plus a few by its single-thread PrunedDP++ as a second opinion.
SEED = 0x6057
BENCH_SPECS = [
    # mid-scale plain path: R-MAT 170k target / 6.8M edges, largest component kept
    {"name": "c2_rmat170k_k5k7",
     "graph": {"kind": "rmat", "V": 170_000, "E": 6_800_000, "seed": SEED + 2},
     "groups": {"kind": "zipf", "n": 5000, "s": 1.5, "smin": 2, "smax": 500, "seed": SEED + 1002},
     "queries": [{"k": 5, "n": 16, "seed": SEED + 2002, "hop": [None]},
                 {"k": 7, "n": 8, "seed": SEED + 2003, "hop": [None]}],
     "solvers": ["TrimCDP-multi-core-CPU", "PrunedDP++"],
     # single-thread PrunedDP++: 80-125 s per k = 5 query here, 700-830 s per k = 7 query
     "limit": {"PrunedDP++": 2}},
    # diameter-bounded path: R-MAT grown until the kept component has ~1M vertices and
    # ~15M edges; k = 5 at D = 3, 4, 5
    {"name": "c3_rmat1M_k5_D345",
     "graph": {"kind": "rmat", "V": 2_000_000, "E": 15_300_000, "seed": SEED + 3},
     "groups": {"kind": "zipf", "n": 10000, "s": 1.5, "smin": 2, "smax": 1000, "seed": SEED + 1003},
     "queries": [{"k": 5, "n": 4, "seed": SEED + 2031, "hop": [3, 4, 5]}],
     "solvers": ["D-TrimCDP-multi-core-CPU", "D-PrunedDP++"],
     "limit": {"D-PrunedDP++": 1}, "per_query": True, "timeout": 1800},
    # batched configuration: R-MAT grown until the kept component has ~4M vertices and
    # ~71M edges; k = 3, 5 unbounded and D = 4, k = 7 unbounded
    {"name": "c4_rmat4M_k357",
     "graph": {"kind": "rmat", "V": 8_650_000, "E": 71_000_000, "seed": SEED + 4},
     "groups": {"kind": "zipf", "n": 20000, "s": 1.5, "smin": 2, "smax": 2000, "seed": SEED + 1004},
     "queries": [{"k": 3, "n": 4, "seed": SEED + 2041, "hop": [None, 4]},
                 {"k": 5, "n": 4, "seed": SEED + 2042, "hop": [None, 4]},
                 {"k": 7, "n": 3, "seed": SEED + 2043, "hop": [None]}],
     "solvers": ["TrimCDP-multi-core-CPU", "D-TrimCDP-multi-core-CPU"],
     "per_query": True, "timeout": 1800},
]


def run_spec(spec):
    """Run the spec's solvers on its queries.  A solver listed in spec["limit"] runs
    on the first `limit` queries of each case only (single-thread solvers at the larger
    configurations); with spec["per_query"] every query is its own solver run under
    spec["timeout"] seconds, and a query that runs out of time records no cost (None).
    Each case also records the solver's own per-query time (its result CSV's time
    column, main loop only) under "ref_time"."""
    g, grp = make_inputs(spec)
    out = {"name": spec["name"], "graph": spec["graph"], "groups": spec["groups"],
           "V": g.V, "E": g.E, "fingerprint": fingerprint(g, grp), "cases": []}
    limits = spec.get("limit", {})
    per_query = spec.get("per_query", False)
    timeout = spec.get("timeout")
    with tempfile.TemporaryDirectory() as d:
        for qs in spec["queries"]:
            q = G.synth_queries(grp.n_groups, qs["n"], qs["k"], qs["seed"])
            G.write_reference_files(d, "fx", g, grp, q)
            for hop in qs["hop"]:
                case = {"k": qs["k"], "hop": hop, "query_seed": qs["seed"],
                        "queries": q.tolist(), "ref": {}, "ref_time": {}}
                for s in spec["solvers"]:
                    is_hop = O.REF_SOLVERS[s][1]
                    if is_hop != (hop is not None):
                        continue
                    n = min(qs["n"], limits.get(s, qs["n"]))
                    if per_query:
                        costs, times = [], []
                        for i in range(n):
                            try:
                                rows, wall = O.run_ref(s, d, "fx", qs["k"], i, i, hop_bound=hop,
                                                       timeout=timeout)
                                costs.append(rows[0]["cost"])
                                times.append(rows[0]["time"])
                            except Exception as e:  # noqa: BLE001 (timeout or failure)
                                print(spec["name"], s, "query", i, "gave no cost:", type(e).__name__,
                                      flush=True)
                                costs.append(None)
                                times.append(None)
                                wall = float("nan")
                            print(spec["name"], "k", qs["k"], "hop", hop, s, "query", i,
                                  costs[-1], f"{wall:.1f}s", flush=True)
                    else:
                        rows, wall = O.run_ref(s, d, "fx", qs["k"], 0, n - 1, hop_bound=hop,
                                               timeout=timeout)
                        rows.sort(key=lambda r: r["task_id"])
                        costs = [r["cost"] for r in rows]
                        times = [r["time"] for r in rows]
                        print(spec["name"], "k", qs["k"], "hop", hop, s, f"{wall:.1f}s", flush=True)
                    case["ref"][s] = costs
                    case["ref_time"][s] = times
                out["cases"].append(case)
    return out


KNOWN_ANSWER = {
    # hand-checked small instances: edges (u, v, w), groups, queries with costs
    "name": "known_answer",
    "graphs": [
        {"V": 4, "edges": [[0, 1, 3], [1, 2, 4], [2, 3, 5]],
         "groups": [[0], [3], [1, 2], [0, 3]],
         "cases": [{"q": [0, 1], "hop": None, "cost": 12},
                   {"q": [0, 2], "hop": None, "cost": 3},
                   {"q": [3], "hop": None, "cost": 0},
                   {"q": [0, 1], "hop": 3, "cost": 12},
                   {"q": [0, 1], "hop": 2, "cost": -1},
                   {"q": [0, 1, 2], "hop": None, "cost": 12}]},
        {"V": 5, "edges": [[0, 1, 2], [0, 2, 2], [0, 3, 2], [1, 4, 1], [4, 3, 1]],
         "groups": [[1], [2], [3], [4]],
         "cases": [{"q": [0, 1, 2], "hop": None, "cost": 6},
                   {"q": [0, 1, 2], "hop": 2, "cost": 6},
                   {"q": [0, 2], "hop": None, "cost": 2},
                   {"q": [1, 3], "hop": None, "cost": 5}]},
        {"V": 6, "edges": [[0, 1, 1], [1, 2, 1], [3, 4, 1], [4, 5, 1]],
         "groups": [[0], [5], [2, 3]],
         "cases": [{"q": [0, 1], "hop": None, "cost": -1},
                   {"q": [0, 2], "hop": None, "cost": 2},
                   {"q": [2], "hop": 0, "cost": 0}]},
    ],
}


def main(names=None):
    """Regenerate every small fixture, or only the named ones (the benchmark-size
    fixtures of BENCH_SPECS are made only when named: they take minutes to hours)."""
    specs = [s for s in SPECS if not names or s["name"] in names]
    specs += [s for s in BENCH_SPECS if names and s["name"] in names]
    for spec in specs:
        f = run_spec(spec)
        with open(os.path.join(HERE, f["name"] + ".json"), "w") as fh:
            json.dump(f, fh, separators=(",", ":"))
    if not names:
        with open(os.path.join(HERE, "known_answer.json"), "w") as fh:
            json.dump(KNOWN_ANSWER, fh, indent=1)


if __name__ == "__main__":
    main(sys.argv[1:])
