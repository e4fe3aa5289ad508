"""Benchmark: exact-cost GST queries/s, batched vs one query at a time, on one B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload c4|c1|c2|c3|c5] [--batch B]

Default workload "c4", the batched configuration: R-MAT (a,b,c) = (0.57, 0.19, 0.19)
with its target vertex count grown until the largest component, which is kept, has
4.03M vertices and 71.0M undirected edges (int32 weights uniform in [1,100]); 20,000
groups with Zipf(1.5) sizes clamped to [2,2000]; 1,024 queries with k in {3,5,7} at
40/40/20 %, half of them with hop bound D = 4.  All inputs are seeded synthetic data
(csrc/gst_synth.cpp); the reference distributes no dataset that runs here.

One step = one batch of B queries (the workload's query stream in order) solved
exactly through the engine's C ABI (gst_solve_batch), graph resident in HBM.  The L2
is flushed (a 512 MB write) between steps.

value      queries/s over the K timed steps, device time (CUDA events on the engine's
           stream around each batch), max over ranks.
e2e        the same steps timed on the host around the C-ABI call, which uploads each
           query from host memory and copies every result (cost + tree) back.
per_query  the same engine, one query at a time (gst_solve), on the first queries of
           the timed batches; batched_over_per_query = value / per_query.
by_k       the same two numbers on batches made of one k only (k = 5 and k = 7).
parity     engine costs against the reference's own solvers on the same queries:
           the committed fixture of this configuration (tests/golden/), the CPU
           baseline sample of this run, and the reference arm's sample when it ran
           on this machine before; a mismatch exits non-zero.
roofline   the level kernel with the most device time in a replay of the first
           timed batches with CUDA events around every level launch: algorithmic
           bytes (level_bytes) / event-timed duration against the measured HBM copy
           bandwidth; traffic from the committed ncu summary (profiles/).
cpu_baseline  the reference's TrimCDP-multi-core-CPU (oracle/_ref, compiled from its
           sources, all host threads up to its own cap of 100) on a bounded sample of
           the timed queries; its graph loading is excluded.
--impl reference  the reference's multi-core CPU solvers (TrimCDP-multi-core-CPU for
           unbounded queries, D-TrimCDP-multi-core-CPU for hop-bounded ones) on the
           host cores, on the first queries of the same timed batches, files written
           by the standalone generator gst_gen (no engine code in the process).
"""
from __future__ import annotations

import argparse
import json
import os
import shutil
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "gpu4gst-sigmod-fullexp_b200")
ORACLE = os.path.join(ROOT, "oracle")
GOLDEN = os.path.join(ROOT, "tests", "golden")
PROFILES = os.path.join(ROOT, "profiles")
sys.path.insert(0, PKG)

METRIC = "exact-cost GST queries/s, batched vs per-query on 1 B200; p50/p99 latency"
SEED = 0x6057
REF_INF = 100000

WORKLOADS = {
    # batched form: k in {3,5,7} at 40/40/20 %, half of the queries with hop bound 4
    "c4": dict(name="rmat4M_71M_k357_halfD4", graph=("rmat", 8_650_000, 71_000_000, SEED + 4),
               groups=("zipf", 20_000, 1.5, 2, 2000, SEED + 1004),
               queries=[(3, 410, SEED + 2041), (5, 410, SEED + 2042), (7, 204, SEED + 2043)],
               hop=(4, 0.5, SEED + 3004), golden="c4_rmat4M_k357"),
    # the batched form's shape at a quarter of its size (1M-vertex component, 18M
    # edges): small enough for profiler captures of every kernel
    "c4q": dict(name="rmat1M_18M_k357_halfD4", graph=("rmat", 2_150_000, 18_000_000, SEED + 4),
                groups=("zipf", 20_000, 1.5, 2, 2000, SEED + 1004),
                queries=[(3, 410, SEED + 2041), (5, 410, SEED + 2042), (7, 204, SEED + 2043)],
                hop=(4, 0.5, SEED + 3004)),
    "c2": dict(name="rmat170k_6.8M_k5k7", graph=("rmat", 170_000, 6_800_000, SEED + 2),
               groups=("zipf", 5000, 1.5, 2, 500, SEED + 1002),
               queries=[(5, 300, SEED + 2002), (7, 300, SEED + 2003)], golden="c2_rmat170k_k5k7"),
    "c1": dict(name="ba20k_k3", graph=("ba", 20_000, 4, SEED + 1),
               groups=("uniform", 500, 5, 50, SEED + 1001),
               queries=[(3, 100, SEED + 2001)], golden="c1_ba20k_k3"),
    # diameter-bounded form: k = 5, D cycling through 3, 4, 5
    "c3": dict(name="rmat1M_15M_k5_D345", graph=("rmat", 2_000_000, 15_300_000, SEED + 3),
               groups=("zipf", 10_000, 1.5, 2, 1000, SEED + 1003),
               queries=[(5, 200, SEED + 2031)], hop_cycle=(3, 4, 5), golden="c3_rmat1M_k5_D345"),
    # serving form: k uniform in 3..8, 30 % with hop bound 4 (a k = 8, D = 4 state table,
    # 8.6M x 256 x 5 cells x 8 B = 88 GB, is refused by admission when it does not fit)
    "c5": dict(name="rmat16M_250M_k3to8_30pctD", graph=("rmat", 16_000_000, 250_000_000, SEED + 5),
               groups=("zipf", 50_000, 1.5, 2, 5000, SEED + 1005),
               queries=[(k, 100, SEED + 2050 + k) for k in range(3, 9)],
               hop=(4, 0.3, SEED + 3005)),
}


def mix_queries(pools, hop, kmax=8):
    """A seeded shuffle of the query pools (one per k), a seeded fraction of them with
    hop bound D; queries of more than kmax groups stay unbounded.  hop = (D, fraction,
    seed).  Returns (queries, hops), hops[i] None for an unbounded query."""
    import numpy as np
    D, frac, hseed = hop
    allq = [q for p in pools for q in p]
    rng = np.random.default_rng(hseed)
    order = rng.permutation(len(allq))
    queries = [allq[i] for i in order]
    hops = [D if x < frac else None for x in rng.random(len(queries))]
    hops = [h if len(q) <= kmax else None for q, h in zip(queries, hops)]
    return queries, hops


def workload_queries(w, pools):
    """The workload's query stream from its pools (one array per k, in w["queries"]
    order): hop-mixed and shuffled, D cycling, or the k classes interleaved."""
    if "hop" in w:
        return mix_queries(pools, w["hop"], w.get("hop_kmax", 8))
    queries = []
    for i in range(max(len(p) for p in pools)):
        for p in pools:
            if i < len(p):
                queries.append(p[i])
    if "hop_cycle" in w:
        cyc = w["hop_cycle"]
        return queries, [cyc[i % len(cyc)] for i in range(len(queries))]
    return queries, [None] * len(queries)


def make_workload(key):
    """Graph, groups and query stream of a workload, through the engine library's
    generator (the engine arm)."""
    import gst_b200 as G
    w = WORKLOADS[key]
    gk = w["graph"]
    if gk[0] == "rmat":
        g = G.synth_rmat(gk[1], gk[2], gk[3])
    else:
        g = G.synth_ba(gk[1], gk[2], gk[3])
    gr = w["groups"]
    if gr[0] == "zipf":
        grp = G.synth_groups_zipf(g.V, gr[1], gr[2], gr[3], gr[4], gr[5])
    else:
        grp = G.synth_groups_uniform(g.V, gr[1], gr[2], gr[3], gr[4])
    pools = [G.synth_queries(grp.n_groups, n, k, s) for k, n, s in w["queries"]]
    queries, hops = workload_queries(w, pools)
    return w, g, grp, queries, hops


def gen_args(w):
    """gst_gen arguments that write workload w's graph, groups and query pools."""
    gk, gr = w["graph"], w["groups"]
    a = [gk[0]] + [str(x) for x in gk[1:]]
    a += [gr[0]] + [str(x) for x in gr[1:]]
    for k, n, s in w["queries"]:
        a += ["pool", str(k), str(n), str(s)]
    return a


def workload_config(w, V, E, queries, hops, B, n_ranks):
    """The `config` object of both arms' lines: the workload only (no engine setting)."""
    hb = [h for h in hops if h is not None]
    return {"workload": w["name"], "V": int(V), "E_directed": int(E),
            "groups": w["groups"][1], "queries": len(queries),
            "k": sorted({len(q) for q in queries}),
            "hop_bounded": round(len(hb) / max(1, len(hops)), 4),
            "hop_bounds": sorted(set(hb)), "global_batch": B * n_ranks,
            "parallelism": f"replicas{n_ranks}"}


def timed_order(n_queries, steps, warmup, B, rank, n_ranks):
    """Indices of the queries of the timed batches of `rank`, in solve order."""
    out = []
    for s in range(steps):
        out += rank_slice(n_queries, warmup + s, B, rank, n_ranks)
    return out


class Clocks:
    """nvidia-smi samples (SM clock, throttle reasons) during the timed region."""

    def __init__(self, index=0):
        self.index = index
        self.samples = []
        self.proc = None

    def __enter__(self):
        if shutil.which("nvidia-smi") is None:
            return self
        q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        self.proc = subprocess.Popen(
            ["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}",
             "--format=csv,noheader,nounits", "-lms", "200"],
            stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        self.t = threading.Thread(target=self._read, daemon=True)
        self.t.start()
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.samples.append([x.strip() for x in line.split(",")])

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        sm = [float(s[0]) for s in self.samples if s[0].replace(".", "").isdigit()]
        mx = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for s in self.samples:
            for n, v in zip(names, s[4:8]):
                if v.strip().lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": sorted(reasons),
                "samples": len(self.samples)}


def peak_hbm():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def dist_env():
    n = int(os.environ.get("WORLD_SIZE", "1"))
    r = int(os.environ.get("RANK", "0"))
    lr = int(os.environ.get("LOCAL_RANK", str(r)))
    return n, r, lr


# ---- the reference's CPU solvers on a sample of the workload ----------------------

UNBOUNDED_SOLVER = "TrimCDP-multi-core-CPU"
HOP_SOLVER = "D-TrimCDP-multi-core-CPU"
# D-TrimCDP-multi-core-CPU keeps a dense table of 20-byte nodes per (vertex, subset, hop):
# 4M x 2^7 x 5 of them (k = 7, D = 4) would take ~75 GB of host memory, so hop-bounded
# samples keep k <= 5
HOP_SAMPLE_KMAX = 5


def _ref_exe(name):
    return os.path.join(ORACLE, "_ref", name)


def run_solver_streaming(exe, data_dir, data_name, T, n, D, budget_s):
    """Run one of the reference's multi-core solvers (executable `exe`, argv of its
    README: type 1 unbounded, type 2 with hop bound D) over the first n queries of
    <data_dir><data_name><T>.csv, timing each query from the solver's own per-query
    output lines ("<name> iteration i" before, "cpu_cost c" / "cost c" after, both
    flushed by endl).  The solver is stopped once `budget_s` seconds have passed since
    its first query started.  Returns (records [(index, cost, seconds)], load_seconds,
    window_seconds): the window runs from the first query's start to the last query's
    end, or to the stop when a query was still running then."""
    os.makedirs(os.path.join(data_dir, "result"), exist_ok=True)
    path = data_dir.rstrip("/") + "/"
    args = [exe, "2" if D is not None else "1", path, data_name, str(T)]
    if D is not None:
        args.append(str(D))
    args += ["0", str(n - 1)]
    t0 = time.perf_counter()
    p = subprocess.Popen(args, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True,
                         bufsize=1)
    recs, t_it, cur, load = [], None, None, None
    t_first = t_last = None
    timer = None

    def stop():
        if p.poll() is None:
            p.kill()
    try:
        for line in p.stdout:
            now = time.perf_counter()
            parts = line.split()
            if len(parts) >= 3 and parts[1] == "iteration":
                cur, t_it = int(parts[2]), now
                if load is None:
                    load = now - t0
                    t_first = now
                    timer = threading.Timer(budget_s, stop)
                    timer.start()
            elif parts and parts[0] in ("cpu_cost", "cost") and t_it is not None and len(parts) > 1:
                recs.append((cur, int(parts[1]), now - t_it))
                t_it = t_last = None
                t_last = now
        p.wait()
        end = time.perf_counter()
    finally:
        if timer:
            timer.cancel()
        stop()
    if t_first is None:
        return recs, time.perf_counter() - t0, 0.0
    # a query cut off by the stop counts its time but not itself
    window = (end if t_it is not None else (t_last or end)) - t_first
    return recs, load, window


def ref_sample(data_dir, data_name, sample, budget_s):
    """The reference's multi-core solvers on `sample` (a list of (index, group ids, hop
    bound or None), in order): unbounded queries through TrimCDP-multi-core-CPU,
    hop-bounded ones (k <= HOP_SAMPLE_KMAX) through D-TrimCDP-multi-core-CPU, one
    solver run each, budget_s seconds of query time split between them by their share
    of the sample.  Both solvers take a query's size from its line, so one query file
    holds every k.  Returns (records [(index, group ids, hop, cost, seconds)], loads,
    skipped hop-bounded queries)."""
    unb = [x for x in sample if x[2] is None]
    hop = [x for x in sample if x[2] is not None and len(x[1]) <= HOP_SAMPLE_KMAX]
    skipped = sum(1 for x in sample if x[2] is not None and len(x[1]) > HOP_SAMPLE_KMAX)
    out, loads, window = [], [], 0.0
    runs = [(UNBOUNDED_SOLVER, unb, None)]
    for D in sorted({x[2] for x in hop}):
        runs.append((HOP_SOLVER, [x for x in hop if x[2] == D], D))
    total = sum(len(r[1]) for r in runs)
    for solver, items, D in runs:
        if not items or not os.path.exists(_ref_exe(solver)):
            continue
        T = max(len(x[1]) for x in items)
        with open(os.path.join(data_dir, f"{data_name}{T}.csv"), "w") as f:
            for _, q, _ in items:
                f.write(" ".join(str(int(a)) for a in q) + "\n")
        share = budget_s * len(items) / total
        recs, load, win = run_solver_streaming(_ref_exe(solver), data_dir, data_name, T, len(items),
                                               D, share)
        loads.append(load)
        window += win
        print(f"bench: {solver}{'' if D is None else f' D={D}'}: {len(recs)} of {len(items)} "
              f"queries in a {win:.1f} s window (graph load {load:.1f} s)", file=sys.stderr)
        for i, cost, dt in recs:
            idx, q, h = items[i]
            out.append((idx, [int(a) for a in q], h, cost, dt))
    return out, loads, skipped, window


def sample_summary(recs, loads, skipped, window, threads):
    n_u = sum(1 for r in recs if r[2] is None)
    n_h = len(recs) - n_u
    txt = (f"first queries of the timed batches: {n_u} unbounded ({UNBOUNDED_SOLVER}) and "
           f"{n_h} hop-bounded ({HOP_SOLVER}) finished in a {window:.1f} s window of query "
           f"time on {threads} threads (a query still running at the stop counts its time; "
           f"graph loading, {sum(loads):.0f} s, excluded)")
    if skipped:
        txt += (f"; {skipped} hop-bounded k > {HOP_SAMPLE_KMAX} queries left out (the "
                f"solver's dense host table would need tens of GB)")
    return txt


def ref_costs_path(w):
    return os.path.join(tempfile.gettempdir(), f"gst_bench_reference_{w['name']}.json")


def run_reference_arm(args):
    """The reference's multi-core CPU solvers on the host cores, on the first queries
    of the engine arm's timed batches.  The workload's files come from the standalone
    generator gst_gen; no engine library is loaded in this process.  The graph load is
    the untimed warm-up; the timed part is K steps' share of a few minutes of query
    time, measured per query from the solver's own output."""
    import numpy as np
    n, rank, _ = dist_env()
    if rank != 0:
        return 0
    w = WORKLOADS[args.workload]
    gen = os.path.join(PKG, "gst_gen")
    missing = [x for x in (gen, _ref_exe(UNBOUNDED_SOLVER)) if not os.path.exists(x)]
    if missing:
        print(json.dumps({"impl": "reference", "unavailable": f"not built: {missing}"}))
        return 0
    d = tempfile.mkdtemp(prefix="gstref_")
    try:
        p = subprocess.run([gen, d, "w"] + gen_args(w), stdout=subprocess.PIPE,
                           stderr=subprocess.STDOUT, text=True, check=True)
        tok = p.stdout.split()
        V, E = int(tok[tok.index("V") + 1]), int(tok[tok.index("E") + 1])
        pools = [np.loadtxt(os.path.join(d, f"w_pool{k}.txt"), dtype=np.int32, ndmin=2)
                 for k, _, _ in w["queries"]]
        queries, hops = workload_queries(w, pools)
        order = timed_order(len(queries), args.steps, args.warmup, args.batch, 0, n)
        sample = [(i, queries[i], hops[i]) for i in order[:64]]
        budget = float(min(300.0, max(60.0, 15.0 * args.steps)))
        recs, loads, skipped, spent = ref_sample(d, "w", sample, budget)
    finally:
        shutil.rmtree(d, ignore_errors=True)
    threads = min(os.cpu_count() or 1, 100)
    if not recs:
        print(json.dumps({"impl": "reference",
                          "unavailable": f"the reference's solvers finished no query within {budget:.0f} s"}))
        return 0
    qps = len(recs) / spent
    with open(ref_costs_path(w), "w") as f:
        json.dump({"workload": w["name"], "records": [[r[1], r[2], r[3]] for r in recs]}, f)
    line = {
        "metric": METRIC, "value": qps, "unit": "queries/s", "n_gpus": n, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * spent / max(1, args.steps),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int32",
        "data": "synthetic", "impl": "reference",
        "config": workload_config(w, V, E, queries, hops, args.batch, n),
        "cpu_baseline": {"value": qps, "unit": "queries/s", "cores": threads, "kind": "reference",
                         "sample": sample_summary(recs, loads, skipped, spent, threads)},
        "e2e": {"value": qps, "unit": "queries/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "reference_costs": [[r[1], r[2], r[3]] for r in recs],
        "note": "warm-up = the solvers' graph loading; steps share a bounded query-time budget "
                f"of {budget:.0f} s, queries timed one by one from the solvers' own output",
    }
    print(json.dumps(line))
    return 0


# ---- engine arm ---------------------------------------------------------------

def level_bytes(answers, queries, hops, bucket_delta=0):
    """Algorithmic bytes of the three level kernels for a set of answered queries:
    sssp per relaxation 8 B edge + the target's k distances (4k B) when the search
    runs group-mask items (hop-bounded queries with D > 0, and every query when the
    search runs in one cost bucket: one relaxation serves all of the item's groups),
    else 16 B (8 B edge + 4 B distance read + 4 B written); grow 24 B per work item (16 B item + 8 B source cell) +
    16 B per relaxation (8 B edge + 8 B target cell); rows 16 B per cell of every
    row merged (the row read once and written back once)."""
    b = {"k_sssp": 0.0, "k_grow": 0.0, "k_rows": 0.0}
    for a, q, h in zip(answers, queries, hops):
        st = a.stats
        rw = (1 << len(q)) * (1 if h is None else h + 1)
        masked = (h is not None and h > 0) or bucket_delta == 0
        b["k_sssp"] += (8.0 + 4.0 * len(q) if masked else 16.0) * st["sssp_relaxations"]
        b["k_grow"] += 24.0 * st["states_expanded"] + 16.0 * st["edge_relaxations"]
        b["k_rows"] += 16.0 * rw * st["rows_merged"]
    return b


def rank_slice(n_queries, step, B, rank, n_ranks):
    """Query indices of `rank`'s batch at `step`: every rank takes its own slice of
    the query stream (replicas, weak scaling), the ranks' slices of a step disjoint
    while B * n_ranks <= n_queries."""
    base = ((step * n_ranks + rank) * B) % n_queries
    return [(base + i) % n_queries for i in range(B)]


def max_over_ranks(values, dist):
    """Element-wise max over the ranks of a list of floats (gloo all-reduce; the
    identity for one process)."""
    if dist is None:
        return list(values)
    import torch
    t = torch.tensor(values, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(x) for x in t]


def serve_run(dg, queries, hops, rate, n, seed):
    """Poisson arrivals at `rate` queries/s through the continuous-batching server
    (gst_submit / gst_wait); latency is the engine's time from submit to result."""
    import numpy as np
    rng = np.random.default_rng(seed)
    gaps = rng.exponential(1.0 / rate, n)
    sv = dg.server()
    tickets = []
    t0 = time.perf_counter()
    due = t0
    for i in range(n):
        due += gaps[i]
        while True:
            left = due - time.perf_counter()
            if left <= 0:
                break
            if left > 2e-3:
                time.sleep(left - 1e-3)
        j = i % len(queries)
        tickets.append(sv.submit(queries[j], hops[j], tag=i))
    res = [sv.wait(t) for t in tickets]
    t1 = time.perf_counter()
    sv.close()
    refused = [r for r in res if r.status == 2]
    bad = [r for r in res if r.status not in (0, 1, 2)]
    lat = [r.stats["latency_ms"] for r in res if r.status in (0, 1)]
    return {"offered_qps": rate, "queries": n, "achieved_qps": n / (t1 - t0),
            "p50_ms": float(np.percentile(lat, 50)) if lat else None,
            "p99_ms": float(np.percentile(lat, 99)) if lat else None,
            "refused_oom_admission": len(refused), "failed": len(bad)}


def golden_cases(name):
    """(group ids, hop, cost) of every query a committed fixture has a reference cost
    for (-1 = infeasible), or None when no fixture exists; the fixture's solvers must
    agree with each other."""
    p = os.path.join(GOLDEN, name + ".json")
    if not os.path.exists(p):
        return None
    with open(p) as f:
        fx = json.load(f)
    out = []
    for case in fx["cases"]:
        for i, q in enumerate(case["queries"]):
            costs = {s: c[i] for s, c in case["ref"].items() if i < len(c) and c[i] is not None}
            if not costs:
                continue
            vals = set(costs.values())
            if len(vals) != 1:
                raise SystemExit(f"bench: the fixture's solvers disagree on {q} hop={case['hop']}: {costs}")
            c = vals.pop()
            out.append((q, case["hop"], -1 if c >= REF_INF else c))
    return out


def check_parity(dg, G, items):
    """Solve (group ids, hop, expected cost) items in batches; returns (checked, agree,
    first mismatches)."""
    bad, agree = [], 0
    for i in range(0, len(items), 32):
        chunk = items[i:i + 32]
        ans = dg.solve_batch([c[0] for c in chunk], [c[1] for c in chunk])
        for (q, h, want), a in zip(chunk, ans):
            got = a.cost if a.ok else (-1 if a.status == G.INFEASIBLE else None)
            if got == want:
                agree += 1
            elif len(bad) < 5:
                bad.append({"q": [int(x) for x in q], "hop": h, "engine": got, "reference": want})
    return len(items), agree, bad


def roofline_traffic(kernel, alg_bytes_per_launch):
    """DRAM bytes per launch of `kernel` from the committed ncu summary (the ratio of its
    measured DRAM traffic to its algorithmic bytes on the captured case, applied to this
    run's algorithmic bytes per launch), or None."""
    p = os.path.join(PROFILES, "traffic.json")
    try:
        with open(p) as f:
            t = json.load(f)
        r = t["kernels"][kernel]["dram_bytes_per_alg_byte"]
        return r * alg_bytes_per_launch, t["kernels"][kernel].get("case")
    except Exception:
        return None, None


def run_ours(args):
    import numpy as np
    import gst_b200 as G
    n_ranks, rank, local_rank = dist_env()
    dist = None
    if n_ranks > 1:
        import torch.distributed as dist  # noqa: F811
        import datetime
        dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=600))
    import torch
    torch.cuda.set_device(local_rank)
    flush = torch.empty(512 * 1024 * 1024, dtype=torch.uint8, device=f"cuda:{local_rank}")

    w, g, grp, queries, hops = make_workload(args.workload)
    B = args.batch
    # the product path: CUDA-graph level loop, no per-kernel events
    eng = G.Engine(local_rank, max_batch=min(B, 64), use_graphs=0 if args.no_graphs else 1)
    dg = eng.graph(g, grp)
    config = workload_config(w, g.V, g.E, queries, hops, B, n_ranks)

    def batch(step):
        idx = rank_slice(len(queries), step, B, rank, n_ranks)
        return [queries[i] for i in idx], [hops[i] for i in idx]

    def usable(ans):
        bad = [a for a in ans if a.status not in (G.OK, G.INFEASIBLE, G.OOM_ADMISSION)]
        if bad:
            raise SystemExit(f"bench: query failed: {G.STATUS[bad[0].status]} {eng.error()}")
        return sum(1 for a in ans if a.status == G.OOM_ADMISSION)

    # launch parameters for this graph shape, chosen on the first batch (cached in the
    # package directory, so a later run on the same shape reuses them)
    tuned = None
    if not args.no_tune:
        cache = os.path.join(PKG, "tune_cache.txt")
        tq, th = batch(0)
        tuned = dg.autotune(tq, th, cache_path=cache)
        tuned = {k: tuned[k] for k in ("split_degree", "bucket_delta", "threads_per_block",
                                       "blocks_per_sm", "max_batch", "search_cut_permille",
                                       "batch_search")}
    for s in range(args.warmup):
        usable(dg.solve_batch(*batch(s)))

    dev_ms, host_ms, lat = [], [], []
    h2d = d2h = launches = refused = 0
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    with Clocks(local_rank) as clk:
        for s in range(args.steps):
            flush.fill_(s & 0xFF)
            torch.cuda.synchronize()
            qs, hs = batch(args.warmup + s)
            t0 = time.perf_counter()
            ans = dg.solve_batch(qs, hs)
            host_ms.append(1e3 * (time.perf_counter() - t0))
            st = ans[0].stats
            dev_ms.append(st["device_ms"])
            refused += usable(ans)
            lat += [a.stats["latency_ms"] for a in ans]
            h2d += st["h2d_bytes"]
            d2h += st["d2h_bytes"]
            launches += st["kernel_launches"]
    torch.cuda.synchronize()
    tot_dev, tot_host = max_over_ranks([sum(dev_ms) / 1e3, sum(host_ms) / 1e3], dist)
    nq_all = args.steps * B * n_ranks
    value = nq_all / tot_dev
    e2e = nq_all / tot_host
    timed = timed_order(len(queries), args.steps, args.warmup, B, rank, n_ranks)

    def one_at_a_time(items):
        dev, host = [], []
        for q, h in items:
            t0 = time.perf_counter()
            a = dg.solve(q, h)
            host.append(time.perf_counter() - t0)
            if a.status in (G.OK, G.INFEASIBLE):
                dev.append(a.stats["device_ms"])
        return dev, host

    # one query at a time, same engine (the reference drivers' mode), on the queries of
    # the timed batches, so that both forms solve the same queries
    per_q, per_q_host = [], []
    if rank == 0:
        per_q, per_q_host = one_at_a_time([(queries[i], hops[i]) for i in timed[: args.single]])

    # the two headline query sizes on their own: batches of k = 5 only and k = 7 only
    # (the workload's queries of that size, in stream order), batched and one at a time
    by_k = {}
    if rank == 0 and not args.no_by_k:
        for kk in (5, 7):
            idx = [i for i in range(len(queries)) if len(queries[i]) == kk]
            if len(idx) < B:
                continue
            bdev = []
            for s in range(3):  # the first batch warms the slot memory for this mix
                sel = [idx[(s * B + j) % len(idx)] for j in range(B)]
                flush.fill_(s & 0xFF)
                torch.cuda.synchronize()
                a = dg.solve_batch([queries[i] for i in sel], [hops[i] for i in sel])
                usable(a)
                if s > 0:
                    bdev.append(a[0].stats["device_ms"])
            one, _ = one_at_a_time([(queries[i], hops[i]) for i in idx[: min(16, B)]])
            bq = 2 * B / (sum(bdev) / 1e3)
            pq = len(one) / (sum(one) / 1e3) if one else None
            by_k[f"k{kk}"] = {"batched_qps": bq, "per_query_qps": pq,
                              "batched_over_per_query": bq / pq if pq else None,
                              "per_query_p50_ms": float(np.percentile(one, 50)) if one else None,
                              "per_query_p99_ms": float(np.percentile(one, 99)) if one else None,
                              "hop_bounded": sum(hops[i] is not None for i in idx) / len(idx)}

    # serving: Poisson arrivals at about 70 % of the batched throughput, ~3 s
    serving = None
    if rank == 0 and not args.no_serve:
        rate = 0.7 * value / n_ranks
        serving = serve_run(dg, queries, hops, rate, max(32, int(3.0 * rate)), SEED + 77)

    # one-label distance cache for hot groups (gst_groups_cache_warm): the groups of
    # the timed queries warmed, then the same queries one at a time and batched (device
    # time); the cache is freed before the roofline replay
    group_cache = None
    if rank == 0 and not args.no_cache:
        cq = [queries[i] for i in timed]
        ch = [hops[i] for i in timed]
        gids = sorted({int(x) for q, h in zip(cq, ch) if h is None for x in q})
        hop_bounds = sorted({h for h in ch if h is not None and h > 0})
        hgids = sorted({int(x) for q, h in zip(cq, ch) if h is not None and h > 0 for x in q})
        # per cache, inside the memory the slot budget leaves free (a hop bound's entry
        # holds D tables of V distances)
        cap, hcap = 12 << 30, 24 << 30
        if gids or hgids:
            t0 = time.perf_counter()
            n_cached = dg.cache_warm(gids, min(cap, 4 * g.V * len(gids))) if gids else 0
            if len(hop_bounds) == 1 and hgids:
                D = hop_bounds[0]
                per = 4 * g.V * (min(D - 1, 7) + 1)
                n_cached += dg.cache_warm_hop(hgids, D, min(hcap, per * len(hgids)))
            warm_ms = 1e3 * (time.perf_counter() - t0)
            one, _ = one_at_a_time(list(zip(cq, ch))[: max(args.single, 1)])
            bat = [dg.solve_batch(*batch(args.warmup + s))[0].stats["device_ms"]
                   for s in range(min(args.steps, 3))]
            dg.cache_warm([], 0)
            if hop_bounds:
                dg.cache_warm_hop([], 1, 0)
            group_cache = {"groups": n_cached, "groups_wanted": len(gids) + len(hgids),
                           "warm_ms": warm_ms,
                           "per_query_qps": len(one) / (sum(one) / 1e3),
                           "batched_qps": B * len(bat) / (sum(bat) / 1e3),
                           "note": "hot groups: the timed queries' groups cached first; the "
                                   "headline value does not use the cache"}

    # roofline: the timed batches replayed with CUDA events around every level
    # kernel launch on the engine's stream (the timed region itself runs the
    # CUDA-graph loop, which has no per-kernel events)
    peak, peak_kind = peak_hbm()
    G.set_profiling(eng, 15)
    kms = {"k_grow": 0.0, "k_rows": 0.0, "k_sssp": 0.0, "k_bs_relax": 0.0}
    kbytes = {"k_grow": 0.0, "k_rows": 0.0, "k_sssp": 0.0, "k_bs_relax": 0.0}
    klaunch = {"k_grow": 0, "k_rows": 0, "k_sssp": 0, "k_bs_relax": 0}
    # work units per kernel: grow edge relaxations, merged rows, distance relaxations,
    # target-row sectors of the batch-shared search's relax steps (32 B per sector read)
    kunits = {"k_grow": 0, "k_rows": 0, "k_sssp": 0, "k_bs_relax": 0}
    unit_of = {"k_grow": "edge_relaxations", "k_rows": "rows_merged",
               "k_sssp": "sssp_relaxations", "k_bs_relax": "shared_sectors"}
    search_ms = 0.0  # the shared searches whole: seeding, scans, copies and control too
    for s in range(min(args.steps, 3)):
        qs, hs = batch(args.warmup + s)
        ans = dg.solve_batch(qs, hs)
        st = ans[0].stats
        kms["k_grow"] += st["grow_ms"]
        kms["k_rows"] += st["rows_ms"]
        kms["k_sssp"] += st["sssp_ms"]
        kms["k_bs_relax"] += st["shared_relax_ms"]
        search_ms += st["shared_ms"]
        for kname, v in level_bytes(ans, qs, hs, tuned["bucket_delta"] if tuned else 0).items():
            kbytes[kname] += v
        kbytes["k_bs_relax"] += 32.0 * st["shared_sectors"]
        for kname, field in (("k_grow", "grow_launches"), ("k_rows", "rows_launches"),
                             ("k_sssp", "sssp_launches"), ("k_bs_relax", "shared_relax_launches")):
            klaunch[kname] += st[field]
        for kname, field in unit_of.items():
            if kname == "k_bs_relax":
                kunits[kname] += st[field]
            else:
                kunits[kname] += sum(a.stats[field] for a in ans)
    G.set_profiling(eng, 0)
    top = max(kms, key=lambda k: kms[k])
    kern = {k: {"ms": kms[k], "alg_bytes": kbytes[k], "launches": klaunch[k],
                "GBps": (kbytes[k] / (kms[k] / 1e3) / 1e9) if kms[k] > 0 else 0.0,
                unit_of[k]: kunits[k],
                "per_s": (kunits[k] / (kms[k] / 1e3)) if kms[k] > 0 else 0.0}
            for k in kms}
    kern["k_bs_relax"]["search_ms"] = search_ms
    achieved = kern[top]["GBps"]
    per_launch = kbytes[top] / max(1, klaunch[top])
    traffic, traffic_case = roofline_traffic(top, per_launch)
    # the ceiling these kernels meet: random 32-byte rows per second (each distance
    # relaxation reads its target's row, each grow relaxation its target's distance row
    # and state cell), measured on this device by gst_probe_random_access
    rand = None
    try:
        rand = G.probe_random_access(local_rank, 4 << 30)
        rand["note"] = ("random 32-byte row gathers from 4 GB (DRAM) and from 32 MB (L2), "
                        "random 4-byte atomicMin; frac = the kernel's relaxations per second "
                        "over the DRAM gather rate (one random row per relaxation)")
        rand["kernels"] = {k: {"relax_per_s": kern[k]["per_s"],
                               "frac": kern[k]["per_s"] / rand["gather32_dram_per_s"]}
                           for k in ("k_sssp", "k_grow", "k_bs_relax") if kern[k]["ms"] > 0}
    except Exception as e:  # noqa: BLE001 (reported, not fatal)
        rand = {"error": str(e)}

    # parity: the engine's costs against the reference's solvers on the same queries
    parity = {"checked": 0, "agree": 0, "sources": {}}
    mismatches = []
    if rank == 0:
        gold = golden_cases(w["golden"]) if w.get("golden") else None
        if gold:
            c, a, bad = check_parity(dg, G, gold)
            parity["sources"][f"tests/golden/{w['golden']}.json"] = {"checked": c, "agree": a}
            parity["checked"] += c
            parity["agree"] += a
            mismatches += bad
        rp = ref_costs_path(w)
        if os.path.exists(rp):
            with open(rp) as f:
                rr = json.load(f)
            if rr.get("workload") == w["name"]:
                items = [(q, h, -1 if c >= REF_INF else c) for q, h, c in rr["records"]]
                c, a, bad = check_parity(dg, G, items)
                parity["sources"]["reference arm (this machine)"] = {"checked": c, "agree": a}
                parity["checked"] += c
                parity["agree"] += a
                mismatches += bad

    line = {
        "metric": METRIC, "value": value, "unit": "queries/s", "n_gpus": n_ranks,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * tot_dev / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int32",
        "data": "synthetic", "config": config,
        "engine": {"tuning": tuned, "l2": "flushed between steps (512 MB write)",
                   "refused_oom_admission": refused},
        "e2e": {"value": e2e, "unit": "queries/s", "h2d_bytes_per_step": h2d // args.steps,
                "d2h_bytes_per_step": d2h // args.steps},
        "latency_ms": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99)),
                       "note": "batched: call start to result ready"},
        "per_query": {"value": (len(per_q) / (sum(per_q) / 1e3)) if per_q else None,
                      "unit": "queries/s",
                      "e2e": (len(per_q_host) / sum(per_q_host)) if per_q_host else None,
                      "p50_ms": float(np.percentile(per_q, 50)) if per_q else None,
                      "p99_ms": float(np.percentile(per_q, 99)) if per_q else None,
                      "queries": len(per_q),
                      "note": "same engine, gst_solve one query at a time, on the first "
                              "queries of the timed batches"},
        "batched_over_per_query": (value / (len(per_q) / (sum(per_q) / 1e3))) if per_q else None,
        "by_k": by_k,
        "serving": serving,
        "group_cache": group_cache,
        "parity": parity,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": traffic, "kernel": top,
                     "peak_kind": peak_kind, "traffic_case": traffic_case,
                     "note": "algorithmic bytes / event-timed kernel time over a replay of "
                             "the first timed batches; traffic: DRAM bytes per launch from "
                             "the ncu summary in profiles/",
                     "kernels": kern, "random_access": rand},
        "gpu_launches": launches,
        "clocks": clk.summary(),
    }
    if rank == 0 and n_ranks == 1 and not args.no_cpu:
        # the reference's multi-core solver on the first unbounded queries of the timed
        # batches, about a minute of query time (files written by the engine library's
        # writer; the solver runs in its own process)
        threads = min(os.cpu_count() or 1, 100)
        sample = [(i, queries[i], None) for i in timed if hops[i] is None][:16]
        if os.path.exists(_ref_exe(UNBOUNDED_SOLVER)) and sample:
            d = tempfile.mkdtemp(prefix="gstcpu_")
            try:
                G.write_reference_files(d, "w", g, grp)
                recs, loads, skipped, spent = ref_sample(d, "w", sample, args.cpu_budget)
            finally:
                shutil.rmtree(d, ignore_errors=True)
            if recs:
                line["cpu_baseline"] = {"value": len(recs) / spent, "unit": "queries/s",
                                        "cores": threads, "kind": "reference",
                                        "sample": sample_summary(recs, loads, skipped, spent,
                                                                 threads)}
                items = [(r[1], r[2], -1 if r[3] >= REF_INF else r[3]) for r in recs]
                c, a, bad = check_parity(dg, G, items)
                parity["sources"]["cpu_baseline sample"] = {"checked": c, "agree": a}
                parity["checked"] += c
                parity["agree"] += a
                mismatches += bad
            else:
                line["cpu_baseline"] = {"value": 0.0, "unit": "queries/s", "cores": threads,
                                        "kind": "reference",
                                        "sample": f"no query finished within {args.cpu_budget:.0f} s "
                                                  f"(graph loading {sum(loads):.0f} s excluded)"}
    if mismatches:
        parity["mismatches"] = mismatches
    if rank == 0:
        print(json.dumps(line))
    dg.close()
    eng.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if mismatches:
        print(f"bench: {len(mismatches)}+ cost mismatches against the reference", file=sys.stderr)
        return 1
    return 0


def run_profile_batch(args):
    """One batch of the workload's first queries with every level kernel launched on its
    own (no CUDA graph), after one untimed batch of the same queries; prints the
    algorithmic bytes and launches per kernel of the second batch as one JSON line.  Run
    under ncu to relate a kernel's measured DRAM traffic to its algorithmic bytes (the
    summaries in profiles/ give the commands)."""
    import gst_b200 as G
    w, g, grp, queries, hops = make_workload(args.workload)
    eng = G.Engine(0, max_batch=args.resident or args.batch, use_graphs=0)
    dg = eng.graph(g, grp)
    qs, hs = queries[: args.batch], hops[: args.batch]
    dg.solve_batch(qs, hs)
    G.set_profiling(eng, 15)
    ans = dg.solve_batch(qs, hs)
    st = ans[0].stats
    b = level_bytes(ans, qs, hs, 0)
    out = {"workload": w["name"], "V": g.V, "E_directed": g.E, "batch": len(qs),
           "kernels": {"k_sssp": {"alg_bytes": b["k_sssp"], "launches": st["sssp_launches"],
                                  "ms": st["sssp_ms"]},
                       "k_grow": {"alg_bytes": b["k_grow"], "launches": st["grow_launches"],
                                  "ms": st["grow_ms"]},
                       "k_rows": {"alg_bytes": b["k_rows"], "launches": st["rows_launches"],
                                  "ms": st["rows_ms"]},
                       "k_bs_relax": {"alg_bytes": 32.0 * st["shared_sectors"],
                                      "launches": st["shared_relax_launches"],
                                      "ms": st["shared_relax_ms"],
                                      "search_ms": st["shared_ms"]}},
           "device_ms": st["device_ms"], "costs": [a.cost for a in ans]}
    print(json.dumps(out))
    dg.close()
    eng.close()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="c4", choices=sorted(WORKLOADS))
    ap.add_argument("--batch", type=int, default=32)
    ap.add_argument("--single", type=int, default=32, help="queries timed one at a time")
    ap.add_argument("--cpu-budget", type=float, default=60.0,
                    help="seconds of query time for the CPU baseline sample")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline sample")
    ap.add_argument("--no-tune", action="store_true", help="default launch parameters")
    ap.add_argument("--no-serve", action="store_true", help="skip the Poisson serving run")
    ap.add_argument("--no-by-k", action="store_true", help="skip the per-k runs")
    ap.add_argument("--no-cache", action="store_true",
                    help="skip the run with the timed queries' groups cached")
    ap.add_argument("--no-graphs", action="store_true",
                    help="host-issued level launches instead of the CUDA-graph loop "
                         "(profilers then see every kernel launch)")
    ap.add_argument("--profile-batch", action="store_true",
                    help="one batch of the first --batch queries with per-kernel launches "
                         "after one untimed batch; prints algorithmic bytes per kernel")
    ap.add_argument("--resident", type=int, default=0,
                    help="with --profile-batch: queries resident at once (default: the batch)")
    args = ap.parse_args()
    if args.profile_batch:
        return run_profile_batch(args)
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return run_reference_arm(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
