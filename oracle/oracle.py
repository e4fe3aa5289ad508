"""Python view of the oracle (TEST INFRASTRUCTURE ONLY).

Loads oracle/liboracle.so (the C restatement in gst_oracle.c) and runs the
reference's own CPU solvers compiled under oracle/_ref/.  Only tests/,
__graft_entry__.smoke() and bench.py's CPU-baseline leg use this module, as the
checker; the engine never calls it.
"""
from __future__ import annotations

import ctypes as C
import os
import re
import subprocess
import tempfile
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
REF_DIR = os.path.join(HERE, "_ref")

_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            subprocess.check_call(["make", "-s", "-C", HERE, "liboracle.so"])
        _lib = C.CDLL(LIB_PATH)
        vp = C.c_void_p
        _lib.oracle_sssp_groups.argtypes = [C.c_int64, vp, vp, vp, C.c_int64, vp, vp]
        _lib.oracle_gst_nonhop.argtypes = [C.c_int64, vp, vp, vp, vp, vp, C.c_int32, vp,
                                           vp, vp, vp, C.c_int64, vp, vp, vp, vp, vp]
        _lib.oracle_gst_hop.argtypes = [C.c_int64, vp, vp, vp, vp, vp, C.c_int32, vp,
                                        C.c_int32, vp, vp, vp, vp, C.c_int64, vp, vp, vp, vp,
                                        vp]
        _lib.oracle_hop_bound_check.argtypes = [C.c_int64, vp, vp, vp, vp, vp, C.c_int32, vp,
                                                C.c_int32, vp, vp, vp]
        _lib.oracle_nonhop_bound_check.argtypes = [C.c_int64, vp, vp, vp, vp, vp, C.c_int32,
                                                   vp, vp, vp, vp]
    return _lib


def _p(a):
    return a.ctypes.data


def sssp_groups(g, members) -> np.ndarray:
    """Distance from the nearest member of `members` to every vertex (int64;
    unreachable = 2**60)."""
    src = np.ascontiguousarray(members, dtype=np.int32)
    dist = np.zeros(g.V, dtype=np.int64)
    rc = lib().oracle_sssp_groups(g.V, _p(g.beg_pos), _p(g.adj), _p(g.weight), src.shape[0],
                                  _p(src), _p(dist))
    assert rc == 0
    return dist


def _solve(g, groups, group_ids, hop_bound):
    gid = np.ascontiguousarray(group_ids, dtype=np.int32)
    cap = g.V + 16
    eu = np.zeros(cap, np.int32)
    ev = np.zeros(cap, np.int32)
    ew = np.zeros(cap, np.int32)
    cost, ne, esum, pops = (C.c_int64() for _ in range(4))
    root, root_d = C.c_int32(), C.c_int32()
    if hop_bound is None or hop_bound < 0:
        rc = lib().oracle_gst_nonhop(g.V, _p(g.beg_pos), _p(g.adj), _p(g.weight),
                                     _p(groups.grp_ptr), _p(groups.members), gid.shape[0],
                                     _p(gid), C.byref(cost), C.byref(root), C.byref(ne), cap,
                                     _p(eu), _p(ev), _p(ew), C.byref(esum), C.byref(pops))
    else:
        rc = lib().oracle_gst_hop(g.V, _p(g.beg_pos), _p(g.adj), _p(g.weight),
                                  _p(groups.grp_ptr), _p(groups.members), gid.shape[0], _p(gid),
                                  hop_bound, C.byref(cost), C.byref(root), C.byref(root_d),
                                  C.byref(ne), cap, _p(eu), _p(ev), _p(ew), C.byref(esum),
                                  C.byref(pops))
    assert rc == 0, f"oracle failed rc={rc}"
    n = min(ne.value, cap)
    edges = np.stack([eu[:n], ev[:n], ew[:n]], axis=1)
    return {"cost": cost.value, "root": root.value, "edges": edges,
            "edge_sum": esum.value, "pops": pops.value}


def gst_nonhop(g, groups, group_ids):
    """Exact optimum of the group Steiner tree query (cost -1 = infeasible)."""
    return _solve(g, groups, group_ids, None)


def gst_hop(g, groups, group_ids, hop_bound: int):
    """Exact optimum of the hop-bounded DP of D-PrunedDP++ (cost -1 = infeasible)."""
    return _solve(g, groups, group_ids, hop_bound)


def nonhop_bound_check(g, groups, group_ids):
    """The unbounded DP pruned with the engine's rules (2c <= ub to grow, 3c <= 2ub to
    keep a merge, one-label and tour bounds at the source, the one-label bound and the
    O(k) tour bound on a grown target) against the star bound; its cost must equal
    gst_nonhop's.  Returns {cost, star (-1: none), pops}."""
    gid = np.ascontiguousarray(group_ids, dtype=np.int32)
    cost, star, pops = C.c_int64(), C.c_int64(), C.c_int64()
    rc = lib().oracle_nonhop_bound_check(g.V, _p(g.beg_pos), _p(g.adj), _p(g.weight),
                                         _p(groups.grp_ptr), _p(groups.members), gid.shape[0],
                                         _p(gid), C.byref(cost), C.byref(star), C.byref(pops))
    assert rc == 0, f"oracle failed rc={rc}"
    return {"cost": cost.value, "star": star.value, "pops": pops.value}


def hop_bound_check(g, groups, group_ids, hop_bound: int):
    """The hop-bounded DP pruned with the engine's bounds (the distances within each
    state's remaining hop budget, against the star of D/2-edge paths); its cost must
    equal gst_hop's.  Returns {cost, star (-1: none), pops}."""
    gid = np.ascontiguousarray(group_ids, dtype=np.int32)
    cost, star, pops = C.c_int64(), C.c_int64(), C.c_int64()
    rc = lib().oracle_hop_bound_check(g.V, _p(g.beg_pos), _p(g.adj), _p(g.weight),
                                      _p(groups.grp_ptr), _p(groups.members), gid.shape[0],
                                      _p(gid), hop_bound, C.byref(cost), C.byref(star),
                                      C.byref(pops))
    assert rc == 0, f"oracle failed rc={rc}"
    return {"cost": cost.value, "star": star.value, "pops": pops.value}


# ---- the reference's own CPU solvers ------------------------------------------

REF_SOLVERS = {
    # binary name: (argv type code, has hop bound, result-file prefix, cost column)
    "PrunedDP++": (1, False, "PrunedDP++_CPU_nonHop_", "CPU_nonHop_cost"),
    "TrimCDP-multi-core-CPU": (1, False, "TrimCDP-multi-core-CPU_", "CPU_nonHop_cost"),
    "D-PrunedDP++": (2, True, "D-PrunedDP++_", "CPU_Hop_cost"),
    "D-TrimCDP-multi-core-CPU": (2, True, None, None),
}


def ref_available(name: str) -> bool:
    return os.path.exists(os.path.join(REF_DIR, name))


def run_ref(name: str, data_dir: str, data_name: str, k: int, q_start: int, q_end: int,
            hop_bound: int | None = None, timeout: float | None = None):
    """Run one of the reference's CPU solvers (argv as in the reference README) on
    files written with gst_b200.write_reference_files; returns a list of dicts
    {task_id, time, cost} parsed from its result CSV, and the wall time."""
    code, hop, prefix, _ = REF_SOLVERS[name]
    exe = os.path.join(REF_DIR, name)
    os.makedirs(os.path.join(data_dir, "result"), exist_ok=True)
    path = data_dir.rstrip("/") + "/"
    args = [exe, str(code), path, data_name, str(k)]
    if hop:
        args.append(str(hop_bound))
    args += [str(q_start), str(q_end)]
    t0 = time.perf_counter()
    proc = subprocess.run(args, stdout=subprocess.PIPE, stderr=subprocess.STDOUT,
                          timeout=timeout, text=True)
    wall = time.perf_counter() - t0
    if proc.returncode != 0:
        raise RuntimeError(f"{name} failed rc={proc.returncode}: {proc.stdout[-2000:]}")
    rdir = os.path.join(data_dir, "result")
    cands = [f for f in os.listdir(rdir) if f.endswith(f"_{q_start}-{q_end}.csv")
             and data_name in f and (prefix is None or f.startswith(prefix))]
    if not cands:
        raise RuntimeError(f"{name}: no result csv in {rdir}")
    cands.sort(key=lambda f: os.path.getmtime(os.path.join(rdir, f)))
    rows = []
    with open(os.path.join(rdir, cands[-1])) as f:
        header = f.readline().strip().split(",")
        for line in f:
            line = line.strip()
            if not line:
                continue
            parts = line.split(",")
            rec = dict(zip(header, parts))
            cost_col = [h for h in header if h.endswith("_cost")][0]
            time_col = [h for h in header if h.endswith("_time")][0]
            rows.append({"task_id": int(rec["task_ID"]), "cost": int(float(rec[cost_col])),
                         "time": float(rec[time_col])})
    return rows, wall
