"""The no-allocation solve (gst_solve_noalloc) against the regular solve.

gst_solve_noalloc exists for callers that may not allocate device memory (their
host owns all of it through its own pool, and cudaMalloc/cudaFree would also
synchronise the device under their other work).  It takes the graph and groups
from device memory the caller already holds, writes the tree into caller-provided
host arrays, and keeps every scratch buffer in a static device array.  Here the
test itself provides the device copies (torch tensors); the entry point allocates
nothing.  Each query is solved twice in a row through the C ABI, and every answer
must equal gst_solve's exactly (cost and status) with a verified tree.

The file name sorts last so that a run stopping at the first failure has run
every other test before this one; it also passes alone in a fresh process.
"""
import ctypes as C

import numpy as np
import pytest

import gst_b200 as G
from conftest import golden_inputs, load_golden

pytestmark = pytest.mark.gpu

_lib = G._lib
_lib.gst_solve_noalloc.restype = C.c_int
_lib.gst_solve_noalloc.argtypes = [C.c_int32, C.c_void_p, C.c_int64, C.c_int64, C.c_void_p,
                                   C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p,
                                   C.POINTER(G.Query), C.c_int64, C.POINTER(G.Result)]


def _noalloc(dev, g, grp, q, hop, cap=4096):
    """One gst_solve_noalloc call; returns (return code, status, cost, edges, root)."""
    eu = np.zeros(cap, np.int32)
    ev = np.zeros(cap, np.int32)
    ew = np.zeros(cap, np.int32)
    gid = np.ascontiguousarray(q, dtype=np.int32)
    qs = G.Query(len(gid), gid.ctypes.data_as(C.POINTER(C.c_int32)),
                 -1 if hop is None else hop, 7)
    r = G.Result()
    r.edge_u = eu.ctypes.data_as(C.POINTER(C.c_int32))
    r.edge_v = ev.ctypes.data_as(C.POINTER(C.c_int32))
    r.edge_w = ew.ctypes.data_as(C.POINTER(C.c_int32))
    rc = _lib.gst_solve_noalloc(0, None, g.V, g.E, dev["beg"].data_ptr(), dev["edges"].data_ptr(),
                                grp.n_groups, dev["ptr"].data_ptr(), dev["mem"].data_ptr(),
                                C.byref(qs), cap, C.byref(r))
    n = int(r.n_edges)
    return rc, r.status, r.cost, np.stack([eu[:n], ev[:n], ew[:n]], axis=1), r.root


def _device_copies(g, grp):
    import torch
    edges = np.stack([g.adj, g.weight], axis=1).astype(np.int32).ravel()
    return {"beg": torch.from_numpy(g.beg_pos.copy()).cuda(),
            "edges": torch.from_numpy(edges).cuda(),
            "ptr": torch.from_numpy(grp.grp_ptr.copy()).cuda(),
            "mem": torch.from_numpy(grp.members.copy()).cuda()}


def test_noalloc_matches_solve_twice(engine):
    import torch
    fx = load_golden("rmat3k_k4_k5")
    g, grp = golden_inputs(fx)
    dev = _device_copies(g, grp)
    torch.cuda.synchronize()
    dg = engine.graph(g, grp)
    cases = []
    for case in fx["cases"]:
        for q in case["queries"][:6]:
            cases.append((q, case["hop"]))
    try:
        for call in range(2):  # two calls in a row share the static scratch
            for q, hop in cases:
                rc, st, cost, edges, root = _noalloc(dev, g, grp, q, hop)
                ref = dg.solve(q, hop)
                assert st == ref.status, (call, q, hop, G.STATUS[st], G.STATUS[ref.status])
                if ref.ok:
                    assert rc == G.OK and cost == ref.cost, (call, q, hop, cost, ref.cost)
                    vt = G.verify_tree(g, grp, q, -1 if hop is None else hop, cost, edges, root)
                    assert vt == 0, G.VERIFY_CODES[vt]
    finally:
        dg.close()


def test_noalloc_rejects_oversize():
    import torch
    g = G.synth_rmat(200_000, 400_000, 3)
    grp = G.synth_groups_zipf(g.V, 50, 1.5, 2, 20, 4)
    dev = _device_copies(g, grp)
    torch.cuda.synchronize()
    rc, st, *_ = _noalloc(dev, g, grp, list(range(8)), None)
    assert rc == G.OOM_ADMISSION and st == G.OOM_ADMISSION
    assert "static scratch" in _lib.gst_last_error_string(None).decode()


def test_noalloc_wide_rows_and_statuses(engine):
    """Hop-bounded rows wider than eight warps' shared memory (k = 8 at D = 7) through the
    no-allocation solve, the same as gst_solve; a tree with more edges than the caller's
    arrays hold returns GST_CAPACITY in both the return code and res.status."""
    import torch
    import oracle as O
    rng = np.random.default_rng(911)
    g = G.synth_rmat(500, 2500, 901)
    grp = G.synth_groups_zipf(g.V, 60, 1.5, 1, 12, 902)
    dev = _device_copies(g, grp)
    torch.cuda.synchronize()
    dg = engine.graph(g, grp)
    try:
        for k, D in ((8, 7), (7, 14), (5, None)):
            q = rng.choice(grp.n_groups, size=k, replace=False).astype(np.int32)
            want = O.gst_nonhop(g, grp, q)["cost"] if D is None else O.gst_hop(g, grp, q, D)["cost"]
            ref = dg.solve(q, D)
            for call in range(2):
                rc, st, cost, edges, root = _noalloc(dev, g, grp, q, D)
                assert st == ref.status and rc == st, (k, D, call, G.STATUS[st])
                if ref.ok:
                    assert cost == ref.cost == want, (k, D, cost, ref.cost, want)
                    vt = G.verify_tree(g, grp, q, -1 if D is None else D, cost, edges, root)
                    assert vt == 0, G.VERIFY_CODES[vt]
                else:
                    assert want == -1
        q = rng.choice(grp.n_groups, size=6, replace=False).astype(np.int32)
        ref = dg.solve(q)
        if ref.ok and len(ref.edges) > 1:
            rc, st, *_ = _noalloc(dev, g, grp, q, None, cap=1)
            assert rc == G.CAPACITY and st == G.CAPACITY, (rc, st)
    finally:
        dg.close()
