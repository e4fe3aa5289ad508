"""The drop-in boundary end to end on the GPU: the reference's own file formats and
argv.  A golden fixture is written in the reference's formats (int64 _beg_pos / _csr /
_weight.bin, .g, <name><k>.csv); gst_cli runs it with the argv of the reference's GPU
drivers (code/TrimCDP-WB/src/GSTnonHop.cu:160-165, code/D-TrimCDP-WB/src/GPUHop.cu:96-99)
and its result CSV's cost column must equal the costs the reference's solvers printed.
gst_graph_create_i64 takes the .bin arrays as read from disk."""
import csv
import os
import subprocess

import numpy as np
import pytest

import gst_b200 as G
from conftest import PKG, golden_inputs, load_golden

pytestmark = pytest.mark.gpu
REF_INF = 100000


def _result_costs(path):
    with open(path) as f:
        rows = [r for r in csv.reader(f) if r]
    hdr = rows[0]
    ci = [i for i, h in enumerate(hdr) if h.endswith("_cost")][0]
    return [int(r[ci]) for r in rows[1:]]


def test_cli_reference_argv_matches_golden(tmp_path):
    fx = load_golden("rmat3k_k4_k5")
    g, grp = golden_inputs(fx)
    cli = os.path.join(PKG, "gst_cli")
    assert os.path.exists(cli), "gst_cli is not built"
    d = str(tmp_path) + "/"
    seen = set()
    for case in fx["cases"]:
        k, hop = case["k"], case["hop"]
        q = np.asarray(case["queries"], dtype=np.int32)
        if k not in seen:
            G.write_reference_files(str(tmp_path), "fx", g, grp, q)
            seen.add(k)
        n = len(q)
        want = next(iter(case["ref"].values()))
        if hop is None:
            argv = [cli, "1", d, "fx", str(k), "0", str(n - 1)]
            out = tmp_path / "result" / f"TrimCDP-WB_fx_T{k}_0-{n - 1}.csv"
        else:
            argv = [cli, "2", d, "fx", str(k), str(hop), "0", str(n - 1)]
            out = tmp_path / "result" / f"D-TrimCDP-WB_fx_T{k}_D{hop}_0-{n - 1}.csv"
        os.makedirs(tmp_path / "result", exist_ok=True)
        p = subprocess.run(argv, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
        assert p.returncode == 0, p.stdout[-2000:]
        got = _result_costs(out)
        assert got == [min(c, REF_INF) for c in want], (k, hop)


def test_graph_create_i64_from_reference_bins(tmp_path, engine):
    fx = load_golden("rmat4k_k7_k8")
    g, grp = golden_inputs(fx)
    G.write_reference_files(str(tmp_path), "fx", g, grp)
    beg = np.fromfile(tmp_path / "fx_beg_pos.bin", dtype=np.int64)
    csr = np.fromfile(tmp_path / "fx_csr.bin", dtype=np.int64)
    wt = np.fromfile(tmp_path / "fx_weight.bin", dtype=np.int64)
    groups = G.read_reference_groups(str(tmp_path / "fx.g"))
    dg = G.DeviceGraph(engine, None, groups, i64=(beg, csr, wt))
    try:
        for case in fx["cases"]:
            hop = case["hop"]
            want = next(iter(case["ref"].values()))
            ans = dg.solve_batch(case["queries"], [hop] * len(case["queries"]))
            for q, a, c in zip(case["queries"], ans, want):
                expect = -1 if c >= REF_INF else c
                got = a.cost if a.ok else (-1 if a.status == G.INFEASIBLE else None)
                assert got == expect, (q, hop, G.STATUS[a.status])
                if a.ok:
                    assert G.verify_tree(g, grp, q, -1 if hop is None else hop, a.cost, a.edges,
                                         a.root) == 0
    finally:
        dg.close()
