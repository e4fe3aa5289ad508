"""The C ABI library loads and exports every function that include/*.h declares
(CPU only: nothing here touches a device)."""
import ctypes as C
import os
import re

import gst_b200 as G

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
INC = os.path.join(ROOT, "include")


def declared_functions():
    names = set()
    for fn in sorted(os.listdir(INC)):
        if not fn.endswith(".h"):
            continue
        with open(os.path.join(INC, fn)) as f:
            src = f.read()
        src = re.sub(r"/\*.*?\*/", " ", src, flags=re.S)
        src = re.sub(r"//[^\n]*", " ", src)
        src = "\n".join(l for l in src.splitlines() if not l.lstrip().startswith("#"))
        src = src.replace('extern "C" {', ";").replace("}", ";").replace("{", ";")
        # a declaration: return type tokens, the gst_ name, an argument list, ';'
        for stmt in src.split(";"):
            m = re.fullmatch(r"\s*(?:const\s+)?\w+\s*\**\s*(gst_\w+)\s*\([^()]*\)\s*", stmt,
                             flags=re.S)
            if m:
                names.add(m.group(1))
    return sorted(names)


def test_headers_declare_the_entry_points():
    names = declared_functions()
    for must in ("gst_engine_create", "gst_graph_create", "gst_groups_create", "gst_solve",
                 "gst_solve_batch", "gst_result_free", "gst_last_error_string",
                 "gst_verify_tree", "gst_read_reference_bin", "gst_write_reference_files"):
        assert must in names, must


def test_library_exports_every_declared_symbol():
    lib = C.CDLL(G.LIB_PATH)
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, f"{G.LIB_PATH} lacks {missing}"


def test_binding_covers_engine_symbols():
    lib = C.CDLL(G.LIB_PATH)
    for n in G.C_ABI_SYMBOLS:
        assert hasattr(lib, n), n


def test_build_tracks_every_device_header():
    """A kernel edited in any csrc header rebuilds the library (every .cuh is a
    dependency of the CUDA sources), so a stale library is never tested or timed."""
    import build
    csrc = os.path.join(os.path.dirname(G.__file__), "csrc")
    cuh = sorted(f for f in os.listdir(csrc) if f.endswith(".cuh"))
    assert cuh and set(cuh) <= set(build.HEADERS), (cuh, build.HEADERS)
    lib = G.LIB_PATH
    deps = [os.path.join(csrc, f) for f in cuh]
    assert not build._stale(lib, deps) or not os.path.exists(lib)


def test_stats_layout_matches_header():
    """gst_stats in include/gst.h and the binding's Stats list the same fields in order."""
    with open(os.path.join(INC, "gst.h")) as f:
        src = f.read()
    body = src[src.index("typedef struct gst_stats"):]
    body = body[:body.index("} gst_stats;")]
    body = re.sub(r"/\*.*?\*/", " ", body, flags=re.S)
    fields = re.findall(r"(?:int64_t|double|int32_t)\s+(\w+);", body)
    assert fields == [n for n, _ in G.Stats._fields_]
