"""ctypes binding of the GST engine's C ABI (include/gst.h, include/gst_io.h).

This module is a thin host-side view of ``libgst_b200.so``: numpy arrays in,
numpy arrays out.  Every solve runs in the CUDA engine behind the C ABI; there is
no Python or CPU solver here.  If the shared library is missing, importing this
module raises, and the engine calls raise ``GstError`` when no CUDA device is
usable — nothing falls back to the CPU.

The query interface mirrors what the reference's drivers pass per query
(code/TrimCDP-WB/src/GSTnonHop.cu:247-497, code/D-TrimCDP-WB/src/GPUHop.cu:172-266):
a CSR graph (beg_pos / csr / weight), a list of vertex groups, and k group ids,
optionally with a hop (diameter) bound D; the result is the optimal cost and the
tree's edge set.
"""
from __future__ import annotations

import ctypes as C
import os
import weakref
from dataclasses import dataclass, field

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
# GST_CHECKED=1 selects the bounds-checked build of the same engine (debugging aid)
LIB_PATH = os.path.join(_HERE, "libgst_b200_checked.so" if os.environ.get("GST_CHECKED") == "1"
                        else "libgst_b200.so")

if not os.path.exists(LIB_PATH):
    raise ImportError(
        f"{LIB_PATH} is missing: build it with `python {_HERE}/build.py` "
        "(the engine has no fallback without its CUDA library)")

_lib = C.CDLL(LIB_PATH)

_i32p = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_i64p = np.ctypeslib.ndpointer(dtype=np.int64, flags="C_CONTIGUOUS")


class HostGraph(C.Structure):
    _fields_ = [("V", C.c_int64), ("E", C.c_int64), ("beg_pos", C.POINTER(C.c_int64)),
                ("adj", C.POINTER(C.c_int32)), ("weight", C.POINTER(C.c_int32))]


class HostGroups(C.Structure):
    _fields_ = [("n_groups", C.c_int32), ("grp_ptr", C.POINTER(C.c_int64)),
                ("members", C.POINTER(C.c_int32))]


def _sig(name, res, args):
    f = getattr(_lib, name)
    f.restype = res
    f.argtypes = args
    return f


_sig("gst_host_graph_free", None, [C.POINTER(HostGraph)])
_sig("gst_host_groups_free", None, [C.POINTER(HostGroups)])
_sig("gst_synth_ba", C.c_int, [C.c_int64, C.c_int32, C.c_uint64, C.c_int32, C.c_int32,
                               C.POINTER(HostGraph)])
_sig("gst_synth_rmat", C.c_int, [C.c_int64, C.c_int64, C.c_double, C.c_double, C.c_double,
                                 C.c_uint64, C.c_int32, C.c_int32, C.c_int32,
                                 C.POINTER(HostGraph)])
_sig("gst_synth_groups_uniform", C.c_int, [C.c_int64, C.c_int32, C.c_int32, C.c_int32,
                                           C.c_uint64, C.POINTER(HostGroups)])
_sig("gst_synth_groups_zipf", C.c_int, [C.c_int64, C.c_int32, C.c_double, C.c_int32,
                                        C.c_int32, C.c_uint64, C.POINTER(HostGroups)])
_sig("gst_synth_queries", C.c_int, [C.c_int32, C.c_int32, C.c_int32, C.c_uint64, _i32p])
_sig("gst_write_reference_files", C.c_int,
     [C.c_char_p, C.c_char_p, C.POINTER(HostGraph), C.POINTER(HostGroups), C.c_int32,
      C.c_int32, C.c_void_p])
_sig("gst_read_reference_bin", C.c_int, [C.c_char_p, C.c_char_p, C.POINTER(HostGraph)])
_sig("gst_read_reference_in", C.c_int, [C.c_char_p, C.POINTER(HostGraph)])
_sig("gst_read_reference_groups", C.c_int, [C.c_char_p, C.POINTER(HostGroups)])
_sig("gst_read_reference_queries", C.c_int32,
     [C.c_char_p, C.c_int32, C.POINTER(C.c_int32), C.c_void_p])
_sig("gst_verify_tree", C.c_int32,
     [C.POINTER(HostGraph), C.POINTER(HostGroups), C.c_int32, _i32p, C.c_int32, C.c_int64,
      C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32])


class GstError(RuntimeError):
    pass


@dataclass
class Graph:
    """CSR graph, both directions stored, adjacency sorted by neighbour id."""
    beg_pos: np.ndarray  # int64[V+1]
    adj: np.ndarray      # int32[E]
    weight: np.ndarray   # int32[E]

    @property
    def V(self) -> int:
        return int(self.beg_pos.shape[0] - 1)

    @property
    def E(self) -> int:
        return int(self.adj.shape[0])

    def host(self) -> HostGraph:
        self.beg_pos = np.ascontiguousarray(self.beg_pos, dtype=np.int64)
        self.adj = np.ascontiguousarray(self.adj, dtype=np.int32)
        self.weight = np.ascontiguousarray(self.weight, dtype=np.int32)
        return HostGraph(self.V, self.E,
                         self.beg_pos.ctypes.data_as(C.POINTER(C.c_int64)),
                         self.adj.ctypes.data_as(C.POINTER(C.c_int32)),
                         self.weight.ctypes.data_as(C.POINTER(C.c_int32)))


@dataclass
class Groups:
    """Vertex groups in CSR form: members of g are members[grp_ptr[g]:grp_ptr[g+1]]."""
    grp_ptr: np.ndarray  # int64[n+1]
    members: np.ndarray  # int32

    @property
    def n_groups(self) -> int:
        return int(self.grp_ptr.shape[0] - 1)

    def host(self) -> HostGroups:
        self.grp_ptr = np.ascontiguousarray(self.grp_ptr, dtype=np.int64)
        self.members = np.ascontiguousarray(self.members, dtype=np.int32)
        return HostGroups(self.n_groups, self.grp_ptr.ctypes.data_as(C.POINTER(C.c_int64)),
                          self.members.ctypes.data_as(C.POINTER(C.c_int32)))

    @staticmethod
    def from_lists(lists) -> "Groups":
        ptr = np.zeros(len(lists) + 1, dtype=np.int64)
        ptr[1:] = np.cumsum([len(x) for x in lists])
        mem = np.concatenate([np.sort(np.asarray(x, dtype=np.int32)) for x in lists]) \
            if lists else np.zeros(0, dtype=np.int32)
        return Groups(ptr, mem.astype(np.int32))


def _take_graph(hg: HostGraph) -> Graph:
    V, E = hg.V, hg.E
    g = Graph(np.ctypeslib.as_array(hg.beg_pos, shape=(V + 1,)).copy(),
              np.ctypeslib.as_array(hg.adj, shape=(E,)).copy() if E else np.zeros(0, np.int32),
              np.ctypeslib.as_array(hg.weight, shape=(E,)).copy() if E else np.zeros(0, np.int32))
    _lib.gst_host_graph_free(C.byref(hg))
    return g


def _take_groups(hg: HostGroups) -> Groups:
    n = hg.n_groups
    ptr = np.ctypeslib.as_array(hg.grp_ptr, shape=(n + 1,)).copy()
    m = int(ptr[-1])
    mem = np.ctypeslib.as_array(hg.members, shape=(m,)).copy() if m else np.zeros(0, np.int32)
    _lib.gst_host_groups_free(C.byref(hg))
    return Groups(ptr, mem)


# ---- synthetic inputs -------------------------------------------------------

def synth_ba(V: int, m: int, seed: int, wmin: int = 1, wmax: int = 100) -> Graph:
    hg = HostGraph()
    if _lib.gst_synth_ba(V, m, seed, wmin, wmax, C.byref(hg)):
        raise GstError("gst_synth_ba: bad arguments")
    return _take_graph(hg)


def synth_rmat(V: int, n_undirected: int, seed: int, a=0.57, b=0.19, c=0.19,
               wmin: int = 1, wmax: int = 100, keep_lcc: bool = True) -> Graph:
    hg = HostGraph()
    if _lib.gst_synth_rmat(V, n_undirected, a, b, c, seed, wmin, wmax, int(keep_lcc),
                           C.byref(hg)):
        raise GstError("gst_synth_rmat: bad arguments")
    return _take_graph(hg)


def synth_groups_uniform(V: int, n_groups: int, smin: int, smax: int, seed: int) -> Groups:
    hg = HostGroups()
    if _lib.gst_synth_groups_uniform(V, n_groups, smin, smax, seed, C.byref(hg)):
        raise GstError("gst_synth_groups_uniform: bad arguments")
    return _take_groups(hg)


def synth_groups_zipf(V: int, n_groups: int, s: float, smin: int, smax: int,
                      seed: int) -> Groups:
    hg = HostGroups()
    if _lib.gst_synth_groups_zipf(V, n_groups, s, smin, smax, seed, C.byref(hg)):
        raise GstError("gst_synth_groups_zipf: bad arguments")
    return _take_groups(hg)


def synth_queries(n_groups: int, n_queries: int, k: int, seed: int) -> np.ndarray:
    out = np.zeros(n_queries * k, dtype=np.int32)
    if _lib.gst_synth_queries(n_groups, n_queries, k, seed, out):
        raise GstError("gst_synth_queries: bad arguments")
    return out.reshape(n_queries, k)


# ---- reference formats ------------------------------------------------------

def write_reference_files(dirname: str, name: str, g: Graph, groups: Groups | None = None,
                          queries: np.ndarray | None = None) -> None:
    hg = g.host()
    hgr = groups.host() if groups is not None else None
    nq, k, qp = 0, 0, None
    if queries is not None and len(queries):
        q = np.ascontiguousarray(queries, dtype=np.int32)
        nq, k, qp = q.shape[0], q.shape[1], q.ctypes.data
    rc = _lib.gst_write_reference_files(dirname.encode(), name.encode(), C.byref(hg),
                                        C.byref(hgr) if hgr is not None else None, nq, k, qp)
    if rc:
        raise GstError(f"gst_write_reference_files failed ({rc})")


def read_reference_bin(dirname: str, name: str) -> Graph:
    hg = HostGraph()
    rc = _lib.gst_read_reference_bin(dirname.encode(), name.encode(), C.byref(hg))
    if rc:
        raise GstError(f"gst_read_reference_bin failed ({rc})")
    return _take_graph(hg)


def read_reference_in(path: str) -> Graph:
    hg = HostGraph()
    rc = _lib.gst_read_reference_in(path.encode(), C.byref(hg))
    if rc:
        raise GstError(f"gst_read_reference_in failed ({rc})")
    return _take_graph(hg)


def read_reference_groups(path: str) -> Groups:
    hg = HostGroups()
    rc = _lib.gst_read_reference_groups(path.encode(), C.byref(hg))
    if rc:
        raise GstError(f"gst_read_reference_groups failed ({rc})")
    return _take_groups(hg)


def read_reference_queries(path: str) -> np.ndarray:
    k = C.c_int32(0)
    n = _lib.gst_read_reference_queries(path.encode(), 0, C.byref(k), None)
    if n < 0:
        raise GstError(f"cannot read queries from {path}")
    out = np.zeros(max(n * k.value, 1), dtype=np.int32)
    _lib.gst_read_reference_queries(path.encode(), n, C.byref(k), out.ctypes.data)
    return out[: n * k.value].reshape(n, k.value)


VERIFY_CODES = {0: "ok", 1: "edge not in graph or wrong weight", 2: "disconnected",
                3: "group not covered", 4: "weight sum != cost", 5: "diameter > hop bound",
                6: "cycle", 7: "bad argument"}


def verify_tree(g: Graph, groups: Groups, group_ids, hop_bound: int, cost: int,
                edges: np.ndarray, root: int) -> int:
    """0 if `edges` (n x 3: u, v, w) is a valid answer tree of cost `cost`."""
    hg, hgr = g.host(), groups.host()
    gid = np.ascontiguousarray(group_ids, dtype=np.int32)
    e = np.ascontiguousarray(edges, dtype=np.int32).reshape(-1, 3)
    u = np.ascontiguousarray(e[:, 0])
    v = np.ascontiguousarray(e[:, 1])
    w = np.ascontiguousarray(e[:, 2])
    return int(_lib.gst_verify_tree(C.byref(hg), C.byref(hgr), len(gid), gid, hop_bound, cost,
                                    e.shape[0], u.ctypes.data, v.ctypes.data, w.ctypes.data,
                                    root))


# ---- engine (include/gst.h) -------------------------------------------------

STATUS = {0: "OK", 1: "INFEASIBLE", 2: "OOM_ADMISSION", 3: "BAD_INPUT", 4: "TIMEOUT",
          5: "DEVICE_ERROR", 6: "CAPACITY", 7: "NOT_READY"}
OK, INFEASIBLE, OOM_ADMISSION, BAD_INPUT, TIMEOUT, DEVICE_ERROR, CAPACITY, NOT_READY = range(8)


class Config(C.Structure):
    _fields_ = [("mem_budget_bytes", C.c_int64), ("split_degree", C.c_int32),
                ("bucket_delta", C.c_int32), ("max_levels", C.c_int32),
                ("threads_per_block", C.c_int32), ("blocks_per_sm", C.c_int32),
                ("max_batch", C.c_int32), ("use_graphs", C.c_int32),
                ("profile_kernels", C.c_int32), ("verbose", C.c_int32),
                ("hop_cut_mult", C.c_int32), ("search_cut_permille", C.c_int32),
                ("hop_cut_permille", C.c_int32), ("batch_search", C.c_int32)]


class Query(C.Structure):
    _fields_ = [("k", C.c_int32), ("group_ids", C.POINTER(C.c_int32)),
                ("hop_bound", C.c_int32), ("user_tag", C.c_uint64)]


class Stats(C.Structure):
    _fields_ = [("levels", C.c_int64), ("states_expanded", C.c_int64),
                ("edge_relaxations", C.c_int64), ("merge_pairs", C.c_int64),
                ("rows_merged", C.c_int64), ("sssp_relaxations", C.c_int64),
                ("kernel_launches", C.c_int64), ("h2d_bytes", C.c_int64),
                ("d2h_bytes", C.c_int64), ("device_ms", C.c_double), ("latency_ms", C.c_double),
                ("grow_ms", C.c_double), ("rows_ms", C.c_double), ("sssp_ms", C.c_double),
                ("queue_max", C.c_int64), ("grow_launches", C.c_int64),
                ("rows_launches", C.c_int64), ("sssp_launches", C.c_int64),
                ("shared_sectors", C.c_int64), ("shared_ms", C.c_double),
                ("shared_launches", C.c_int64), ("shared_relax_launches", C.c_int64),
                ("shared_relax_ms", C.c_double)]


class Result(C.Structure):
    _fields_ = [("status", C.c_int32), ("cost", C.c_int32), ("root", C.c_int32),
                ("root_hop", C.c_int32), ("n_edges", C.c_int64),
                ("edge_u", C.POINTER(C.c_int32)), ("edge_v", C.POINTER(C.c_int32)),
                ("edge_w", C.POINTER(C.c_int32)), ("user_tag", C.c_uint64), ("stats", Stats)]


_vp = C.c_void_p
_sig("gst_config_default", None, [C.POINTER(Config)])
_sig("gst_engine_create", C.c_int, [C.c_int32, C.POINTER(Config), C.POINTER(_vp)])
_sig("gst_engine_destroy", C.c_int, [_vp])
_sig("gst_last_error_string", C.c_char_p, [_vp])
_sig("gst_graph_create", C.c_int, [_vp, C.c_int64, C.c_int64, _vp, _vp, _vp, C.POINTER(_vp)])
_sig("gst_graph_create_i64", C.c_int, [_vp, C.c_int64, C.c_int64, _vp, _vp, _vp,
                                       C.POINTER(_vp)])
_sig("gst_graph_destroy", C.c_int, [_vp])
_sig("gst_groups_create", C.c_int, [_vp, C.c_int32, _vp, _vp, C.POINTER(_vp)])
_sig("gst_groups_destroy", C.c_int, [_vp])
_sig("gst_solve", C.c_int, [_vp, _vp, C.POINTER(Query), C.POINTER(Result)])
_sig("gst_solve_batch", C.c_int, [_vp, _vp, C.c_int32, C.POINTER(Query), C.POINTER(Result)])
_sig("gst_result_free", None, [C.POINTER(Result)])
_sig("gst_engine_set_profiling", C.c_int, [_vp, C.c_int32])
_sig("gst_autotune", C.c_int, [_vp, _vp, C.c_int32, C.POINTER(Query), C.c_char_p,
                               C.POINTER(Config)])
_sig("gst_server_create", C.c_int, [_vp, _vp, C.POINTER(_vp)])
_sig("gst_submit", C.c_int, [_vp, C.POINTER(Query), C.POINTER(C.c_uint64)])
_sig("gst_poll", C.c_int, [_vp, C.c_uint64, C.POINTER(Result)])
_sig("gst_wait", C.c_int, [_vp, C.c_uint64, C.POINTER(Result)])
_sig("gst_server_destroy", C.c_int, [_vp])
_sig("gst_probe_random_access", C.c_int, [C.c_int32, C.c_int64, C.POINTER(C.c_double),
                                          C.POINTER(C.c_double), C.POINTER(C.c_double)])

C_ABI_SYMBOLS = [
    "gst_config_default", "gst_engine_create", "gst_engine_destroy", "gst_last_error_string",
    "gst_graph_create", "gst_graph_create_i64", "gst_graph_destroy", "gst_groups_create",
    "gst_groups_destroy", "gst_solve", "gst_solve_batch", "gst_result_free",
    "gst_server_create", "gst_submit", "gst_poll", "gst_wait", "gst_server_destroy",
    "gst_debug_slot_state", "gst_solve_noalloc", "gst_engine_set_profiling", "gst_autotune",
    "gst_groups_cache_warm", "gst_groups_cache_warm_hop", "gst_probe_random_access",
]


def probe_random_access(device: int = 0, nbytes: int = 4 << 30) -> dict:
    """Random-access ceilings of the device (include/gst.h: gst_probe_random_access):
    random 32-byte row gathers per second from `nbytes` and from an L2-resident 32 MB,
    and random 4-byte atomicMin reductions per second."""
    g, l2, red = C.c_double(), C.c_double(), C.c_double()
    rc = _lib.gst_probe_random_access(device, nbytes, C.byref(g), C.byref(l2), C.byref(red))
    if rc:
        raise GstError(f"gst_probe_random_access: {STATUS.get(rc, rc)}")
    return {"gather32_dram_per_s": g.value, "gather32_l2_per_s": l2.value,
            "red32_dram_per_s": red.value, "bytes": nbytes}


def set_profiling(eng: "Engine", bits: int) -> None:
    """Bracket the grow (1) / rows (2) / sssp (4) launches of later solves with CUDA
    events (include/gst.h: gst_engine_set_profiling)."""
    rc = _lib.gst_engine_set_profiling(eng._h, bits)
    if rc:
        raise GstError(f"gst_engine_set_profiling: {STATUS.get(rc, rc)}")


def default_config(**kw) -> Config:
    c = Config()
    _lib.gst_config_default(C.byref(c))
    for k, v in kw.items():
        setattr(c, k, v)
    return c


@dataclass
class Answer:
    status: int
    cost: int
    root: int
    root_hop: int
    edges: np.ndarray            # n x 3 (u, v, w), u < v
    stats: dict = field(default_factory=dict)
    user_tag: int = 0

    @property
    def ok(self) -> bool:
        return self.status == OK


def _answer(r: Result) -> Answer:
    n = int(r.n_edges)
    if n > 0:
        e = np.stack([np.ctypeslib.as_array(r.edge_u, shape=(n,)).copy(),
                      np.ctypeslib.as_array(r.edge_v, shape=(n,)).copy(),
                      np.ctypeslib.as_array(r.edge_w, shape=(n,)).copy()], axis=1)
    else:
        e = np.zeros((0, 3), dtype=np.int32)
    st = {f: getattr(r.stats, f) for f, _ in Stats._fields_}
    a = Answer(int(r.status), int(r.cost), int(r.root), int(r.root_hop), e, st, int(r.user_tag))
    _lib.gst_result_free(C.byref(r))
    return a


class Engine:
    """One engine per CUDA device (include/gst.h: gst_engine_create)."""

    def __init__(self, device: int = 0, config: Config | None = None, **kw):
        self._h = _vp()
        self._graphs = weakref.WeakSet()  # closed before the engine
        cfg = config if config is not None else default_config(**kw)
        rc = _lib.gst_engine_create(device, C.byref(cfg), C.byref(self._h))
        if rc:
            raise GstError(f"gst_engine_create: {STATUS.get(rc, rc)}: "
                           f"{_lib.gst_last_error_string(None).decode()}")

    def error(self) -> str:
        return _lib.gst_last_error_string(self._h).decode()

    def close(self):
        if self._h:
            for dg in list(self._graphs):
                dg.close()
            _lib.gst_engine_destroy(self._h)
            self._h = _vp()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def graph(self, g: Graph, groups: Groups) -> "DeviceGraph":
        return DeviceGraph(self, g, groups)


class DeviceGraph:
    """A graph and its groups resident on the engine's device.  With `i64` = (beg_pos,
    csr, weight) int64 arrays (the reference's _beg_pos/_csr/_weight.bin as read) the
    graph goes through gst_graph_create_i64 instead, and `g` may be None."""

    def __init__(self, eng: Engine, g: Graph | None, groups: Groups, i64=None):
        self.eng, self.g, self.groups = eng, g, groups
        self._g, self._grp = _vp(), _vp()
        self._servers = weakref.WeakSet()  # closed before the graph
        eng._graphs.add(self)
        if i64 is not None:
            beg, csr, wt = (np.ascontiguousarray(a, dtype=np.int64) for a in i64)
            rc = _lib.gst_graph_create_i64(eng._h, beg.shape[0] - 1, csr.shape[0], beg.ctypes.data,
                                           csr.ctypes.data, wt.ctypes.data, C.byref(self._g))
            if rc:
                raise GstError(f"gst_graph_create_i64: {STATUS.get(rc, rc)}: {eng.error()}")
        else:
            hg = g.host()
            rc = _lib.gst_graph_create(eng._h, g.V, g.E, hg.beg_pos, hg.adj, hg.weight,
                                       C.byref(self._g))
            if rc:
                raise GstError(f"gst_graph_create: {STATUS.get(rc, rc)}: {eng.error()}")
        gr = groups.host()
        rc = _lib.gst_groups_create(self._g, gr.n_groups, gr.grp_ptr, gr.members,
                                    C.byref(self._grp))
        if rc:
            raise GstError(f"gst_groups_create: {STATUS.get(rc, rc)}: {eng.error()}")

    def cache_warm(self, group_ids, max_bytes: int) -> int:
        """Keep the one-label distances of these groups on the device (include/gst.h:
        gst_groups_cache_warm); returns how many of them are cached."""
        a = np.ascontiguousarray(group_ids, dtype=np.int32)
        n = C.c_int32(0)
        rc = _lib.gst_groups_cache_warm(self._grp, len(a), a.ctypes.data_as(C.POINTER(C.c_int32)),
                                        C.c_int64(max_bytes), C.byref(n))
        if rc:
            raise GstError(f"gst_groups_cache_warm: {STATUS.get(rc, rc)}: {self.eng.error()}")
        return n.value

    def cache_warm_hop(self, group_ids, hop_bound: int, max_bytes: int) -> int:
        """The same for hop-bounded queries with this bound (include/gst.h:
        gst_groups_cache_warm_hop)."""
        a = np.ascontiguousarray(group_ids, dtype=np.int32)
        n = C.c_int32(0)
        rc = _lib.gst_groups_cache_warm_hop(self._grp, len(a),
                                            a.ctypes.data_as(C.POINTER(C.c_int32)),
                                            C.c_int32(hop_bound), C.c_int64(max_bytes),
                                            C.byref(n))
        if rc:
            raise GstError(f"gst_groups_cache_warm_hop: {STATUS.get(rc, rc)}: {self.eng.error()}")
        return n.value

    def close(self):
        for sv in list(self._servers):
            sv.close()
        if self._grp:
            _lib.gst_groups_destroy(self._grp)
            self._grp = _vp()
        if self._g:
            _lib.gst_graph_destroy(self._g)
            self._g = _vp()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @staticmethod
    def _queries(group_ids_list, hop_bounds, tags):
        n = len(group_ids_list)
        qs = (Query * max(n, 1))()
        keep = []
        for i, gids in enumerate(group_ids_list):
            a = np.ascontiguousarray(gids, dtype=np.int32)
            keep.append(a)
            hb = hop_bounds[i] if hop_bounds is not None else -1
            qs[i] = Query(len(a), a.ctypes.data_as(C.POINTER(C.c_int32)),
                          -1 if hb is None else int(hb), tags[i] if tags is not None else i)
        return qs, keep

    def solve(self, group_ids, hop_bound: int | None = None) -> Answer:
        qs, keep = self._queries([group_ids], [hop_bound], None)
        r = Result()
        rc = _lib.gst_solve(self._g, self._grp, C.byref(qs[0]), C.byref(r))
        if rc not in (OK, INFEASIBLE, BAD_INPUT, TIMEOUT, CAPACITY, OOM_ADMISSION,
                      DEVICE_ERROR):
            raise GstError(f"gst_solve: {STATUS.get(rc, rc)}: {self.eng.error()}")
        return _answer(r)

    def solve_batch(self, group_ids_list, hop_bounds=None) -> list:
        n = len(group_ids_list)
        qs, keep = self._queries(group_ids_list, hop_bounds, None)
        rs = (Result * max(n, 1))()
        rc = _lib.gst_solve_batch(self._g, self._grp, n, qs, rs)
        if rc != OK:
            raise GstError(f"gst_solve_batch: {STATUS.get(rc, rc)}: {self.eng.error()}")
        return [_answer(rs[i]) for i in range(n)]

    def server(self) -> "Server":
        return Server(self)

    def autotune(self, group_ids_list, hop_bounds=None, cache_path: str | None = None) -> dict:
        """Choose launch parameters for this graph's shape on a sample of queries
        (include/gst.h: gst_autotune); returns the chosen settings."""
        n = len(group_ids_list)
        qs, keep = self._queries(group_ids_list, hop_bounds, None)
        cfg = Config()
        rc = _lib.gst_autotune(self._g, self._grp, n, qs,
                               cache_path.encode() if cache_path else None, C.byref(cfg))
        if rc:
            raise GstError(f"gst_autotune: {STATUS.get(rc, rc)}: {self.eng.error()}")
        return {f: getattr(cfg, f) for f, _ in Config._fields_}


class Server:
    """Continuous-batching server over a resident graph (include/gst.h:
    gst_server_create / gst_submit / gst_poll / gst_wait).  Queries are admitted
    into free slots at DP-level boundaries while others run on the GPU."""

    def __init__(self, dg: DeviceGraph):
        self.dg = dg
        self._h = _vp()
        dg._servers.add(self)
        rc = _lib.gst_server_create(dg._g, dg._grp, C.byref(self._h))
        if rc:
            raise GstError(f"gst_server_create: {STATUS.get(rc, rc)}: {dg.eng.error()}")

    def submit(self, group_ids, hop_bound: int | None = None, tag: int = 0) -> int:
        a = np.ascontiguousarray(group_ids, dtype=np.int32)
        q = Query(len(a), a.ctypes.data_as(C.POINTER(C.c_int32)),
                  -1 if hop_bound is None else int(hop_bound), tag)
        t = C.c_uint64(0)
        rc = _lib.gst_submit(self._h, C.byref(q), C.byref(t))
        if rc:
            raise GstError(f"gst_submit: {STATUS.get(rc, rc)}: {self.dg.eng.error()}")
        return int(t.value)

    def poll(self, ticket: int):
        """The Answer, or None while the query runs."""
        r = Result()
        rc = _lib.gst_poll(self._h, ticket, C.byref(r))
        if rc == NOT_READY:
            return None
        if rc == BAD_INPUT and r.status == 0:
            raise GstError(f"gst_poll: {self.dg.eng.error()}")
        return _answer(r)

    def wait(self, ticket: int) -> Answer:
        r = Result()
        _lib.gst_wait(self._h, ticket, C.byref(r))
        return _answer(r)

    def close(self):
        if self._h:
            _lib.gst_server_destroy(self._h)
            self._h = _vp()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
