"""risgraph_b200: B200-native incremental dependency-tree maintenance.

Python view of the C ABI in include/risgraph_b200.h, shaped like the
reference's Graph (core/graph.hpp:41): the same method names (add_edge,
del_edge, build_tree, update_tree_add, update_tree_del, need_update_tree_add,
need_update_tree_del), with the per-algorithm hooks chosen by name
("bfs", "sssp", "sswp", "wcc") instead of lambdas.  All work runs in
librisgraph_b200.so on the GPU; there is no CPU fallback, and a missing or
unloadable library raises.
"""
from __future__ import annotations

import ctypes
import os
import re

import numpy as np

__all__ = ["Graph", "Server", "Frontend", "RGError", "EDGE_DTYPE", "REQUEST_DTYPE", "COMPLETION_DTYPE",
           "CLIENT_REQUEST_DTYPE", "CLIENT_RESPONSE_DTYPE", "WAL_RECORD_DTYPE", "ALGOS", "lib", "gen", "wal_read",
           "wal_replay", "LIB_PATH"]

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "librisgraph_b200.so")
HEADER = os.path.join(os.path.dirname(PKG), "include", "risgraph_b200.h")

ALGOS = {"bfs": 0, "sssp": 1, "sswp": 2, "wcc": 3}
EDGE_DTYPE = np.dtype([("src", "<u8"), ("dst", "<u8"), ("data", "<u8")])  # rg_edge
REQUEST_DTYPE = np.dtype([("instance", "<u4"), ("type", "<u4"), ("src", "<u8"), ("dst", "<u8"), ("data", "<u8"),
                          ("tag", "<u8")])  # rg_request
COMPLETION_DTYPE = np.dtype([("tag", "<u8"), ("submit_ns", "<u8"), ("done_ns", "<u8"), ("instance", "<u4"),
                             ("type", "<u4"), ("status", "<i4"), ("epoch_size", "<u4"), ("version", "<u8")])  # rg_completion
# the reference's wire structs (core/rpc.hpp:19-38) and WAL record (src/all_inc_rpc.cpp:306-316)
CLIENT_REQUEST_DTYPE = np.dtype([("client_id", "<u4"), ("type", "<u4"), ("src", "<u8"), ("dst", "<u8"),
                                 ("data", "<u8"), ("request_time_ns", "<i8")])  # rg_client_update_request
CLIENT_RESPONSE_DTYPE = np.dtype([("client_id", "<u4"), ("pad", "<u4"), ("version_id", "<u8")])
WAL_RECORD_DTYPE = np.dtype([("type", "<u4"), ("client_id", "<u4"), ("src", "<u8"), ("dst", "<u8"),
                             ("data", "<u8")])  # rg_wal_record

_u64 = ctypes.c_uint64
_ptr = ctypes.c_void_p
_int = ctypes.c_int
_lib = None


class ServerStats(ctypes.Structure):  # rg_server_stats
    _fields_ = [("completed", ctypes.c_uint64), ("epochs", ctypes.c_uint64), ("largest_epoch", ctypes.c_uint64),
                ("p50_us", ctypes.c_double), ("p99_us", ctypes.c_double), ("p999_us", ctypes.c_double),
                ("max_us", ctypes.c_double), ("mean_us", ctypes.c_double)]


class FrontendStats(ctypes.Structure):  # rg_frontend_stats
    _fields_ = [("connections", ctypes.c_uint64), ("requests", ctypes.c_uint64), ("updates", ctypes.c_uint64),
                ("sync_requests", ctypes.c_uint64), ("wal_blocks", ctypes.c_uint64), ("failed", ctypes.c_uint64),
                ("time_offset_ns", ctypes.c_int64), ("p50_us", ctypes.c_double), ("p99_us", ctypes.c_double),
                ("p999_us", ctypes.c_double), ("max_us", ctypes.c_double), ("mean_us", ctypes.c_double)]


class TuneReport(ctypes.Structure):  # rg_tune_report
    _fields_ = [("build_ms_before", ctypes.c_double), ("build_ms_after", ctypes.c_double),
                ("apply_ms_before", ctypes.c_double), ("apply_ms_after", ctypes.c_double),
                ("options", ctypes.c_uint64 * 16), ("trials", ctypes.c_uint64)]


class LoadConfig(ctypes.Structure):  # rg_load_config
    _fields_ = [("instance", ctypes.c_uint32), ("clients", ctypes.c_uint32), ("think_us", ctypes.c_double),
                ("duration_s", ctypes.c_double), ("max_updates", ctypes.c_uint64), ("offset", ctypes.c_uint64),
                ("pairs", ctypes.c_void_p),
                ("n_pairs", ctypes.c_uint64), ("imported", ctypes.c_uint64), ("weighted", ctypes.c_int),
                ("open_loop", ctypes.c_int), ("seed", ctypes.c_uint64), ("latencies_ns", ctypes.c_void_p),
                ("latencies_cap", ctypes.c_uint64)]


class LoadResult(ctypes.Structure):  # rg_load_result
    _fields_ = [("completed", ctypes.c_uint64), ("adds", ctypes.c_uint64), ("dels", ctypes.c_uint64),
                ("failed", ctypes.c_uint64), ("seconds", ctypes.c_double), ("updates_per_s", ctypes.c_double),
                ("p50_us", ctypes.c_double), ("p99_us", ctypes.c_double), ("p999_us", ctypes.c_double),
                ("max_us", ctypes.c_double), ("mean_us", ctypes.c_double), ("epochs", ctypes.c_uint64),
                ("mean_epoch", ctypes.c_double)]


class RGError(RuntimeError):
    def __init__(self, status: int, where: str):
        L = lib()
        msg = L.rg_last_error().decode() or L.rg_status_string(status).decode()
        super().__init__(f"{where}: {msg} (status {status})")
        self.status = status


def _declare(L):
    P = _ptr
    sig = {
        "rg_create": [_u64, _u64, _int, _int, _int, _int, P],
        "rg_destroy": [P],
        "rg_add_edges": [P, P, _u64, _int, P],
        "rg_del_edges": [P, P, _u64, _int, P],
        "rg_add_pairs": [P, P, _u64, _int, P],
        "rg_del_pairs": [P, P, _u64, _int, P],
        "rg_get_edge_num": [P, P, _u64, P],
        "rg_get_degrees": [P, P, P],
        "rg_build_tree": [P, _int, _u64, P],
        "rg_update_tree_add": [P, _int, P, _u64, _int, P],
        "rg_update_tree_del": [P, _int, P, _u64, _int, P],
        "rg_classify": [P, _int, P, P, _u64, _int, P],
        "rg_apply_add": [P, _int, P, _u64, _int, P],
        "rg_apply_del": [P, _int, P, _u64, _int, P],
        "rg_apply_add_del": [P, _int, P, _u64, P, _u64, _int],
        "rg_apply_add_pairs": [P, _int, P, _u64, _int, P],
        "rg_apply_del_pairs": [P, _int, P, _u64, _int, P],
        "rg_get_labels": [P, P, P, P],
        "rg_get_modified": [P, P, _u64, P],
        "rg_clear_modified": [P],
        "rg_value_checksum": [P, P],
        "rg_last_stats": [P, P, P, P],
        "rg_device_bytes": [P, P],
        "rg_set_stream": [P, P],
        "rg_get_stream": [P, P],
        "rg_launch_count": [P, P],
        "rg_profile": [P, _int],
        "rg_profile_read": [P, P, P],
        "rg_level_trace": [P, P, _u64, P, P],
        "rg_level_times": [P, P, _u64, P],
        "rg_phase_trace": [P, P],
        "rg_level_stamps": [P, P, _u64, P],
        "rg_build_tree_csr_static": [_int, _u64, _u64, _u64, P, P, P, P, P, P],
        "rg_set_option": [P, _int, _u64],
        "rg_get_option": [P, _int, P],
        "rg_autotune": [P, _int, _u64, P, _u64, _int, _int, P],
        "rg_history_enable": [P, _u64],
        "rg_history_record": [P, _u64, _int],
        "rg_history_get": [P, P, _u64, _u64, P, P],
        "rg_history_gc": [P, _u64],
        "rg_history_nodes": [P, P, P],
        "rg_server_create": [_u64, ctypes.c_double, _u64, _int, P],
        "rg_server_attach": [P, P, _int, _int, P],
        "rg_server_detach": [P, ctypes.c_uint32],
        "rg_server_history": [P, ctypes.c_uint32, _int, P],
        "rg_server_submit": [P, P, _u64],
        "rg_server_poll": [P, P, _u64, P],
        "rg_server_drain": [P, _u64],
        "rg_server_stats_get": [P, P, _int],
        "rg_server_run_load": [P, P, _u64, P],
        "rg_server_destroy": [P],
        "rg_server_poll_wait": [P, P, _u64, P, _u64],
        "rg_frontend_start": [P, ctypes.c_uint32, ctypes.c_char_p, ctypes.c_uint16, ctypes.c_char_p, ctypes.c_uint32,
                              P],
        "rg_frontend_port": [P, P],
        "rg_frontend_stats_get": [P, P],
        "rg_frontend_stop": [P, _u64],
        "rg_wal_read": [ctypes.c_char_p, P, _u64, P],
        "rg_wal_replay": [P, _int, ctypes.c_char_p, _int, P],
    }
    for name, args in sig.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = _int
    L.rg_status_string.argtypes = [_int]
    L.rg_status_string.restype = ctypes.c_char_p
    L.rg_last_error.argtypes = []
    L.rg_last_error.restype = ctypes.c_char_p
    for name, args, res in [
        ("rg_gen_splitmix64", [_u64], _u64),
        ("rg_gen_weight", [_u64, _u64], _u64),
        ("rg_gen_rmat", [ctypes.c_uint32, _u64, _u64, ctypes.c_double, ctypes.c_double, ctypes.c_double, _u64, P],
         None),
        ("rg_gen_er_rmat_mix",
         [ctypes.c_uint32, _u64, _u64, ctypes.c_double, ctypes.c_double, ctypes.c_double, _u64, P], None),
        ("rg_gen_weights", [P, _u64, P], None),
        ("rg_gen_max_out_degree_vertex", [P, _u64, _u64], _u64),
        ("rg_gen_write_binary", [ctypes.c_char_p, P, _u64], _int),
        ("rg_gen_value_checksum", [P, _u64], _u64),
    ]:
        f = getattr(L, name)
        f.argtypes = args
        f.restype = res


def lib():
    """Load librisgraph_b200.so (built in-tree by risgraph_b200.build)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m risgraph_b200.build`")
        L = ctypes.CDLL(LIB_PATH)
        _declare(L)
        _lib = L
    return _lib


def header_functions(path: str = HEADER) -> list[str]:
    """Function names declared in a C header of include/."""
    src = open(path).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return re.findall(r"^\s*(?:const\s+)?[A-Za-z_][\w\s\*]*?\b(rg\w*)\s*\(", src, flags=re.M)


def _p(a):
    return None if a is None else ctypes.c_void_p(a.ctypes.data)


def _check(rc, where):
    if rc != 0:
        raise RGError(rc, where)


def as_edges(edges) -> np.ndarray:
    """Accept an rg_edge structured array, an (n,3) or (n,2) integer array."""
    if isinstance(edges, np.ndarray) and edges.dtype == EDGE_DTYPE:
        return np.ascontiguousarray(edges)
    a = np.asarray(edges, dtype=np.uint64)
    if a.ndim == 1:
        a = a.reshape(1, -1)
    out = np.zeros(a.shape[0], EDGE_DTYPE)
    out["src"] = a[:, 0]
    out["dst"] = a[:, 1]
    if a.shape[1] > 2:
        out["data"] = a[:, 2]
    return out


class Graph:
    """Device-resident evolving graph with one dependency-tree label array.

    Constructor arguments follow Graph(vertices, hint_edges, symmetric, dual,
    trace_modified) of core/graph.hpp:61-100; `weighted` chooses
    Graph<uint64_t> over Graph<void>.
    """

    def __init__(self, vertices: int, hint_edges: int = 0, symmetric: bool = False, dual: bool = True,
                 trace_modified: bool = False, weighted: bool = False):
        self.vertices = int(vertices)
        self.symmetric = bool(symmetric)
        self.weighted = bool(weighted)
        self.trace_modified = bool(trace_modified)
        h = ctypes.c_void_p()
        _check(lib().rg_create(self.vertices, int(hint_edges), int(symmetric), int(dual), int(trace_modified),
                               int(weighted), ctypes.byref(h)), "rg_create")
        self._h = h
        self.algo = None

    # -- lifecycle
    def close(self):
        if getattr(self, "_h", None):
            lib().rg_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # -- adjacency (core/graph.hpp:198-253)
    def _edge_op(self, fn, edges, directed, where):
        e = as_edges(edges)
        old = np.zeros(len(e), np.uint64)
        _check(fn(self._h, _p(e), len(e), int(directed), _p(old)), where)
        return old

    def add_edges(self, edges, directed: bool = True) -> np.ndarray:
        return self._edge_op(lib().rg_add_edges, edges, directed, "rg_add_edges")

    def del_edges(self, edges, directed: bool = True) -> np.ndarray:
        return self._edge_op(lib().rg_del_edges, edges, directed, "rg_del_edges")

    def add_edge(self, src, dst, data=0, directed: bool = True) -> int:
        return int(self.add_edges([(src, dst, data)], directed)[0])

    def del_edge(self, src, dst, data=0, directed: bool = True) -> int:
        return int(self.del_edges([(src, dst, data)], directed)[0])

    def _pair_op(self, fn, pairs, directed, where, want_old=True):
        p = np.ascontiguousarray(pairs, dtype=np.uint64).reshape(-1)
        n = p.size // 2
        old = np.zeros(n, np.uint64) if want_old else None
        _check(fn(self._h, _p(p), n, int(directed), _p(old)), where)
        return old

    def add_pairs(self, pairs, directed: bool = True, want_old: bool = True):
        return self._pair_op(lib().rg_add_pairs, pairs, directed, "rg_add_pairs", want_old)

    def del_pairs(self, pairs, directed: bool = True, want_old: bool = True):
        return self._pair_op(lib().rg_del_pairs, pairs, directed, "rg_del_pairs", want_old)

    def get_edge_num(self, edges) -> np.ndarray:
        e = as_edges(edges)
        out = np.zeros(len(e), np.uint64)
        _check(lib().rg_get_edge_num(self._h, _p(e), len(e), _p(out)), "rg_get_edge_num")
        return out

    def degrees(self):
        o = np.zeros(self.vertices, np.uint64)
        i = np.zeros(self.vertices, np.uint64)
        _check(lib().rg_get_degrees(self._h, _p(o), _p(i)), "rg_get_degrees")
        return o, i

    # -- trees (core/graph.hpp:873-1718)
    def build_tree(self, algo: str, root: int = 0) -> int:
        tot = np.zeros(1, np.uint64)
        _check(lib().rg_build_tree(self._h, ALGOS[algo], int(root), _p(tot)), "rg_build_tree")
        self.algo = algo
        return int(tot[0])

    def update_tree_add(self, algo: str, edges, directed: bool = True) -> int:
        e = as_edges(edges)
        tot = np.zeros(1, np.uint64)
        _check(lib().rg_update_tree_add(self._h, ALGOS[algo], _p(e), len(e), int(directed), _p(tot)),
               "rg_update_tree_add")
        return int(tot[0])

    def update_tree_del(self, algo: str, edges, directed: bool = True) -> int:
        e = as_edges(edges)
        tot = np.zeros(1, np.uint64)
        _check(lib().rg_update_tree_del(self._h, ALGOS[algo], _p(e), len(e), int(directed), _p(tot)),
               "rg_update_tree_del")
        return int(tot[0])

    def classify(self, algo: str, edges, is_del=None, directed: bool = True) -> np.ndarray:
        e = as_edges(edges)
        out = np.zeros(len(e), np.uint8)
        d = None if is_del is None else np.ascontiguousarray(is_del, dtype=np.uint8)
        _check(lib().rg_classify(self._h, ALGOS[algo], _p(e), _p(d), len(e), int(directed), _p(out)),
               "rg_classify")
        return out

    def need_update_tree_add(self, algo: str, edge, directed: bool = True) -> bool:
        return bool(self.classify(algo, [edge], None, directed)[0])

    def need_update_tree_del(self, algo: str, edge, directed: bool = True) -> bool:
        return bool(self.classify(algo, [edge], np.ones(1, np.uint8), directed)[0])

    def apply_add(self, algo: str, edges, directed: bool = True) -> np.ndarray:
        return self._apply(lib().rg_apply_add, algo, as_edges(edges), directed, "rg_apply_add")

    def apply_del(self, algo: str, edges, directed: bool = True) -> np.ndarray:
        return self._apply(lib().rg_apply_del, algo, as_edges(edges), directed, "rg_apply_del")

    def apply_add_del(self, algo: str, adds, dels, directed: bool = True):
        """rg_apply_add of `adds` then rg_apply_del of `dels` in one submission."""
        a, d = as_edges(adds), as_edges(dels)
        _check(lib().rg_apply_add_del(self._h, ALGOS[algo], _p(a), len(a), _p(d), len(d), int(directed)),
               "rg_apply_add_del")
        self.algo = algo

    def apply_add_pairs(self, algo: str, pairs, directed: bool = True, want_old: bool = False):
        p = np.ascontiguousarray(pairs, dtype=np.uint64).reshape(-1)
        return self._apply(lib().rg_apply_add_pairs, algo, p, directed, "rg_apply_add_pairs", p.size // 2, want_old)

    def apply_del_pairs(self, algo: str, pairs, directed: bool = True, want_old: bool = False):
        p = np.ascontiguousarray(pairs, dtype=np.uint64).reshape(-1)
        return self._apply(lib().rg_apply_del_pairs, algo, p, directed, "rg_apply_del_pairs", p.size // 2, want_old)

    def _apply(self, fn, algo, arr, directed, where, n=None, want_old=True):
        n = len(arr) if n is None else n
        old = np.zeros(n, np.uint64) if want_old else None
        _check(fn(self._h, ALGOS[algo], _p(arr), n, int(directed), _p(old)), where)
        return old

    # -- results
    def labels(self, value=True, parent=True, parent_w=True):
        V = self.vertices
        val = np.empty(V, np.uint64) if value else None
        par = np.empty(V, np.uint64) if parent else None
        pw = np.empty(V, np.uint64) if parent_w else None
        _check(lib().rg_get_labels(self._h, _p(val), _p(par), _p(pw)), "rg_get_labels")
        return val, par, pw

    def values(self) -> np.ndarray:
        return self.labels(True, False, False)[0]

    def autotune(self, algo: str, root: int = 0, sample=None, directed: bool = True, reps: int = 5) -> dict:
        """rg_autotune: pick the level-mode options for this graph; returns the report."""
        rep = TuneReport()
        e = as_edges(sample) if sample is not None else None
        _check(lib().rg_autotune(self._h, ALGOS[algo], int(root), _p(e), 0 if e is None else len(e), int(directed),
                                 int(reps), ctypes.byref(rep)), "rg_autotune")
        self.algo = algo
        names = {v: k for k, v in self.OPTIONS.items()}
        return {"build_ms_before": rep.build_ms_before, "build_ms_after": rep.build_ms_after,
                "apply_ms_before": rep.apply_ms_before, "apply_ms_after": rep.apply_ms_after,
                "options": {names[i]: int(rep.options[i]) for i in range(16) if i in names},
                "trials": int(rep.trials)}

    # -- versioned label history (MVVec, core/mvvec.hpp)
    def history_enable(self, capacity_nodes: int):
        _check(lib().rg_history_enable(self._h, int(capacity_nodes)), "rg_history_enable")

    def history_record(self, version: int, all_vertices: bool = False):
        _check(lib().rg_history_record(self._h, int(version), int(all_vertices)), "rg_history_record")

    def history_get(self, vids, version: int):
        """(values, found) of the vertices as of `version`."""
        v = np.ascontiguousarray(vids, dtype=np.uint64)
        out = np.zeros(len(v), np.uint64)
        found = np.zeros(len(v), np.uint8)
        _check(lib().rg_history_get(self._h, _p(v), len(v), int(version), _p(out), _p(found)), "rg_history_get")
        return out, found.astype(bool)

    def history_gc(self, version: int):
        _check(lib().rg_history_gc(self._h, int(version)), "rg_history_gc")

    def history_nodes(self):
        u = np.zeros(2, np.uint64)
        _check(lib().rg_history_nodes(self._h, _p(u[0:1]), _p(u[1:2])), "rg_history_nodes")
        return int(u[0]), int(u[1])

    def checksum(self) -> int:
        c = np.zeros(1, np.uint64)
        _check(lib().rg_value_checksum(self._h, _p(c)), "rg_value_checksum")
        return int(c[0])

    def get_modified(self) -> np.ndarray:
        n = np.zeros(1, np.uint64)
        _check(lib().rg_get_modified(self._h, None, 0, _p(n)), "rg_get_modified")
        out = np.zeros(int(n[0]), np.uint64)
        _check(lib().rg_get_modified(self._h, _p(out), len(out), _p(n)), "rg_get_modified")
        return out

    def clear_modified(self):
        _check(lib().rg_clear_modified(self._h), "rg_clear_modified")

    def last_stats(self):
        a = np.zeros(3, np.uint64)
        _check(lib().rg_last_stats(self._h, _p(a[0:1]), _p(a[1:2]), _p(a[2:3])), "rg_last_stats")
        return {"levels": int(a[0]), "invalidated": int(a[1]), "recomputes": int(a[2])}

    def set_stream(self, stream_ptr: int | None):
        """Run this graph's work on a raw cudaStream_t (e.g. torch.cuda.Stream().cuda_stream)."""
        _check(lib().rg_set_stream(self._h, ctypes.c_void_p(stream_ptr or 0)), "rg_set_stream")

    def launch_count(self) -> int:
        n = np.zeros(1, np.uint64)
        _check(lib().rg_launch_count(self._h, _p(n)), "rg_launch_count")
        return int(n[0])

    def profile(self, enable: bool = True):
        _check(lib().rg_profile(self._h, int(enable)), "rg_profile")

    def profile_read(self):
        n = np.zeros(1, np.uint64)
        ms = np.zeros(1, np.float64)
        _check(lib().rg_profile_read(self._h, _p(n), _p(ms)), "rg_profile_read")
        return int(n[0]), float(ms[0])

    def level_trace(self):
        """(frontier sizes per push level, edge slots scanned) of the last tree call."""
        n = np.zeros(1, np.uint64)
        e = np.zeros(1, np.uint64)
        _check(lib().rg_level_trace(self._h, None, 0, _p(n), _p(e)), "rg_level_trace")
        sizes = np.zeros(int(n[0]), np.uint64)
        _check(lib().rg_level_trace(self._h, _p(sizes), len(sizes), _p(n), _p(e)), "rg_level_trace")
        return sizes, int(e[0])

    def level_device_times(self):
        """Per level device ms of the last tree call from the level loop's own
        device-clock stamps (graph-launched calls included)."""
        n = np.zeros(1, np.uint64)
        _check(lib().rg_level_stamps(self._h, None, 0, _p(n)), "rg_level_stamps")
        ns = np.zeros(int(n[0]) + 1, np.uint64)
        _check(lib().rg_level_stamps(self._h, _p(ns), len(ns), _p(n)), "rg_level_stamps")
        return np.diff(ns.astype(np.int64)) / 1e6

    OPTIONS = {"dense_pull": 0, "dense_div": 1, "lbs_min": 2, "bfs_bottom_up": 3, "recompute_min": 4, "bu_div": 5,
               "pull_div": 6, "tiny_edges": 7, "pull_split": 8, "max_levels": 9,
               "pull_groups": 10, "fused_max": 11, "phase_trace": 12, "inline_max": 13, "cluster_edges": 14}

    # rg_phase_trace's phase words (RG_PH_* in the header), in order
    PHASES = ("begin", "unpack", "lookup", "grow", "write", "count", "old", "seed", "del_repair", "end")

    def set_option(self, name: str, value: int):
        _check(lib().rg_set_option(self._h, self.OPTIONS[name], int(value)), "rg_set_option")

    def get_option(self, name: str) -> int:
        v = np.zeros(1, np.uint64)
        _check(lib().rg_get_option(self._h, self.OPTIONS[name], _p(v)), "rg_get_option")
        return int(v[0])

    def level_times(self):
        """Per push level device ms of the last tree call (profile() must be on)."""
        n = np.zeros(1, np.uint64)
        _check(lib().rg_level_times(self._h, None, 0, _p(n)), "rg_level_times")
        ms = np.zeros(int(n[0]), np.float64)
        _check(lib().rg_level_times(self._h, _p(ms), len(ms), _p(n)), "rg_level_times")
        return ms

    def phase_times(self):
        """Device time (us) of each phase of the last fused submission, per
        batch that ran in a fused kernel: {"insert"|"delete": {phase: us}},
        plus "staging" (header and edges across the bus) per kernel.  The
        phase_trace option must be on; a phase a batch skipped is absent."""
        t = np.zeros(64, np.uint64)
        _check(lib().rg_phase_trace(self._h, _p(t)), "rg_phase_trace")
        out = {}
        for b, name in ((0, "insert"), (1, "delete")):
            w = t[16 * b:16 * b + 16].astype(np.int64)
            if w[15] != 1:
                continue
            d, prev = {"staging": (int(t[33 + 2 * b]) - int(t[32 + 2 * b])) / 1e3}, int(w[0])
            for k in range(1, len(self.PHASES)):
                if w[k] >= prev and w[k] - prev < 10**9:
                    d[self.PHASES[k]] = (int(w[k]) - prev) / 1e3
                    prev = int(w[k])
            d["total"] = (prev - int(w[0])) / 1e3
            out[name] = d
        return out

    def device_bytes(self) -> int:
        b = np.zeros(1, np.uint64)
        _check(lib().rg_device_bytes(self._h, _p(b)), "rg_device_bytes")
        return int(b[0])


from . import gen  # noqa: E402  (synthetic inputs; needs lib())


def _struct_dict(st) -> dict:
    return {name: getattr(st, name) for name, _ in st._fields_}


class Server:
    """Served mode (rg_server_*): continuous batching of single-edge updates
    over resident graph instances admitted against an HBM budget.

    per_update=True applies every update alone (the plain one-update path).
    While a graph is attached, only the server may touch it; detach (or
    close) before calling the graph's own methods again.
    """

    def __init__(self, hbm_budget_bytes: int = 0, target_epoch_ms: float = 0.5, max_epoch: int = 65536,
                 per_update: bool = False):
        h = ctypes.c_void_p()
        _check(lib().rg_server_create(int(hbm_budget_bytes), float(target_epoch_ms), int(max_epoch),
                                      int(per_update), ctypes.byref(h)), "rg_server_create")
        self._h = h
        self._graphs = {}

    def close(self):
        if getattr(self, "_h", None):
            lib().rg_server_destroy(self._h)
            self._h = None
            self._graphs = {}

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def attach(self, graph: Graph, directed: bool = True) -> int:
        if graph.algo is None:
            raise RuntimeError("build the graph's tree before attaching it")
        inst = ctypes.c_uint32()
        _check(lib().rg_server_attach(self._h, graph._h, ALGOS[graph.algo], int(directed), ctypes.byref(inst)),
               "rg_server_attach")
        self._graphs[inst.value] = graph
        return inst.value

    def history(self, instance: int, enable: bool = True) -> int:
        """Record the label history after every epoch; returns the last version."""
        v = np.zeros(1, np.uint64)
        _check(lib().rg_server_history(self._h, int(instance), int(enable), _p(v)), "rg_server_history")
        return int(v[0])

    def detach(self, instance: int):
        _check(lib().rg_server_detach(self._h, int(instance)), "rg_server_detach")
        self._graphs.pop(int(instance), None)

    def submit(self, requests):
        r = np.ascontiguousarray(requests, dtype=REQUEST_DTYPE)
        _check(lib().rg_server_submit(self._h, _p(r), len(r)), "rg_server_submit")

    def poll(self, cap: int = 1 << 16) -> np.ndarray:
        out = np.zeros(cap, dtype=COMPLETION_DTYPE)
        n = _u64()
        _check(lib().rg_server_poll(self._h, _p(out), cap, ctypes.byref(n)), "rg_server_poll")
        return out[: n.value]

    def drain(self, timeout_ms: int = 60000):
        _check(lib().rg_server_drain(self._h, int(timeout_ms)), "rg_server_drain")

    def stats(self, reset: bool = False) -> dict:
        st = ServerStats()
        _check(lib().rg_server_stats_get(self._h, ctypes.byref(st), int(reset)), "rg_server_stats_get")
        return _struct_dict(st)

    def run_load(self, loads) -> list[dict]:
        """loads: dicts with instance, clients, pairs (uint64 (n,2)), imported,
        and optionally think_us, duration_s, max_updates, offset, weighted, open_loop, seed."""
        keep = []
        cfgs = (LoadConfig * len(loads))()
        for i, d in enumerate(loads):
            pairs = np.ascontiguousarray(d["pairs"], dtype=np.uint64).reshape(-1, 2)
            keep.append(pairs)
            cfgs[i] = LoadConfig(int(d["instance"]), int(d["clients"]), float(d.get("think_us", 0.0)),
                                 float(d.get("duration_s", 1.0)), int(d.get("max_updates", 0)),
                                 int(d.get("offset", 0)), pairs.ctypes.data, len(pairs), int(d["imported"]),
                                 int(d.get("weighted", 0)), int(d.get("open_loop", 0)), int(d.get("seed", 1)), None, 0)
        res = (LoadResult * len(loads))()
        _check(lib().rg_server_run_load(self._h, cfgs, len(loads), res), "rg_server_run_load")
        return [_struct_dict(r) for r in res]


class Frontend:
    """Network front end (rg_frontend_*): the reference's ClientUpdateRequest /
    ClientUpdateResponse structs (core/rpc.hpp:19-38) over TCP into one
    instance of a Server, with an optional write-ahead log (group commit,
    src/all_inc_rpc.cpp:306-335).  The server should be one that nothing else
    polls: the front end drains its completions."""

    def __init__(self, server: "Server", instance: int, host: str = "127.0.0.1", port: int = 0,
                 wal_path: str | None = None, sync_requests: int = 0):
        h = ctypes.c_void_p()
        _check(lib().rg_frontend_start(server._h, int(instance), host.encode(), int(port),
                                       wal_path.encode() if wal_path else None, int(sync_requests), ctypes.byref(h)),
               "rg_frontend_start")
        self._h = h
        p = ctypes.c_uint16()
        _check(lib().rg_frontend_port(self._h, ctypes.byref(p)), "rg_frontend_port")
        self.port = p.value

    def stats(self) -> dict:
        st = FrontendStats()
        _check(lib().rg_frontend_stats_get(self._h, ctypes.byref(st)), "rg_frontend_stats_get")
        return _struct_dict(st)

    def stop(self, timeout_ms: int = 60000):
        if getattr(self, "_h", None):
            h, self._h = self._h, None
            _check(lib().rg_frontend_stop(h, int(timeout_ms)), "rg_frontend_stop")

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.stop()


def wal_read(path: str) -> np.ndarray:
    """The records of a WAL file, in log order (WAL_RECORD_DTYPE)."""
    n = _u64()
    _check(lib().rg_wal_read(path.encode(), None, 0, ctypes.byref(n)), "rg_wal_read")
    out = np.zeros(n.value, WAL_RECORD_DTYPE)
    _check(lib().rg_wal_read(path.encode(), _p(out), n.value, ctypes.byref(n)), "rg_wal_read")
    return out


def wal_replay(graph: Graph, algo: str, path: str, directed: bool = True) -> int:
    """Re-apply a WAL to a graph whose labels are built for algo; returns the records applied."""
    n = _u64()
    _check(lib().rg_wal_replay(graph._h, ALGOS[algo], path.encode(), int(directed), ctypes.byref(n)),
           "rg_wal_replay")
    return n.value
