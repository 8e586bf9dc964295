"""ctypes view of the CPU oracle port (oracle/librg_oracle.so) and a runner for
the reference-built oracle (oracle/_ref/ref_driver).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline leg, never by the product package.
"""
from __future__ import annotations

import ctypes
import json
import os
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "librg_oracle.so")
REF_DRIVER = os.path.join(HERE, "_ref", "ref_driver")

ALGOS = {"bfs": 0, "sssp": 1, "sswp": 2, "wcc": 3}
WEIGHTED = {"bfs": False, "sssp": True, "sswp": True, "wcc": False}

_u64 = ctypes.c_uint64
_ptr = ctypes.c_void_p
_lib = None


def _p(a):
    return None if a is None else a.ctypes.data_as(_ptr)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"oracle port not built: {LIB_PATH} (run make -C oracle)")
        L = ctypes.CDLL(LIB_PATH)
        L.rgo_create.restype = _ptr
        L.rgo_create.argtypes = [_u64, _u64, ctypes.c_int, ctypes.c_int, ctypes.c_int]
        L.rgo_destroy.argtypes = [_ptr]
        for n in ("rgo_add_edge", "rgo_del_edge"):
            getattr(L, n).restype = _u64
            getattr(L, n).argtypes = [_ptr, _u64, _u64, _u64, ctypes.c_int]
        L.rgo_get_edge_num.restype = _u64
        L.rgo_get_edge_num.argtypes = [_ptr, _u64, _u64, _u64]
        L.rgo_get_outgoing_degree.restype = _u64
        L.rgo_get_outgoing_degree.argtypes = [_ptr, _u64]
        L.rgo_get_incoming_degree.restype = _u64
        L.rgo_get_incoming_degree.argtypes = [_ptr, _u64]
        L.rgo_build_tree.restype = _u64
        L.rgo_build_tree.argtypes = [_ptr, ctypes.c_int, _u64]
        for n in ("rgo_update_tree_add", "rgo_update_tree_del"):
            getattr(L, n).restype = _u64
            getattr(L, n).argtypes = [_ptr, ctypes.c_int, _u64, _u64, _u64, _u64, ctypes.c_int]
        for n in ("rgo_update_tree_add_batch", "rgo_update_tree_del_batch"):
            getattr(L, n).restype = _u64
            getattr(L, n).argtypes = [_ptr, ctypes.c_int, _u64, _ptr, _ptr, _ptr, _u64, ctypes.c_int]
        L.rgo_need_update_tree_add.restype = ctypes.c_int
        L.rgo_need_update_tree_add.argtypes = [_ptr, ctypes.c_int, _u64, _u64, _u64, ctypes.c_int]
        L.rgo_need_update_tree_del.restype = ctypes.c_int
        L.rgo_need_update_tree_del.argtypes = [_ptr, _u64, _u64, _u64, ctypes.c_int]
        L.rgo_get_labels.argtypes = [_ptr, _ptr, _ptr, _ptr]
        L.rgo_recomputes.restype = _u64
        L.rgo_recomputes.argtypes = [_ptr]
        L.rgo_run_inc.restype = _u64
        L.rgo_run_inc.argtypes = [_ptr, ctypes.c_int, _u64, _ptr, _u64, _u64, _u64, _ptr]
        L.rgo_run_batch.restype = _u64
        L.rgo_run_batch.argtypes = [_ptr, ctypes.c_int, _u64, _ptr, _u64, _u64, _u64, _u64, _ptr]
        L.rgo_load.argtypes = [_ptr, _ptr, _u64, ctypes.c_int]
        L.rgo_validate_tree.restype = _u64
        L.rgo_validate_tree.argtypes = [_ptr, ctypes.c_int, _u64, _ptr, _ptr, _ptr, ctypes.POINTER(ctypes.c_int)]
        L.rg_gen_value_checksum.restype = _u64
        L.rg_gen_value_checksum.argtypes = [_ptr, _u64]
        L.rg_gen_weight.restype = _u64
        L.rg_gen_weight.argtypes = [_u64, _u64]
        _lib = L
    return _lib


def checksum(values: np.ndarray) -> int:
    v = np.ascontiguousarray(values, dtype=np.uint64)
    return int(lib().rg_gen_value_checksum(_p(v), v.size))


class OracleGraph:
    """The reference's Graph (core/graph.hpp:41) for one algorithm's hooks."""

    def __init__(self, algo: str, vertices: int, hint_edges: int = 0, dual: bool | None = None,
                 inc_mode: bool = False):
        self.algo = algo
        self.a = ALGOS[algo]
        self.V = vertices
        self.symmetric = algo == "wcc"
        self.directed = algo != "wcc"
        if dual is None:
            dual = not (algo == "wcc" and inc_mode)
        self.h = lib().rgo_create(vertices, hint_edges, int(self.symmetric), int(dual), int(WEIGHTED[algo]))

    def close(self):
        if self.h:
            lib().rgo_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def load(self, pairs: np.ndarray):
        pairs = np.ascontiguousarray(pairs, dtype=np.uint64).reshape(-1)
        lib().rgo_load(self.h, _p(pairs), pairs.size // 2, int(self.directed))

    def add_edge(self, s, d, w=0):
        return lib().rgo_add_edge(self.h, s, d, w, int(self.directed))

    def del_edge(self, s, d, w=0):
        return lib().rgo_del_edge(self.h, s, d, w, int(self.directed))

    def get_edge_num(self, s, d, w=0):
        return lib().rgo_get_edge_num(self.h, s, d, w)

    def out_degree(self, v):
        return int(lib().rgo_get_outgoing_degree(self.h, v))

    def in_degree(self, v):
        return int(lib().rgo_get_incoming_degree(self.h, v))

    def build_tree(self, root=0):
        return lib().rgo_build_tree(self.h, self.a, root)

    def update_tree_add(self, s, d, w=0, root=0):
        return lib().rgo_update_tree_add(self.h, self.a, root, s, d, w, int(self.directed))

    def update_tree_del(self, s, d, w=0, root=0):
        return lib().rgo_update_tree_del(self.h, self.a, root, s, d, w, int(self.directed))

    def update_tree_add_batch(self, src, dst, w, root=0):
        src, dst, w = (np.ascontiguousarray(x, dtype=np.uint64) for x in (src, dst, w))
        return lib().rgo_update_tree_add_batch(self.h, self.a, root, _p(src), _p(dst), _p(w), src.size,
                                               int(self.directed))

    def update_tree_del_batch(self, src, dst, w, root=0):
        src, dst, w = (np.ascontiguousarray(x, dtype=np.uint64) for x in (src, dst, w))
        return lib().rgo_update_tree_del_batch(self.h, self.a, root, _p(src), _p(dst), _p(w), src.size,
                                               int(self.directed))

    def need_update_tree_add(self, s, d, w=0):
        return bool(lib().rgo_need_update_tree_add(self.h, self.a, s, d, w, int(self.directed)))

    def need_update_tree_del(self, s, d, w=0):
        return bool(lib().rgo_need_update_tree_del(self.h, s, d, w, int(self.directed)))

    def labels(self):
        val = np.empty(self.V, np.uint64)
        par = np.empty(self.V, np.uint64)
        pw = np.empty(self.V, np.uint64)
        lib().rgo_get_labels(self.h, _p(val), _p(par), _p(pw))
        return val, par, pw

    def run_inc(self, pairs, imported, steps, root=0):
        pairs = np.ascontiguousarray(pairs, dtype=np.uint64).reshape(-1)
        sums = np.zeros(steps, np.uint64)
        n = lib().rgo_run_inc(self.h, self.a, root, _p(pairs), pairs.size // 2, imported, steps, _p(sums))
        return sums[:n]

    def run_batch(self, pairs, imported, batch, n_batches, root=0):
        pairs = np.ascontiguousarray(pairs, dtype=np.uint64).reshape(-1)
        sums = np.zeros(n_batches, np.uint64)
        n = lib().rgo_run_batch(self.h, self.a, root, _p(pairs), pairs.size // 2, imported, batch, n_batches,
                                _p(sums))
        return sums[:n]

    def validate(self, val, par, pw, root=0):
        """0 if (val, par, pw) is a valid dependency tree of this graph, else (vertex, kind)."""
        val, par, pw = (np.ascontiguousarray(x, dtype=np.uint64) for x in (val, par, pw))
        kind = ctypes.c_int(0)
        r = lib().rgo_validate_tree(self.h, self.a, root, _p(val), _p(par), _p(pw), ctypes.byref(kind))
        return 0 if r == 0 else (int(r) - 1, kind.value)

    def recomputes(self):
        return int(lib().rgo_recomputes(self.h))


def ref_available() -> bool:
    return os.path.exists(REF_DRIVER)


def ref_run(mode: str, algo: str, pairs, V: int, root, *args, threads: int | None = None,
            workdir: str | None = None, timeout: float | None = None, bind: bool = False):
    """Run the reference-built oracle; returns (json, dict of arrays).

    `pairs` is an (n,2) uint64 array (written to a file in the reference's
    binary format) or a graph spec string the driver generates itself
    ("rmat:<scale>:<seed>", "mix:<scale>:<edges>:<seed>", optionally with an
    "@<lo>:<hi>" window).  `root` may be "maxdeg".  threads = OpenMP threads
    (all host cores when None); bind pins them (OMP_PROC_BIND=true)."""
    own = workdir is None
    tmp = workdir or tempfile.mkdtemp(prefix="rgref_")
    try:
        if isinstance(pairs, str):
            path = pairs
        else:
            path = os.path.join(tmp, "g.bin")
            np.ascontiguousarray(pairs, dtype=np.uint64).tofile(path)
        out = os.path.join(tmp, "out")
        cmd = [REF_DRIVER, mode, algo, path, str(V), str(root)] + [str(a) for a in args] + [out]
        if mode == "build" and args:
            cmd = [REF_DRIVER, mode, algo, path, str(V), str(root), out] + [str(a) for a in args]
        env = dict(os.environ)
        env["OMP_NUM_THREADS"] = str(threads or os.cpu_count() or 1)
        if bind:
            env["OMP_PROC_BIND"] = "true"
        r = subprocess.run(cmd, capture_output=True, text=True, env=env, timeout=timeout)
        if r.returncode != 0:
            raise RuntimeError(f"ref_driver {mode} {algo} failed ({r.returncode}): {r.stderr[-300:]}")
        info = json.loads(r.stdout.strip().splitlines()[-1])
        arrays = {}
        for ext in ("val", "par", "pw", "sums"):
            f = out + "." + ext
            if os.path.exists(f):
                arrays[ext] = np.fromfile(f, dtype=np.uint64)
        return info, arrays
    finally:
        if own:
            import shutil
            shutil.rmtree(tmp, ignore_errors=True)
