"""rg_build_tree_csr_static, the build_tree entry point that allocates nothing.

It exists for callers that may not allocate device memory when they need a
tree: a serving process whose device memory belongs to another framework's
pool, fixed at start-up, or a latency-critical path where cudaMalloc/cudaFree
would synchronise the device.  It keeps its working memory in one static
device array (RG_STATIC_MAX_VERTICES vertices at most) and works on a CSR the
caller already holds in device memory.

This file runs last (pytest collects test_zz_* after the others), calls the
entry point through the C ABI twice in a row per algorithm, and checks the
values against rg_build_tree on the same graph (exact: the values are
integers) and the parents structurally.  It passes in a fresh process and
after the rest of the suite.
"""
import ctypes

import numpy as np
import pytest

import risgraph_b200 as rg
from risgraph_b200 import gen

from helpers import ALGOS, WEIGHTED, gpu_graph, oracle_graph

pytestmark = pytest.mark.gpu

MAX_V = 1 << 20


def csr(pairs, V, algo):
    """Distinct edges of the graph the reference drivers build, as CSR."""
    p = np.asarray(pairs, dtype=np.uint64).reshape(-1, 2)
    src, dst = p[:, 0].astype(np.int64), p[:, 1].astype(np.int64)
    if algo == "wcc":   # undirected: both orientations
        src, dst = np.concatenate([src, dst]), np.concatenate([dst, src])
    key = np.unique(src * V + dst)
    s, d = key // V, key % V
    row = np.zeros(V + 1, np.int64)
    np.add.at(row, s + 1, 1)
    row = np.cumsum(row)
    w = None
    if WEIGHTED[algo]:
        w = gen.weights(np.stack([s, d], 1).astype(np.uint64)).astype(np.int32)
    return row, d.astype(np.int32), w


def run_static(algo, V, row, col, w, root):
    import torch
    dev = torch.device("cuda")
    t_row = torch.from_numpy(row).to(dev)
    t_col = torch.from_numpy(col).to(dev)
    t_w = torch.from_numpy(w).to(dev) if w is not None else None
    vals = torch.empty(V, dtype=torch.int64, device=dev)
    pars = torch.empty(V, dtype=torch.int64, device=dev)
    stream = torch.cuda.current_stream().cuda_stream
    rc = rg.lib().rg_build_tree_csr_static(
        rg.ALGOS[algo], root, V, len(col), ctypes.c_void_p(t_row.data_ptr()), ctypes.c_void_p(t_col.data_ptr()),
        ctypes.c_void_p(t_w.data_ptr()) if t_w is not None else None, ctypes.c_void_p(vals.data_ptr()),
        ctypes.c_void_p(pars.data_ptr()), ctypes.c_void_p(stream))
    assert rc == 0, rg.lib().rg_last_error().decode()
    torch.cuda.synchronize()
    return vals.cpu().numpy().view(np.uint64), pars.cpu().numpy().view(np.uint64)


@pytest.mark.parametrize("algo", ALGOS)
def test_static_build_matches_rg_build_tree(algo):
    scale = 14
    pairs = gen.rmat(scale, seed=17)
    V = 1 << scale
    root = gen.max_out_degree_vertex(pairs, V)
    g = gpu_graph(algo, V, pairs)
    g.build_tree(algo, root)
    expect = g.values()
    og = oracle_graph(algo, V, pairs)
    row, col, w = csr(pairs, V, algo)
    for _ in range(2):   # two calls in a row share the static scratch
        vals, pars = run_static(algo, V, row, col, w, root)
        np.testing.assert_array_equal(vals, expect)
        pw = np.zeros(V, np.uint64)
        if WEIGHTED[algo]:
            has = pars < V
            # weight of the parent edge: the CSR weight of (parent -> v)
            key = np.repeat(np.arange(V), np.diff(row)) * V + col.astype(np.int64)
            lut = dict(zip(key.tolist(), w.tolist()))
            for v in np.nonzero(has)[0].tolist():
                pw[v] = lut[int(pars[v]) * V + v]
        assert og.validate(vals, pars, pw, root) == 0


def static_call(algo, V, E, row, col, w, vals, pars, root=0):
    P = ctypes.c_void_p
    return rg.lib().rg_build_tree_csr_static(
        rg.ALGOS[algo], root, V, E, P(row.data_ptr()), P(col.data_ptr()), P(w.data_ptr()) if w is not None else None,
        P(vals.data_ptr()), P(pars.data_ptr()), None)


@pytest.mark.parametrize("algo", ["sssp", "wcc"])
def test_static_build_at_the_vertex_limit(algo):
    """A graph of exactly RG_STATIC_MAX_VERTICES vertices reaches the ends of
    the label, queue and stamp regions of the static array (WCC starts with
    every vertex in the queue)."""
    scale = 20
    pairs = gen.rmat(scale, n_edges=4 << scale, seed=23)
    V = 1 << scale
    assert V == MAX_V
    root = gen.max_out_degree_vertex(pairs, V)
    g = gpu_graph(algo, V, pairs)
    g.build_tree(algo, root)
    expect = g.values()
    g.close()
    row, col, w = csr(pairs, V, algo)
    vals, _ = run_static(algo, V, row, col, w, root)
    np.testing.assert_array_equal(vals, expect)


def test_static_setup_call_and_no_device_allocation():
    """The set-up call (vertices == 0, every pointer NULL) succeeds; after a
    first build, a second build of the same graph leaves the device's free
    memory unchanged: the call takes nothing beyond its static array."""
    import torch
    assert rg.lib().rg_build_tree_csr_static(0, 0, 0, 0, None, None, None, None, None, None) == 0
    scale = 12
    pairs = gen.rmat(scale, seed=29)
    V = 1 << scale
    row, col, w = csr(pairs, V, "sssp")
    dev = torch.device("cuda")
    t_row, t_col, t_w = (torch.from_numpy(x).to(dev) for x in (row, col, w))
    vals = torch.empty(V, dtype=torch.int64, device=dev)
    pars = torch.empty(V, dtype=torch.int64, device=dev)
    assert static_call("sssp", V, len(col), t_row, t_col, t_w, vals, pars) == 0
    torch.cuda.synchronize()
    first = vals.clone()
    free0, _ = torch.cuda.mem_get_info()
    assert static_call("sssp", V, len(col), t_row, t_col, t_w, vals, pars) == 0
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0
    assert torch.equal(first, vals)


def test_static_rejects_malformed_csr_and_missing_weights():
    """Each malformed input comes back as a status.  The arrays passed have
    exactly the sizes declared, and the kernel checks offsets and columns
    before it reads through them, so nothing is accessed out of range."""
    import torch
    dev = torch.device("cuda")
    V = 4
    vals = torch.empty(V, dtype=torch.int64, device=dev)
    pars = torch.empty(V, dtype=torch.int64, device=dev)

    def t(a, dt):
        return torch.tensor(a, dtype=dt, device=dev)

    # 0 -> 1 -> 2 -> column 7, which is >= V
    row = t([0, 1, 2, 3, 3], torch.int64)
    col = t([1, 2, 7], torch.int32)
    assert static_call("bfs", V, 3, row, col, None, vals, pars) == 2
    assert b"column" in rg.lib().rg_last_error()
    # vertex 1's offsets decrease (2 > 1)
    row = t([0, 2, 1, 3, 3], torch.int64)
    col = t([1, 2, 3], torch.int32)
    assert static_call("bfs", V, 3, row, col, None, vals, pars) == 1
    # SSSP and SSWP without weights
    row = t([0, 1, 2, 3, 3], torch.int64)
    for algo in ("sssp", "sswp"):
        assert static_call(algo, V, 3, row, col, None, vals, pars) == 1
        assert b"weights" in rg.lib().rg_last_error()
    # the same well-formed graph still builds afterwards
    assert static_call("bfs", V, 3, row, col, None, vals, pars) == 0
    torch.cuda.synchronize()
    assert vals.cpu().tolist() == [0, 1, 2, 3]


def test_static_rejects_graphs_over_the_limit():
    rc = rg.lib().rg_build_tree_csr_static(rg.ALGOS["bfs"], 0, MAX_V + 1, 0, ctypes.c_void_p(8), ctypes.c_void_p(8),
                                           None, ctypes.c_void_p(8), None, None)
    assert rc == 1
    assert b"RG_STATIC_MAX_VERTICES" in rg.lib().rg_last_error()
