"""Shared helpers for the parity tests: the same seeded inputs drive the CUDA
path (through the C ABI) and the CPU oracle."""
import numpy as np

from oracle import oracle as O
from risgraph_b200 import gen

WEIGHTED = {"bfs": False, "sssp": True, "sswp": True, "wcc": False}
ALGOS = ["bfs", "sssp", "sswp", "wcc"]


def rmat_pairs(scale, seed=1, n_edges=None):
    return gen.rmat(scale, n_edges, seed=seed)


def gpu_graph(algo, V, pairs, hint=None, inc_mode=False, trace=False):
    """Graph with pairs loaded the way the reference drivers load them."""
    import risgraph_b200 as rg
    sym = algo == "wcc"
    dual = not (algo == "wcc" and inc_mode)
    g = rg.Graph(V, hint or max(len(pairs), 1024), symmetric=sym, dual=dual, trace_modified=trace,
                 weighted=WEIGHTED[algo])
    if len(pairs):
        g.add_pairs(pairs, directed=(algo != "wcc"), want_old=False)
    return g


def oracle_graph(algo, V, pairs, inc_mode=False):
    og = O.OracleGraph(algo, V, max(len(pairs), 1), inc_mode=inc_mode)
    if len(pairs):
        og.load(pairs)
    return og


def edges_of(algo, pairs):
    return gen.edges_with_weights(pairs, WEIGHTED[algo])
