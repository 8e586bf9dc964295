"""Synthetic inputs in the reference's binary edge-list format (core/io.hpp:26-36).

Thin numpy wrappers over the rg_gen_* entry points of librisgraph_b200.so
(include/rg_gen.h).  Host-only code: no GPU needed.
"""
from __future__ import annotations

import ctypes

import numpy as np

RMAT_ABC = (0.57, 0.19, 0.19)


def _lib():
    from . import lib
    return lib()


def _p(a):
    return ctypes.c_void_p(a.ctypes.data)


def rmat(scale: int, n_edges: int | None = None, seed: int = 1, abc=RMAT_ABC, first: int = 0) -> np.ndarray:
    """(n,2) uint64 RMAT edges (duplicates and self-loops kept), seeded order."""
    n = (16 << scale) if n_edges is None else int(n_edges)
    out = np.empty((n, 2), np.uint64)
    _lib().rg_gen_rmat(scale, first, n, abc[0], abc[1], abc[2], seed, _p(out))
    return out


def er_rmat_mix(scale: int, n_edges: int, seed: int = 1, abc=RMAT_ABC, first: int = 0) -> np.ndarray:
    """Half uniform-random endpoints (even indices), half RMAT (odd indices)."""
    out = np.empty((int(n_edges), 2), np.uint64)
    _lib().rg_gen_er_rmat_mix(scale, first, int(n_edges), abc[0], abc[1], abc[2], seed, _p(out))
    return out


def weights(pairs: np.ndarray) -> np.ndarray:
    """splitmix64(src<<32|dst) % 255 + 1 per edge."""
    p = np.ascontiguousarray(pairs, dtype=np.uint64)
    out = np.empty(p.size // 2, np.uint64)
    _lib().rg_gen_weights(_p(p), p.size // 2, _p(out))
    return out


def max_out_degree_vertex(pairs: np.ndarray, vertices: int) -> int:
    p = np.ascontiguousarray(pairs, dtype=np.uint64)
    return int(_lib().rg_gen_max_out_degree_vertex(_p(p), p.size // 2, vertices))


def write_binary(path: str, pairs: np.ndarray) -> None:
    p = np.ascontiguousarray(pairs, dtype=np.uint64)
    rc = _lib().rg_gen_write_binary(path.encode(), _p(p), p.size // 2)
    if rc != 0:
        raise OSError(f"writing {path} failed ({rc})")


def read_binary(path: str) -> np.ndarray:
    """mmap_binary (core/io.hpp:26-36): (n,2) uint64 view of the file."""
    return np.memmap(path, dtype=np.uint64, mode="r").reshape(-1, 2)


def checksum(values: np.ndarray) -> int:
    v = np.ascontiguousarray(values, dtype=np.uint64)
    return int(_lib().rg_gen_value_checksum(_p(v), v.size))


def edges_with_weights(pairs: np.ndarray, weighted: bool) -> np.ndarray:
    """rg_edge array for pairs; weights from weights() when weighted, else 0."""
    from . import EDGE_DTYPE
    p = np.asarray(pairs, dtype=np.uint64).reshape(-1, 2)
    e = np.zeros(len(p), EDGE_DTYPE)
    e["src"] = p[:, 0]
    e["dst"] = p[:, 1]
    if weighted:
        e["data"] = weights(p)
    return e
