"""Paths that ordinary inputs rarely reach: the deletion repair's full-
recompute fallback, the level bound of the device loop, the served drain's
timeout, and the label history replayed through the reference's own MVVec.
Every failure here is made on the host or by a bound the test lowers; nothing
faults, traps or hangs the GPU."""
import os
import subprocess
import tempfile

import numpy as np
import pytest

import risgraph_b200 as rg
from risgraph_b200 import gen

from helpers import WEIGHTED, gpu_graph, oracle_graph

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
MVVEC = os.path.join(os.path.dirname(HERE), "oracle", "_ref", "mvvec_driver")


@pytest.mark.parametrize("algo", ["bfs", "sssp", "wcc"])
def test_deletion_repair_falls_back_to_a_full_build(algo):
    """Deleting every copy of every edge out of the root (the hub, vertex 0;
    for WCC every edge touching it) cuts the whole tree off: no vertex can be
    rescued, the invalidated set passes the threshold of core/graph.hpp:1252
    (max(recompute_min, |V|/20)), and the repair rebuilds from scratch.  The
    values still equal the reference's (the oracle repairs the same batch)."""
    scale = 14
    pairs = gen.rmat(scale, seed=61)
    V = 1 << scale
    directed = algo != "wcc"
    g = gpu_graph(algo, V, pairs, inc_mode=True)
    og = oracle_graph(algo, V, pairs, inc_mode=True)
    root = 0
    g.set_option("recompute_min", 1)
    g.build_tree(algo, root)
    og.build_tree(root)
    sel = pairs[:, 0] == root if directed else (pairs[:, 0] == root) | (pairs[:, 1] == root)
    dels = gen.edges_with_weights(pairs[sel], WEIGHTED[algo])
    old = g.apply_del(algo, dels, directed)
    st = g.last_stats()
    assert st["recomputes"] > 0, st
    og_old = np.array([og.del_edge(int(e["src"]), int(e["dst"]), int(e["data"])) for e in dels], np.uint64)
    # copies of one edge in one batch may take their old counts in another order:
    # compare the edges whose last copy went, not the positions (an undirected
    # edge named either way round is one edge)
    def key(d, o):
        s, t = d["src"][o == 1], d["dst"][o == 1]
        if not directed:
            s, t = np.minimum(s, t), np.maximum(s, t)
        return sorted(set(zip(s.tolist(), t.tolist())))
    assert key(dels, old) == key(dels, og_old)
    gone = dels[og_old == 1]
    og.update_tree_del_batch(gone["src"], gone["dst"], gone["data"], root)
    val, par, pw = g.labels()
    np.testing.assert_array_equal(val, og.labels()[0])
    assert og.validate(val, par, pw, root) == 0
    g.close()


@pytest.mark.parametrize("algo", ["sssp", "wcc"])
def test_level_bound_stops_the_loop_and_the_graph_stays_usable(algo):
    """With RG_OPT_MAX_LEVELS lowered to 2 the device loop stops at its bound
    (k_loop_cond) and the call returns RG_ETIMEOUT; the error is cleared, and
    with the default bound back the next build and an update give the
    reference's values."""
    scale = 12
    pairs = gen.rmat(scale, seed=62)
    V = 1 << scale
    imported = int(len(pairs) * 0.9)
    directed = algo != "wcc"
    g = gpu_graph(algo, V, pairs[:imported], hint=len(pairs))
    og = oracle_graph(algo, V, pairs[:imported])
    g.set_option("max_levels", 2)
    assert g.get_option("max_levels") == 2
    with pytest.raises(rg.RGError) as e:
        g.build_tree(algo, 0)
    assert e.value.status == 6  # RG_ETIMEOUT
    g.set_option("max_levels", 0)
    g.build_tree(algo, 0)
    og.build_tree(0)
    np.testing.assert_array_equal(g.values(), og.labels()[0])
    g.apply_add_pairs(algo, pairs[imported:imported + 100], directed)
    ref = oracle_graph(algo, V, pairs[:imported + 100])
    ref.build_tree(0)
    np.testing.assert_array_equal(g.values(), ref.labels()[0])
    g.close()


def test_server_drain_times_out_and_recovers():
    """rg_server_drain with a zero timeout while 50,000 submitted updates are
    still queued returns RG_ETIMEOUT; a drain with room then returns RG_OK and
    every update completes."""
    scale = 14
    pairs = gen.rmat(scale, seed=63)
    V = 1 << scale
    imported = int(len(pairs) * 0.9)
    g = gpu_graph("sssp", V, pairs[:imported], hint=len(pairs), inc_mode=True)
    g.build_tree("sssp", 0)
    n = 50000
    reqs = np.zeros(n, rg.REQUEST_DTYPE)
    adds = gen.edges_with_weights(pairs[imported:imported + n // 2], True)
    dels = gen.edges_with_weights(pairs[:n // 2], True)
    with rg.Server(per_update=True, max_epoch=4096) as srv:
        k = srv.attach(g)
        reqs["instance"] = k
        reqs["type"][0::2], reqs["type"][1::2] = 0, 1
        for f in ("src", "dst", "data"):
            reqs[f][0::2], reqs[f][1::2] = adds[f], dels[f]
        reqs["tag"] = np.arange(n)
        srv.submit(reqs)
        assert rg.lib().rg_server_drain(srv._h, 0) == 6   # RG_ETIMEOUT: the per-update path is still busy
        srv.drain(120000)
        got = srv.poll(1 << 17)
        srv.detach(k)
    assert len(got) == n and (got["status"] == 0).all()
    ref = oracle_graph("sssp", V, np.concatenate([pairs[n // 2:imported], pairs[imported:imported + n // 2]]))
    ref.build_tree(0)
    np.testing.assert_array_equal(g.values(), ref.labels()[0])
    g.close()


def mvvec_replay(length, ops):
    """Run ops [(op, a, b, c)] through the reference's MVVec; returns the gets."""
    with tempfile.TemporaryDirectory() as d:
        p = os.path.join(d, "ops.bin")
        np.asarray(ops, np.uint64).reshape(-1, 4).tofile(p)
        subprocess.run([MVVEC, str(length), p, p + ".out"], check=True, capture_output=True)
        return np.fromfile(p + ".out", np.uint64)


@pytest.mark.parametrize("algo", ["sssp", "bfs"])
def test_history_matches_reference_mvvec(algo):
    """The device history against the reference's MVVec (core/mvvec.hpp:23-162):
    the same set calls (every modified vertex's value at each version, as
    src/sssp_inc_rt.cpp:338-343 records them, including a version recorded
    twice, which overwrites) give the same get results at every version.
    After rg_history_gc(T), every read at a version >= T still equals the
    reference's read before any gc.  (The reference's own gc drops the node a
    reader at T sees when a newer one exists, and its drivers never call it, so
    post-gc reads are compared with the reference's pre-gc reads.)"""
    assert os.path.exists(MVVEC), "oracle/_ref/mvvec_driver is missing: build it with oracle/ref/build_ref.sh"
    scale = 11
    pairs = gen.rmat(scale, seed=64)
    V = 1 << scale
    imported = int(len(pairs) * 0.9)
    g = rg.Graph(V, len(pairs), trace_modified=True, weighted=WEIGHTED[algo])
    g.add_pairs(pairs[:imported], True, want_old=False)
    g.build_tree(algo, 0)
    g.history_enable(V * 8 + 100000)
    g.clear_modified()
    g.history_record(0, all_vertices=True)
    ops = [(0, v, 0, x) for v, x in enumerate(g.values().tolist())]
    steps, lo = 40, imported
    version = 0
    for k in range(steps):
        g.apply_add_pairs(algo, pairs[lo:lo + 8])
        g.apply_del_pairs(algo, pairs[lo - imported:lo - imported + 8])
        lo += 8
        if k != 20:          # step 20 records at the same version as step 19: an overwrite
            version += 1
        mod = g.get_modified()
        vals = g.values()
        ops += [(0, int(v), version, int(vals[v])) for v in mod]
        g.history_record(version)
    last = version
    rng = np.random.default_rng(5)
    vids = rng.choice(V, 300, replace=False)
    queries = [(v, t) for t in range(last + 1) for v in vids.tolist()]
    ref = mvvec_replay(V, ops + [(1, v, t, 0) for v, t in queries])
    ours = np.concatenate([g.history_get(vids.astype(np.uint64), t)[0] for t in range(last + 1)])
    np.testing.assert_array_equal(ours, ref)
    T = last // 2
    used_before, _ = g.history_nodes()
    g.history_gc(T)
    used_after, _ = g.history_nodes()
    assert used_after < used_before
    after = np.concatenate([g.history_get(vids.astype(np.uint64), t)[0] for t in range(T, last + 1)])
    np.testing.assert_array_equal(after, ref[T * len(vids):])
    g.close()


@pytest.mark.parametrize("algo", ["bfs", "sssp", "sswp", "wcc"])
def test_deletion_repair_splits_heavy_vertices(algo):
    """The parent edges of the eight heaviest vertices (in-lists of thousands of
    entries) are deleted, every copy of each: the one-CTA repair hands the
    hubs to the grid-wide repair, whose rescue, expansion and pull spread each
    hub's list over all warps.  Values equal the oracle's after the same batch."""
    scale = 16
    pairs = gen.rmat(scale, seed=91)
    V = 1 << scale
    directed = algo != "wcc"
    g = gpu_graph(algo, V, pairs, inc_mode=True)
    og = oracle_graph(algo, V, pairs, inc_mode=True)
    root = gen.max_out_degree_vertex(pairs, V)
    g.build_tree(algo, root)
    og.build_tree(root)
    val, par, pw = g.labels()
    _, indeg = g.degrees()
    order = np.argsort(-indeg.astype(np.int64))
    hubs = [int(v) for v in order[:64] if par[v] != V and v != root][:8]
    assert len(hubs) == 8 and indeg[hubs[0]] > 2048   # above the split threshold (HEAVY_DEG)
    one = np.zeros(len(hubs), rg.EDGE_DTYPE)
    one["src"], one["dst"] = par[hubs], hubs
    if WEIGHTED[algo]:
        one["data"] = pw[hubs]
    counts = g.get_edge_num(one)
    if not directed:   # an undirected edge is stored once per orientation: one delete removes a copy of both
        counts = np.maximum(counts, 1)
    dels = np.repeat(one, counts.astype(np.int64))
    g.apply_del(algo, dels, directed)
    og_old = np.array([og.del_edge(int(e["src"]), int(e["dst"]), int(e["data"])) for e in dels], np.uint64)
    gone = dels[og_old == 1]
    og.update_tree_del_batch(gone["src"], gone["dst"], gone["data"], root)
    val, par, pw = g.labels()
    np.testing.assert_array_equal(val, og.labels()[0])
    assert og.validate(val, par, pw, root) == 0
    g.close()
