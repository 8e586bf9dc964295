"""Versioned label history (the device MVVec): values read back as of any
recorded version equal the values the graph had at that version."""
import numpy as np
import pytest

import risgraph_b200 as rg
from risgraph_b200 import gen

from helpers import WEIGHTED

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("algo", ["sssp", "wcc"])
def test_history_matches_snapshots(algo):
    scale = 12
    pairs = gen.rmat(scale, seed=41)
    V = 1 << scale
    imported = int(len(pairs) * 0.9)
    directed = algo != "wcc"
    g = rg.Graph(V, len(pairs), symmetric=not directed, dual=directed, trace_modified=True, weighted=WEIGHTED[algo])
    g.add_pairs(pairs[:imported], directed, want_old=False)
    g.build_tree(algo, 0)
    g.history_enable(V + 200000)
    g.history_record(0, all_vertices=True)
    snaps = [g.values()]
    steps = 60
    for k in range(1, steps + 1):
        lo = imported + (k - 1) * 20
        g.apply_add_pairs(algo, pairs[lo:lo + 20], directed)
        g.apply_del_pairs(algo, pairs[lo - imported:lo - imported + 20], directed)
        g.history_record(k)
        snaps.append(g.values())
    rng = np.random.default_rng(1)
    for version in (0, 1, 17, 30, steps):
        vids = rng.choice(V, 500, replace=False).astype(np.uint64)
        vals, found = g.history_get(vids, version)
        assert found.all()
        np.testing.assert_array_equal(vals, snaps[version][vids])
    used_before, cap = g.history_nodes()
    assert V <= used_before <= cap
    g.history_gc(30)
    used_after, _ = g.history_nodes()
    assert used_after <= used_before
    vids = np.arange(V, dtype=np.uint64)
    for version in (30, 45, steps):
        vals, found = g.history_get(vids, version)
        assert found.all()
        np.testing.assert_array_equal(vals, snaps[version])
    g.close()


def test_history_needs_trace_and_reports_full_pool():
    V = 1 << 10
    pairs = gen.rmat(10, seed=2)
    g = rg.Graph(V, len(pairs), weighted=True)
    g.add_pairs(pairs, True, want_old=False)
    g.build_tree("sssp", 0)
    with pytest.raises(rg.RGError) as e:
        g.history_enable(100)
    assert e.value.status == 8  # RG_ESTATE: no trace_modified
    g.close()
    g = rg.Graph(V, len(pairs), trace_modified=True, weighted=True)
    g.add_pairs(pairs, True, want_old=False)
    g.build_tree("sssp", 0)
    g.history_enable(100)
    with pytest.raises(rg.RGError) as e:
        g.history_record(0, all_vertices=True)
    assert e.value.status == 5  # RG_ENOSPACE
    assert g.history_nodes() == (100, 100)
    g.close()


def test_served_epochs_record_history():
    """A served instance with history on: after the load, version k holds the
    values after k epochs, and the last version equals the current values."""
    scale = 11
    pairs = gen.rmat(scale, seed=43)
    V = 1 << scale
    imported = int(len(pairs) * 0.9)
    g = rg.Graph(V, len(pairs), trace_modified=True, weighted=True)
    g.add_pairs(pairs[:imported], True, want_old=False)
    g.build_tree("sssp", 0)
    g.history_enable(4 * V + 100000)
    g.history_record(0, all_vertices=True)
    before = g.values()
    with rg.Server(max_epoch=256) as srv:
        k = srv.attach(g)
        srv.history(k, True)
        srv.run_load([dict(instance=k, clients=8, pairs=pairs, imported=imported, max_updates=800,
                           duration_s=30.0, think_us=20.0, weighted=True, seed=3)])
        last = srv.history(k, True)
        srv.detach(k)
    assert last >= 1
    vids = np.arange(V, dtype=np.uint64)
    vals, found = g.history_get(vids, last)
    assert found.all()
    np.testing.assert_array_equal(vals, g.values())
    vals0, _ = g.history_get(vids, 0)
    np.testing.assert_array_equal(vals0, before)
    g.close()
