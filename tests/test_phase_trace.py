"""Phase trace of the fused update path (RG_OPT_PHASE_TRACE, rg_phase_trace):
device-clock stamps at the phase boundaries of the fused kernels.  The
reference has no counterpart; it times its phases with wall clocks
(src/sssp_inc.cpp prints read/exec times)."""
import numpy as np
import pytest

import risgraph_b200 as rg
from risgraph_b200 import gen

from helpers import gpu_graph, oracle_graph


@pytest.mark.gpu
def test_phase_trace_reports_both_batches_and_keeps_values():
    scale = 12
    pairs = gen.rmat(scale, seed=5)
    V = 1 << scale
    imported = int(len(pairs) * 0.9)
    root = gen.max_out_degree_vertex(pairs, V)
    g = gpu_graph("sssp", V, pairs[:imported], hint=len(pairs), inc_mode=True)
    g.build_tree("sssp", root)
    assert g.get_option("phase_trace") == 0
    g.set_option("phase_trace", 1)
    e = gen.edges_with_weights(pairs, True)
    lo = imported
    for b in (1, 64, 1500):
        g.apply_add_del("sssp", e[lo:lo + b], e[lo - imported:lo - imported + b])
        t = g.phase_times()
        assert set(t) <= {"insert", "delete"} and "insert" in t, t
        for name, d in t.items():
            # batches of at most RG_OPT_INLINE_MAX (16) edges come in the
            # launch parameters: nothing is staged across the bus
            assert (d["staging"] > 0 if b > 16 else d["staging"] == 0) and d["total"] > 0, (name, d)
            assert all(v >= 0 for v in d.values()), (name, d)
            assert d["total"] <= sum(v for k, v in d.items() if k not in ("total", "staging")) + 1e-3
            assert {"lookup", "count", "seed"} <= set(d), (name, d)
        lo += b
    # one batch alone reports no delete batch
    g.apply_add("sssp", e[lo:lo + 8])
    lo += 8
    assert set(g.phase_times()) == {"insert"}
    g.set_option("phase_trace", 0)
    assert g.get_option("phase_trace") == 0
    # tracing changes no value: the window lost its first 1565 edges and gained the next 1573
    og = oracle_graph("sssp", V, np.concatenate([pairs[1 + 64 + 1500:imported], pairs[imported:lo]]))
    og.build_tree(root)
    np.testing.assert_array_equal(g.values(), og.labels()[0])
    g.close()


@pytest.mark.gpu
def test_level_stamps_cover_graph_launched_builds():
    """rg_level_stamps: the level loop stamps each level's start on the device
    clock, graph-launched builds included; one stamp per traced level plus the
    end of the last, in order."""
    scale = 14
    pairs = gen.rmat(scale, seed=7)
    V = 1 << scale
    root = gen.max_out_degree_vertex(pairs, V)
    for algo in ("bfs", "sssp"):
        g = gpu_graph(algo, V, pairs)
        g.build_tree(algo, root)
        sizes, _ = g.level_trace()
        ms = g.level_device_times()
        assert len(ms) == len(sizes) > 2
        assert (ms >= 0).all() and ms.sum() > 0
        g.close()
