"""Every path of the fused insert+delete submission (rg_apply_add_del) against
the oracle's batch loop (the _inc_batch step, src/sssp_inc_batch.cpp:141-175):
the insert batch's repair finishing in the kernel or leaving a level loop
behind it (then the delete batch runs as its own phase), and the delete
batch's repair finishing in place, leaving push levels, or handing over to the
grid-wide repair.  RG_OPT_TINY_EDGES = 0 turns off the in-place push levels,
so every non-empty frontier takes the graph's level loop."""
import numpy as np
import pytest

from risgraph_b200 import gen

from helpers import ALGOS, edges_of, gpu_graph, oracle_graph


@pytest.mark.gpu
@pytest.mark.parametrize("algo", ALGOS)
@pytest.mark.parametrize("batch", [1, 300, 1500])
@pytest.mark.parametrize("tiny", [0, None])
def test_mixed_submissions_match_oracle(algo, batch, tiny):
    scale = 13
    pairs = gen.rmat(scale, seed=33)
    V = 1 << scale
    imported = int(len(pairs) * 0.8)
    nb = 40 if batch == 1 else 8
    g = gpu_graph(algo, V, pairs[:imported], hint=len(pairs), inc_mode=True)
    og = oracle_graph(algo, V, pairs[:imported], inc_mode=True)
    root = 0 if algo == "wcc" else gen.max_out_degree_vertex(pairs[:imported], V)
    g.build_tree(algo, root)
    og.build_tree(root)
    if tiny is not None:
        g.set_option("tiny_edges", tiny)
    ref = og.run_batch(pairs, imported, batch, nb, root)
    e = edges_of(algo, pairs)
    directed = algo != "wcc"
    for k in range(nb):
        lo = imported + k * batch
        g.apply_add_del(algo, e[lo:lo + batch], e[lo - imported:lo - imported + batch], directed)
        assert g.checksum() == int(ref[k]), f"batch {k}"
    val, par, pw = g.labels()
    assert og.validate(val, par, pw, root) == 0
    np.testing.assert_array_equal(val, og.labels()[0])
    g.close()


@pytest.mark.gpu
@pytest.mark.parametrize("algo", ALGOS)
@pytest.mark.parametrize("batch", [1, 7, 16])
def test_inline_batches_match_staged_and_oracle(algo, batch):
    """Batches of at most RG_OPT_INLINE_MAX edges travel in the fused kernel's
    launch parameters.  Two graphs in lockstep, one with the inline path and
    one with it off (staged through mapped memory), take the same single-batch
    inserts and deletes (rg_apply_add / rg_apply_del, old counts returned) and
    insert+delete submissions; both match the oracle's batch loop after every
    step, and their old counts agree."""
    scale = 13
    pairs = gen.rmat(scale, seed=41)
    V = 1 << scale
    imported = int(len(pairs) * 0.8)
    nb = 30
    root = 0 if algo == "wcc" else gen.max_out_degree_vertex(pairs[:imported], V)
    og = oracle_graph(algo, V, pairs[:imported], inc_mode=True)
    og.build_tree(root)
    ref = og.run_batch(pairs, imported, batch, nb, root)
    graphs = []
    for inline in (None, 0):
        g = gpu_graph(algo, V, pairs[:imported], hint=len(pairs), inc_mode=True)
        if inline is not None:
            g.set_option("inline_max", inline)
        g.build_tree(algo, root)
        graphs.append(g)
    assert graphs[0].get_option("inline_max") == 16 and graphs[1].get_option("inline_max") == 0
    e = edges_of(algo, pairs)
    directed = algo != "wcc"
    for k in range(nb):
        lo = imported + k * batch
        adds, dels = e[lo:lo + batch], e[lo - imported:lo - imported + batch]
        olds = []
        for g in graphs:
            if k % 2 == 0:   # one submission for both batches
                g.apply_add_del(algo, adds, dels, directed)
            else:            # one submission each, with the old counts back
                olds.append((g.apply_add(algo, adds, directed), g.apply_del(algo, dels, directed)))
            assert g.checksum() == int(ref[k]), f"batch {k}"
        if olds:
            for a, b in zip(olds[0], olds[1]):
                np.testing.assert_array_equal(a, b)
    for g in graphs:
        val, par, pw = g.labels()
        assert og.validate(val, par, pw, root) == 0
        np.testing.assert_array_equal(val, og.labels()[0])
        g.close()
