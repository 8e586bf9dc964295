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
