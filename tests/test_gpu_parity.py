"""CUDA path vs the oracle, through the C ABI: values bit-exact, parents checked
structurally (they are race-dependent in the reference too)."""
import json
import os

import numpy as np
import pytest

import risgraph_b200 as rg
from risgraph_b200 import gen

from helpers import ALGOS, WEIGHTED, edges_of, gpu_graph, oracle_graph
from oracle import oracle as O

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def check_tree(g, og, root=0):
    val, par, pw = g.labels()
    r = og.validate(val, par, pw, root)
    assert r == 0, f"invalid dependency tree at vertex/kind {r}"
    return val


# ---------------------------------------------------------------- full build
@pytest.mark.parametrize("algo", ALGOS)
@pytest.mark.parametrize("scale", [10, 14])
def test_build_tree_parity(algo, scale):
    pairs = gen.rmat(scale, seed=11)
    V = 1 << scale
    root = gen.max_out_degree_vertex(pairs, V)
    g = gpu_graph(algo, V, pairs)
    og = oracle_graph(algo, V, pairs)
    g.build_tree(algo, root)
    og.build_tree(root)
    val = check_tree(g, og, root)
    np.testing.assert_array_equal(val, og.labels()[0])
    # idempotent: a second build gives the same values
    g.build_tree(algo, root)
    np.testing.assert_array_equal(g.values(), val)


@pytest.mark.parametrize("algo", ALGOS)
@pytest.mark.parametrize("split,groups", [(0, 2), (1, 2), (1, 3), (1, 6)])
def test_build_tree_parity_pull_levels(algo, split, groups):
    """Every large level pulls over the sliced in-edge copy, BFS included (no
    bottom-up levels), in one launch or split (hub slices first, then the
    other rows in groups - 1 launches)."""
    scale = 14
    V = 1 << scale
    pairs = gen.er_rmat_mix(scale, 32 * V, seed=29)
    root = gen.max_out_degree_vertex(pairs, V)
    g = gpu_graph(algo, V, pairs)
    g.set_option("dense_pull", 1)
    g.set_option("bfs_bottom_up", 0)
    g.set_option("pull_split", split)
    g.set_option("pull_groups", groups)
    og = oracle_graph(algo, V, pairs)
    og.build_tree(root)
    g.build_tree(algo, root)
    np.testing.assert_array_equal(check_tree(g, og, root), og.labels()[0])


def test_build_tree_parity_values_beyond_16_bits():
    """Large SSSP distances through pull levels: a 700-hop chain from the root
    ends in a vertex with 4,000 out-edges into a random graph, so the large
    frontiers that pull hold values past 65,535."""
    V = 1 << 14
    rng = np.random.default_rng(31)
    chain = np.stack([np.arange(0, 699), np.arange(1, 700)], axis=1)
    fan = np.stack([np.full(4000, 699), rng.integers(700, V, 4000)], axis=1)
    rest = rng.integers(700, V, size=(16 * V, 2))
    pairs = np.concatenate([chain, fan, rest]).astype(np.uint64)
    g = gpu_graph("sssp", V, pairs)
    og = oracle_graph("sssp", V, pairs)
    og.build_tree(0)
    g.build_tree("sssp", 0)
    val = check_tree(g, og, 0)
    np.testing.assert_array_equal(val, og.labels()[0])
    reached = val[val < (1 << 27)]
    assert reached.max() > 65535 and np.median(reached) > 65535


PUSH_MODES = {
    # every level of the build in one push mode
    "edge_balanced": {"lbs_min": 1, "dense_div": 1},
    "dense": {"dense_div": 1 << 30},
    "sparse": {"lbs_min": 1 << 40, "dense_div": 1},
    # successive levels in one thread-block cluster (the graph's frontiers all fit)
    "cluster": {"cluster_edges": 1 << 20},
}


@pytest.mark.parametrize("algo", ALGOS)
@pytest.mark.parametrize("mode", sorted(PUSH_MODES))
def test_build_tree_parity_push_modes(algo, mode):
    """Builds pushed level by level in one mode: the edge-balanced and dense
    modes commit each level through per-vertex packed keys, the sparse and
    cluster modes through the 16-byte CAS; values equal the oracle's, trees
    are valid, and an incremental batch on top still matches."""
    scale = 13
    V = 1 << scale
    pairs = gen.er_rmat_mix(scale, 24 * V, seed=17)
    root = gen.max_out_degree_vertex(pairs, V)
    g = gpu_graph(algo, V, pairs)
    for k, v in {"dense_pull": 0, "bfs_bottom_up": 0, "tiny_edges": 0, "cluster_edges": 0, **PUSH_MODES[mode]}.items():
        g.set_option(k, v)
    og = oracle_graph(algo, V, pairs)
    og.build_tree(root)
    g.build_tree(algo, root)
    val = check_tree(g, og, root)
    np.testing.assert_array_equal(val, og.labels()[0])
    extra = gen.rmat(scale, 2000, seed=23)
    g.apply_add_pairs(algo, extra, directed=(algo != "wcc"))
    og2 = oracle_graph(algo, V, np.concatenate([pairs, extra]))
    og2.build_tree(root)
    np.testing.assert_array_equal(check_tree(g, og2, root), og2.labels()[0])


@pytest.mark.parametrize("algo", ALGOS)
def test_build_tree_parity_er_rmat_mix(algo):
    """Half uniform, half RMAT endpoints: nearly every vertex has in-edges and
    the RMAT hubs are cut into several pull pieces, so the sliced in-edge copy
    has more rows than vertices."""
    scale = 14
    V = 1 << scale
    pairs = gen.er_rmat_mix(scale, 64 * V, seed=5)
    root = gen.max_out_degree_vertex(pairs, V)
    g = gpu_graph(algo, V, pairs)
    og = oracle_graph(algo, V, pairs)
    g.build_tree(algo, root)
    og.build_tree(root)
    val = check_tree(g, og, root)
    np.testing.assert_array_equal(val, og.labels()[0])


@pytest.mark.parametrize("name", [n for n in json.load(open(os.path.join(GOLDEN, "index.json")))])
def test_golden_reference_fixtures(name):
    """Against values and per-step checksums produced by the reference itself."""
    z = np.load(os.path.join(GOLDEN, name + ".npz"))
    m = json.loads(str(z["meta"]))
    pairs = gen.rmat(m["scale"], seed=m["seed"])
    algo, V, root = m["algo"], m["V"], m["root"]
    directed = algo != "wcc"
    if m["mode"] == "build":
        g = gpu_graph(algo, V, pairs)
        g.build_tree(algo, root)
    else:
        imported = int(len(pairs) * m["rate"])
        g = gpu_graph(algo, V, pairs[:imported], hint=len(pairs), inc_mode=True)
        g.build_tree(algo, root)
        sums = []
        if m["mode"] == "inc":
            for i in range(imported, imported + m["steps"]):
                g.apply_add_pairs(algo, pairs[i:i + 1], directed)
                g.apply_del_pairs(algo, pairs[i - imported:i - imported + 1], directed)
                sums.append(g.checksum())
        else:
            b = m["batch"]
            for k in range(m["nbatches"]):
                lo = imported + k * b
                if lo >= len(pairs):
                    break
                hi = min(lo + b, len(pairs))
                g.apply_add_pairs(algo, pairs[lo:hi], directed)
                g.apply_del_pairs(algo, pairs[lo - imported:hi - imported], directed)
                sums.append(g.checksum())
        np.testing.assert_array_equal(np.array(sums, np.uint64), z["sums"])
    np.testing.assert_array_equal(g.values(), z["val"])


# ------------------------------------------------------- incremental, single
@pytest.mark.parametrize("algo", ALGOS)
def test_inc_single_updates_vs_oracle(algo):
    """bfs_inc-style sliding window: insert raw[i], delete raw[i-imported], each
    repaired immediately; value checksum compared after every step."""
    scale, steps = 14, 1500
    pairs = gen.rmat(scale, seed=5)
    V = 1 << scale
    imported = int(len(pairs) * 0.9)
    g = gpu_graph(algo, V, pairs[:imported], hint=len(pairs), inc_mode=True)
    og = oracle_graph(algo, V, pairs[:imported], inc_mode=True)
    g.build_tree(algo, 0)
    og.build_tree(0)
    ref = og.run_inc(pairs, imported, steps, 0)
    directed = algo != "wcc"
    for k in range(steps):
        i = imported + k
        g.apply_add_pairs(algo, pairs[i:i + 1], directed)
        g.apply_del_pairs(algo, pairs[k:k + 1], directed)
        assert g.checksum() == int(ref[k]), f"step {k}"
    val = check_tree(g, og)
    np.testing.assert_array_equal(val, og.labels()[0])


def test_bfs_inc_rmat16_10k_steps():
    """Plain incremental BFS at its headline size: RMAT-16 (65,536 vertices,
    1,048,576 edges), the first 90% loaded, root 0, then 10,000 sliding-window
    steps (insert raw[i], delete raw[i - imported]), each repaired at once;
    the depth of every vertex is compared after every step through the
    value checksum: against the reference-built driver (required: a GPU run
    without oracle/_ref/ref_driver fails here rather than falling back) and
    against the oracle port."""
    scale, steps = 16, 10000
    pairs = gen.rmat(scale, seed=16)
    V = 1 << scale
    imported = int(len(pairs) * 0.9)
    g = gpu_graph("bfs", V, pairs[:imported], hint=len(pairs), inc_mode=True)
    og = oracle_graph("bfs", V, pairs[:imported], inc_mode=True)
    g.build_tree("bfs", 0)
    og.build_tree(0)
    ref = og.run_inc(pairs, imported, steps, 0)
    assert len(ref) == steps
    from oracle import oracle as O
    assert O.ref_available(), "oracle/_ref/ref_driver is missing: build it with oracle/ref/build_ref.sh"
    _, arrays = O.ref_run("inc", "bfs", pairs, V, 0, 0.9, steps)
    np.testing.assert_array_equal(arrays["sums"][:steps], ref)
    sums = np.zeros(steps, np.uint64)
    for k in range(steps):
        i = imported + k
        g.apply_add_pairs("bfs", pairs[i:i + 1], True)
        g.apply_del_pairs("bfs", pairs[k:k + 1], True)
        sums[k] = g.checksum()
    np.testing.assert_array_equal(sums, ref)
    val = check_tree(g, og)
    np.testing.assert_array_equal(val, og.labels()[0])


@pytest.mark.parametrize("algo", ALGOS)
def test_reference_api_sequence(algo):
    """The driver sequence with host decisions (src/sssp_inc.cpp:295-324):
    add_edge -> if old==0 update_tree_add; del_edge -> if old==1 update_tree_del."""
    scale, steps = 12, 300
    pairs = gen.rmat(scale, seed=9)
    V = 1 << scale
    imported = int(len(pairs) * 0.9)
    g = gpu_graph(algo, V, pairs[:imported], hint=len(pairs), inc_mode=True)
    og = oracle_graph(algo, V, pairs[:imported], inc_mode=True)
    g.build_tree(algo, 0)
    og.build_tree(0)
    ref = og.run_inc(pairs, imported, steps, 0)
    directed = algo != "wcc"
    e_all = edges_of(algo, pairs)
    for k in range(steps):
        e = e_all[imported + k:imported + k + 1]
        if g.add_edges(e, directed)[0] == 0:
            g.update_tree_add(algo, e, directed)
        e = e_all[k:k + 1]
        if g.del_edges(e, directed)[0] == 1:
            g.update_tree_del(algo, e, directed)
        assert g.checksum() == int(ref[k]), f"step {k}"
    check_tree(g, og)


# -------------------------------------------------------- incremental, batch
@pytest.mark.parametrize("algo", ALGOS)
@pytest.mark.parametrize("batch", [1, 64, 4096])
def test_batches_vs_oracle(algo, batch):
    scale = 14
    pairs = gen.rmat(scale, seed=21)
    V = 1 << scale
    imported = int(len(pairs) * 0.9)
    nb = max(1, min(12, (len(pairs) - imported) // batch))
    g = gpu_graph(algo, V, pairs[:imported], hint=len(pairs), inc_mode=True)
    og = oracle_graph(algo, V, pairs[:imported], inc_mode=True)
    g.build_tree(algo, 0)
    og.build_tree(0)
    ref = og.run_batch(pairs, imported, batch, nb, 0)
    directed = algo != "wcc"
    for k in range(nb):
        lo = imported + k * batch
        hi = min(lo + batch, len(pairs))
        g.apply_add_pairs(algo, pairs[lo:hi], directed)
        g.apply_del_pairs(algo, pairs[lo - imported:hi - imported], directed)
        assert g.checksum() == int(ref[k]), f"batch {k}"
    val = check_tree(g, og)
    np.testing.assert_array_equal(val, og.labels()[0])


# ------------------------------------------------------------ classification
@pytest.mark.parametrize("algo", ALGOS)
def test_classify_matches_tree_semantics(algo):
    """need_update_tree_add is a pure function of values (bit-exact vs oracle);
    need_update_tree_del is checked against the GPU's own parents."""
    scale = 12
    pairs = gen.rmat(scale, seed=4)
    V = 1 << scale
    g = gpu_graph(algo, V, pairs[:50000])
    og = oracle_graph(algo, V, pairs[:50000])
    g.build_tree(algo, 0)
    og.build_tree(0)
    directed = algo != "wcc"
    cand = edges_of(algo, pairs[50000:52000])
    unsafe = g.classify(algo, cand, None, directed)
    exp = np.array([og.need_update_tree_add(int(e["src"]), int(e["dst"]), int(e["data"])) for e in cand])
    np.testing.assert_array_equal(unsafe.astype(bool), exp)
    # deletes: unsafe iff the edge is dst's parent edge (either way if undirected)
    old = edges_of(algo, pairs[:2000])
    unsafe = g.classify(algo, old, np.ones(len(old), np.uint8), directed).astype(bool)
    val, par, pw = g.labels()
    exp = (par[old["dst"].astype(np.int64)] == old["src"]) & (pw[old["dst"].astype(np.int64)] == old["data"])
    if not directed:
        exp |= (par[old["src"].astype(np.int64)] == old["dst"]) & (pw[old["src"].astype(np.int64)] == old["data"])
    np.testing.assert_array_equal(unsafe, exp)


# -------------------------------------------------------------- adjacency
@pytest.mark.parametrize("weighted,symmetric", [(False, False), (True, False), (False, True)])
def test_multiplicity_and_degrees(weighted, symmetric):
    """Old multiplicities, get_edge_num and degrees (IndexedEdgeStorage,
    core/storage.hpp:345-423) with heavy duplication inside one batch.  Inside
    a batch the reference's order is a thread race, so the multiset of old
    counts per (unordered, if undirected) key is compared."""
    V = 512
    rng = np.random.default_rng(3)
    e = np.zeros(3000, rg.EDGE_DTYPE)
    e["src"] = rng.integers(0, 64, 3000)
    e["dst"] = rng.integers(0, 64, 3000)
    e["data"] = rng.integers(1, 4, 3000) if weighted else 0
    algo = "sssp" if weighted else ("wcc" if symmetric else "bfs")
    directed = not symmetric
    g = rg.Graph(V, 4096, symmetric=symmetric, weighted=weighted)
    og = oracle_graph(algo, V, np.zeros((0, 2), np.uint64))

    def key(arr, old):
        s, d = arr["src"].tolist(), arr["dst"].tolist()
        if symmetric:
            s, d = [min(a, b) for a, b in zip(s, d)], [max(a, b) for a, b in zip(s, d)]
        return sorted(zip(s, d, arr["data"].tolist(), old.tolist()))

    old = g.add_edges(e, directed)
    exp = np.array([og.add_edge(int(x["src"]), int(x["dst"]), int(x["data"])) for x in e], np.uint64)
    assert key(e, old) == key(e, exp)
    d = e[:1500]
    old = g.del_edges(d, directed)
    exp = np.array([og.del_edge(int(x["src"]), int(x["dst"]), int(x["data"])) for x in d], np.uint64)
    assert key(d, old) == key(d, exp)
    absent = np.zeros(3, rg.EDGE_DTYPE)
    absent["src"] = [500, 501, 502]
    absent["dst"] = [7, 8, 9]
    assert (g.del_edges(absent, directed) == 0).all()
    q = e[:500]
    num = g.get_edge_num(q)
    exp = np.array([og.get_edge_num(int(x["src"]), int(x["dst"]), int(x["data"])) for x in q])
    np.testing.assert_array_equal(num, exp)
    od, idg = g.degrees()
    np.testing.assert_array_equal(od, [og.out_degree(v) for v in range(V)])
    np.testing.assert_array_equal(idg, [og.in_degree(v) for v in range(V)])


def test_undirected_old_num_conventions():
    """add_edge(e,false) returns the other orientation's old count, minus one
    for a self-loop (core/graph.hpp:206-211); del_edge(e,false) the second
    call's (:232-237)."""
    og = oracle_graph("wcc", 16, np.zeros((0, 2), np.uint64))
    g = rg.Graph(16, 64, symmetric=True)
    seq = [(3, 3), (3, 3), (1, 2), (2, 1), (1, 2), (4, 4)]
    for s, d in seq:
        assert g.add_edge(s, d, directed=False) == og.add_edge(s, d)
    for s, d in seq[::-1] + [(5, 6), (3, 3), (3, 3)]:
        assert g.del_edge(s, d, directed=False) == og.del_edge(s, d)


# --------------------------------------------------------------- edge cases
def test_errors_are_status_codes():
    g = rg.Graph(100, 1000, weighted=True)
    with pytest.raises(rg.RGError) as ei:
        g.add_edge(5, 100, 3)
    assert ei.value.status == 2
    # weights are uint64 as in the reference (core/type.hpp:25) below 2^64 - 2^27,
    # where the reference's u64 sum value + weight would wrap
    assert g.add_edge(5, 6, 1 << 31) == 0
    assert g.add_edge(5, 7, (1 << 64) - (1 << 27) - 1) == 0
    with pytest.raises(rg.RGError) as ei:
        g.add_edge(5, 6, (1 << 64) - (1 << 27))
    assert ei.value.status == 3
    with pytest.raises(rg.RGError) as ei:
        g.update_tree_add("sssp", [(1, 2, 3)])
    assert ei.value.status == 8   # no labels built yet
    with pytest.raises(rg.RGError):
        g.build_tree("sssp", 1000)
    g.build_tree("sssp", 0)
    # empty batches are no-ops
    assert len(g.add_edges(np.zeros(0, rg.EDGE_DTYPE))) == 0
    assert g.update_tree_add("sssp", np.zeros(0, rg.EDGE_DTYPE)) == 0
    assert g.update_tree_del("sssp", np.zeros(0, rg.EDGE_DTYPE)) == 0
    g.apply_add("sssp", np.zeros(0, rg.EDGE_DTYPE))


@pytest.mark.parametrize("algo", ["sssp", "sswp"])
def test_full_width_weights_vs_oracle(algo):
    """uint64 weights (core/type.hpp:25): a fifth of the edges carry weights in
    (2^27, 2^64 - 2^27), some of them parallel edges that differ only in a large
    weight.  Build, a batch of inserts and a batch of deletes (one copy of each
    parallel pair among them) give the oracle's values; every parent weight
    reads back in full, and multiplicities are those of distinct weights."""
    scale = 12
    pairs = gen.rmat(scale, seed=71)
    V = 1 << scale
    rng = np.random.default_rng(71)
    e = gen.edges_with_weights(pairs, True)
    big = rng.random(len(e)) < 0.2
    choices = np.array([(1 << 27) + 1, (1 << 31) + 5, (1 << 32) + 7, 1 << 40, (1 << 63) + 3,
                        (1 << 64) - (1 << 27) - 1], dtype=np.uint64)
    e["data"][big] = rng.choice(choices, int(big.sum()))
    # parallel edges: the same endpoints with a second, different large weight
    par_e = e[big][:300].copy()
    par_e["data"] = np.where(par_e["data"] == choices[3], choices[4], choices[3])
    imported = int(len(e) * 0.9)
    load = np.concatenate([e[:imported], par_e])
    g = rg.Graph(V, len(e) + len(par_e), weighted=True)
    g.add_edges(load)
    og = O.OracleGraph(algo, V, len(e) + len(par_e))
    for x in load:
        og.add_edge(int(x["src"]), int(x["dst"]), int(x["data"]))
    root = gen.max_out_degree_vertex(pairs, V)
    g.build_tree(algo, root)
    og.build_tree(root)
    val, par, pw = g.labels()
    np.testing.assert_array_equal(val, og.labels()[0])
    assert og.validate(val, par, pw, root) == 0
    if algo == "sswp":
        assert (pw > (1 << 31)).any()   # some parents are large-weight edges, read back in full
    # multiplicities of the parallel edges: distinct weights are distinct edges
    # (RMAT repeats endpoints, so some weights recur: the oracle's counts decide)
    want = np.array([og.get_edge_num(int(x["src"]), int(x["dst"]), int(x["data"])) for x in par_e], np.uint64)
    np.testing.assert_array_equal(g.get_edge_num(par_e), want)
    # incremental: insert the rest, then delete the first copies of the parallel pairs and some loaded edges
    adds = e[imported:]
    g.apply_add(algo, adds)
    gone_a = [x for x in adds if og.add_edge(int(x["src"]), int(x["dst"]), int(x["data"])) == 0]
    og.update_tree_add_batch(*(np.array([x[f] for x in gone_a], np.uint64) for f in ("src", "dst", "data")), root)
    dels = np.concatenate([e[big][:300][:150], e[:2000]])
    old = g.apply_del(algo, dels)
    og_old = np.array([og.del_edge(int(x["src"]), int(x["dst"]), int(x["data"])) for x in dels], np.uint64)
    # copies of one edge in one batch may take their old counts in another order
    last = lambda o: sorted(set(zip(dels["src"][o == 1].tolist(), dels["dst"][o == 1].tolist(),
                                    dels["data"][o == 1].tolist())))
    assert last(old) == last(og_old)
    gone = dels[og_old == 1]
    og.update_tree_del_batch(gone["src"], gone["dst"], gone["data"], root)
    val, par, pw = g.labels()
    np.testing.assert_array_equal(val, og.labels()[0])
    assert og.validate(val, par, pw, root) == 0
    g.close()


@pytest.mark.parametrize("algo", ALGOS)
def test_empty_graph_and_isolated_root(algo):
    V = 64
    g = rg.Graph(V, 128, symmetric=algo == "wcc", weighted=WEIGHTED[algo])
    g.build_tree(algo, 5)
    og = oracle_graph(algo, V, np.zeros((0, 2), np.uint64))
    og.build_tree(5)
    np.testing.assert_array_equal(g.values(), og.labels()[0])
    # first edge ever, then its removal
    e = edges_of(algo, np.array([[5, 9]], np.uint64))
    g.apply_add(algo, e, algo != "wcc")
    og.add_edge(5, 9, int(e["data"][0]))
    og.update_tree_add(5, 9, int(e["data"][0]), 5)
    np.testing.assert_array_equal(g.values(), og.labels()[0])
    g.apply_del(algo, e, algo != "wcc")
    og.del_edge(5, 9, int(e["data"][0]))
    og.update_tree_del(5, 9, int(e["data"][0]), 5)
    np.testing.assert_array_equal(g.values(), og.labels()[0])


@pytest.mark.parametrize("algo", ALGOS)
def test_insert_then_delete_restores_values(algo):
    """Size-independent property: a batch inserted and then deleted leaves the
    values exactly where they were."""
    scale = 16
    pairs = gen.rmat(scale, seed=2)
    V = 1 << scale
    base, extra = pairs[:800000], pairs[800000:900000]
    g = gpu_graph(algo, V, base, hint=len(pairs))
    g.build_tree(algo, 0)
    before = g.values()
    d = algo != "wcc"
    old = g.apply_add_pairs(algo, extra, d, want_old=True)
    mid = g.values()
    g.build_tree(algo, 0)
    np.testing.assert_array_equal(g.values(), mid)   # incremental == from scratch
    g.apply_del_pairs(algo, extra, d)
    np.testing.assert_array_equal(g.values(), before)
    assert old is not None


def test_trace_modified_lists_changed_vertices():
    pairs = gen.rmat(12, seed=8)
    V = 4096
    g = gpu_graph("sssp", V, pairs[:60000], trace=True)
    g.build_tree("sssp", 0)
    before = g.values()
    g.clear_modified()
    g.apply_add_pairs("sssp", pairs[60000:60100])
    after = g.values()
    mod = set(g.get_modified().tolist())
    changed = set(np.nonzero(before != after)[0].tolist())
    assert changed <= mod


def test_pool_compaction_under_churn():
    """Many small insert batches make segments grow repeatedly; the abandoned
    regions exhaust the pool and it must be compacted in place of failing."""
    pairs = gen.rmat(12, seed=13)
    V = 4096
    g = rg.Graph(V, len(pairs), weighted=True)
    for lo in range(0, len(pairs), 1024):
        g.add_pairs(pairs[lo:lo + 1024], want_old=False)
    og = oracle_graph("sssp", V, pairs)
    g.build_tree("sssp", 0)
    og.build_tree(0)
    np.testing.assert_array_equal(g.values(), og.labels()[0])
    check_tree(g, og)


def test_pool_exhaustion_is_a_status():
    """A hint far below the real edge count ends in RG_ENOSPACE, not a fault."""
    pairs = gen.rmat(12, seed=13)
    g = rg.Graph(4096, 1000, weighted=True)
    with pytest.raises(rg.RGError) as ei:
        g.add_pairs(pairs, want_old=False)
    assert ei.value.status == 5


@pytest.mark.parametrize("algo", ALGOS)
@pytest.mark.parametrize("batch", [1, 37, 2048, 3000])
def test_apply_add_del_one_submission(algo, batch):
    """rg_apply_add_del (inserts then deletes of a sliding-window batch, one
    device submission up to 2048 + 2048 edges) gives the oracle's values after
    every batch."""
    scale = 12
    pairs = gen.rmat(scale, seed=31)
    V = 1 << scale
    imported = int(len(pairs) * 0.9)
    nb = 6 if batch < 2048 else 2
    g = gpu_graph(algo, V, pairs[:imported], hint=len(pairs), inc_mode=True)
    og = oracle_graph(algo, V, pairs[:imported], inc_mode=True)
    g.build_tree(algo, 0)
    og.build_tree(0)
    ref = og.run_batch(pairs, imported, batch, nb, 0)
    directed = algo != "wcc"
    for k in range(len(ref)):
        lo = imported + k * batch
        hi = min(lo + batch, len(pairs))
        adds = edges_of(algo, pairs[lo:hi])
        dels = edges_of(algo, pairs[lo - imported:hi - imported])
        g.apply_add_del(algo, adds, dels, directed)
        assert g.checksum() == int(ref[k]), f"batch {k}"
    check_tree(g, og)


@pytest.mark.parametrize("algo", ["bfs", "sssp"])
def test_autotune_keeps_values(algo):
    """rg_autotune only picks kernels: the tuned graph's values equal the
    oracle's, and the chosen options are among the candidates."""
    scale = 14
    pairs = gen.rmat(scale, seed=12)
    V = 1 << scale
    root = gen.max_out_degree_vertex(pairs, V)
    imported = int(len(pairs) * 0.95)
    g = gpu_graph(algo, V, pairs[:imported], hint=len(pairs))
    og = oracle_graph(algo, V, pairs[:imported])
    sample = edges_of(algo, pairs[imported:imported + 64])
    rep = g.autotune(algo, root, sample=sample, reps=3)
    assert rep["trials"] >= 10
    assert rep["build_ms_after"] > 0 and rep["apply_ms_after"] > 0
    assert rep["options"]["tiny_edges"] in (0, 8192, 32768, 131072)
    og.build_tree(root)
    np.testing.assert_array_equal(g.values(), og.labels()[0])
    check_tree(g, og, root)


@pytest.mark.parametrize("algo", ALGOS)
@pytest.mark.parametrize("cluster_edges", [0, 16384, 1 << 20])
def test_cluster_levels_in_builds_and_batches(algo, cluster_edges):
    """Mid-size frontiers run in one thread-block cluster (RG_OPT_CLUSTER_EDGES):
    off, with a slot limit that some levels pass (the loop leaves the cluster
    mid-way and the level loop carries on), and for every level that fits.
    A build, then sliding-window batches whose repairs use the same loop,
    match the oracle after every batch; the level trace stays in order."""
    scale = 14
    pairs = gen.rmat(scale, seed=71)
    V = 1 << scale
    imported = int(len(pairs) * 0.9)
    directed = algo != "wcc"
    root = 0 if algo == "wcc" else gen.max_out_degree_vertex(pairs[:imported], V)
    g = gpu_graph(algo, V, pairs[:imported], hint=len(pairs), inc_mode=True)
    g.set_option("cluster_edges", cluster_edges)
    g.set_option("fused_max", 0)   # every batch through the grid-wide kernels and the level loop
    og = oracle_graph(algo, V, pairs[:imported], inc_mode=True)
    og.build_tree(root)
    g.build_tree(algo, root)
    np.testing.assert_array_equal(g.values(), og.labels()[0])
    assert (g.level_device_times() >= 0).all()
    batch, nb = 2000, 5
    ref = og.run_batch(pairs, imported, batch, nb, root)
    e = edges_of(algo, pairs)
    for k in range(nb):
        lo = imported + k * batch
        g.apply_add(algo, e[lo:lo + batch], directed)
        g.apply_del(algo, e[lo - imported:lo - imported + batch], directed)
        assert g.checksum() == int(ref[k]), f"batch {k}"
    val, par, pw = g.labels()
    assert og.validate(val, par, pw, root) == 0
    g.close()
