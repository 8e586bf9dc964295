"""Served mode (rg_server_*): every result equals the oracle's for the graph
after the served updates, whether an instance runs alone or in a mix of
instances, batched or one update at a time."""
import numpy as np
import pytest

import risgraph_b200 as rg
from risgraph_b200 import gen

from helpers import WEIGHTED, gpu_graph, oracle_graph

pytestmark = pytest.mark.gpu


def make_instance(algo, scale, seed, rate=0.9):
    pairs = gen.rmat(scale, seed=seed)
    V = 1 << scale
    imported = int(len(pairs) * rate)
    root = gen.max_out_degree_vertex(pairs, V)
    g = gpu_graph(algo, V, pairs[:imported], hint=len(pairs), inc_mode=True)
    g.build_tree(algo, root)
    return dict(algo=algo, V=V, pairs=pairs, imported=imported, root=root, g=g)


def expected_values(inst, adds, dels):
    """Values of the graph after `adds` inserts and `dels` deletes of the
    sliding window: the loaded prefix minus the first `dels` pairs plus the
    next `adds` pairs."""
    p, imp = inst["pairs"], inst["imported"]
    final = np.concatenate([p[dels:imp], p[imp:imp + adds]])
    og = oracle_graph(inst["algo"], inst["V"], final)
    og.build_tree(inst["root"])
    return og.labels()[0]


def load_of(inst, instance, clients, max_updates, seed):
    return dict(instance=instance, clients=clients, pairs=inst["pairs"], imported=inst["imported"],
                max_updates=max_updates, duration_s=60.0, think_us=20.0,
                weighted=WEIGHTED[inst["algo"]], seed=seed)


def serve(insts, updates, per_update=False, clients=32):
    with rg.Server(per_update=per_update, max_epoch=4096) as srv:
        ids = [srv.attach(i["g"], directed=i["algo"] != "wcc") for i in insts]
        res = srv.run_load([load_of(i, k, clients, updates, 7 + n) for n, (i, k) in enumerate(zip(insts, ids))])
        st = srv.stats()
        for k in ids:
            srv.detach(k)
    return res, st


def test_alone_and_in_mix_agree():
    updates = 3000
    alone = make_instance("sssp", 13, 5)
    (r_alone,), _ = serve([alone], updates)
    assert r_alone["completed"] == updates and r_alone["failed"] == 0
    v_alone = alone["g"].values()
    np.testing.assert_array_equal(v_alone, expected_values(alone, r_alone["adds"], r_alone["dels"]))

    mix = [make_instance("sssp", 13, 5), make_instance("bfs", 14, 6), make_instance("wcc", 12, 8),
           make_instance("sswp", 11, 9)]
    res, st = serve(mix, updates)
    for inst, r in zip(mix, res):
        assert r["completed"] == updates and r["failed"] == 0
        np.testing.assert_array_equal(inst["g"].values(), expected_values(inst, r["adds"], r["dels"]))
    # the same instance gives the same result alone and in the mix
    np.testing.assert_array_equal(mix[0]["g"].values(), v_alone)
    assert st["completed"] == updates * len(mix)
    assert st["p50_us"] <= st["p99_us"] <= st["p999_us"] <= st["max_us"]


def test_per_update_mode_agrees():
    updates = 400
    inst = make_instance("bfs", 12, 3)
    (r,), st = serve([inst], updates, per_update=True, clients=8)
    assert r["completed"] == updates and r["failed"] == 0
    assert st["largest_epoch"] == 1  # one update per apply
    np.testing.assert_array_equal(inst["g"].values(), expected_values(inst, r["adds"], r["dels"]))


def test_submit_poll_and_delete_then_insert():
    inst = make_instance("sssp", 10, 4)
    g, V = inst["g"], inst["V"]
    # an edge that is not in the graph: delete (no-op) then insert must leave it present
    present = set(map(tuple, inst["pairs"][:inst["imported"]].tolist()))
    a, b = next((u, v) for u in range(1, V) for v in range(V - 1, 0, -1) if (u, v) not in present)
    c, d = 3, 4
    num = g.get_edge_num(np.array([(a, b, gen_w(a, b))], dtype=np.uint64))
    assert num[0] == 0
    reqs = np.zeros(3, dtype=rg.REQUEST_DTYPE)
    reqs[0] = (0, 1, a, b, gen_w(a, b), 100)
    reqs[1] = (0, 0, a, b, gen_w(a, b), 101)
    reqs[2] = (0, 0, c, d, gen_w(c, d), 102)
    with rg.Server(max_epoch=1024) as srv:
        k = srv.attach(g)
        assert k == 0
        srv.submit(reqs)
        srv.drain(60000)
        done = srv.poll()
        assert sorted(done["tag"].tolist()) == [100, 101, 102]
        assert (done["status"] == 0).all()
        assert (done["done_ns"] >= done["submit_ns"]).all()
        with pytest.raises(rg.RGError) as e:
            bad = reqs[:1].copy()
            bad["src"] = V
            srv.submit(bad)
        assert e.value.status == 2  # RG_EINVAL_VID
        with pytest.raises(rg.RGError) as e:
            bad = reqs[:1].copy()
            bad["instance"] = 5
            srv.submit(bad)
        assert e.value.status == 1
        srv.detach(k)
    num = g.get_edge_num(np.array([(a, b, gen_w(a, b)), (c, d, gen_w(c, d))], dtype=np.uint64))
    assert num[0] == 1 and num[1] >= 1
    og = oracle_graph("sssp", V, inst["pairs"][:inst["imported"]])
    og.add_edge(a, b, gen_w(a, b))
    og.add_edge(c, d, gen_w(c, d))
    og.build_tree(inst["root"])
    np.testing.assert_array_equal(g.values(), og.labels()[0])


def test_hbm_admission():
    a = make_instance("bfs", 12, 1)
    b = make_instance("bfs", 12, 2)
    budget = a["g"].device_bytes() + b["g"].device_bytes() // 2
    with rg.Server(hbm_budget_bytes=budget, max_epoch=256) as srv:
        ka = srv.attach(a["g"])
        with pytest.raises(rg.RGError) as e:
            srv.attach(b["g"])
        assert e.value.status == 4  # RG_ENOMEM_HBM
        srv.detach(ka)
        kb = srv.attach(b["g"])  # admitted once memory is free
        srv.detach(kb)


def gen_w(u, v):
    return int(rg.lib().rg_gen_weight(u, v))


def test_open_loop_poisson_load():
    inst = make_instance("wcc", 12, 12)
    with rg.Server(max_epoch=1024) as srv:
        k = srv.attach(inst["g"], directed=False)
        load = load_of(inst, k, 16, 1500, 3)
        load.update(open_loop=1, think_us=200.0)
        r, = srv.run_load([load])
        srv.detach(k)
    assert r["completed"] == 1500 and r["failed"] == 0
    np.testing.assert_array_equal(inst["g"].values(), expected_values(inst, r["adds"], r["dels"]))


def test_attached_graphs_run_no_cluster_levels():
    """A served graph runs without cluster levels (other instances' epochs keep
    SMs busy, and a cluster level waits for a GPC of free SMs); detach gives
    the graph its setting back, and served values still match."""
    inst = make_instance("sssp", 12, 4)
    g = inst["g"]
    g.set_option("cluster_edges", 1 << 20)
    with rg.Server(max_epoch=4096) as srv:
        k = srv.attach(g)
        assert g.get_option("cluster_edges") == 0
        r, = srv.run_load([load_of(inst, k, 16, 2000, 3)])
        srv.detach(k)
    assert g.get_option("cluster_edges") == 1 << 20
    assert r["completed"] == 2000 and r["failed"] == 0
    np.testing.assert_array_equal(g.values(), expected_values(inst, r["adds"], r["dels"]))
