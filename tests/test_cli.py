"""The command-line drivers (bfs|sssp|sswp|wcc{,_inc,_inc_batch,_inc_rt}):
same arguments as the reference's, final values equal the oracle's for the
final graph of the sliding window."""
import os
import subprocess

import numpy as np
import pytest

from risgraph_b200 import build as B
from risgraph_b200 import gen

from helpers import oracle_graph
from oracle import oracle as O

BIN = B.BIN


def run(name, args, env=None, check=True):
    e = dict(os.environ)
    e.update(env or {})
    r = subprocess.run([os.path.join(BIN, name)] + [str(a) for a in args], capture_output=True, text=True, env=e,
                       timeout=600)
    if check:
        assert r.returncode == 0, r.stderr[-2000:]
    return r


def test_drivers_built_and_usage():
    for name in B.DRIVER_NAMES:
        assert os.path.islink(os.path.join(BIN, name)), name
    r = run("sssp_inc_rt", [], check=False)
    assert r.returncode == 1 and "usage: " in r.stderr and "graph root imported_rate timeout_ms percent clients" in r.stderr
    r = run("wcc_inc_batch", [], check=False)
    assert r.returncode == 1 and "graph imported_rate batch_size" in r.stderr


def test_facade_header_compiles(tmp_path):
    src = tmp_path / "f.cpp"
    src.write_text('''
#include "risgraph_b200.hpp"
int main() {
  rg::Graph<uint64_t> graph(16, 64, false, true);
  auto labels = graph.alloc_vertex_tree_array<uint64_t>();
  rg::Graph<uint64_t>::edge_type e{1, 2, 3};
  if (!graph.add_edge(e, true)) graph.update_tree_add(rg::SSSP{0}, labels, e, true);
  graph.build_tree(rg::SSSP{0}, labels);
  bool unsafe = graph.need_update_tree_del(rg::SSSP{0}, labels, e, true);
  if (graph.del_edge(e, true) == 1) graph.update_tree_del(rg::SSSP{0}, labels, e, true);
  rg::Graph<void> wcc(16, 64, true, false);
  auto wl = wcc.alloc_vertex_tree_array<uint64_t>();
  wcc.build_tree(rg::WCC{}, wl);
  return (int)labels[0].data + (int)unsafe + (int)wl[1].parent.nbr;
}
''')
    r = subprocess.run(["/usr/bin/g++", "-std=c++17", "-fsyntax-only", "-I" + os.path.join(B.ROOT, "include"),
                        str(src)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


@pytest.mark.gpu
@pytest.mark.parametrize("algo", ["bfs", "sssp", "sswp", "wcc"])
@pytest.mark.parametrize("mode", ["", "_inc", "_inc_batch", "_inc_rt"])
def test_driver_values_match_oracle(tmp_path, algo, mode):
    scale = 10
    pairs = gen.rmat(scale, seed=21)
    path = tmp_path / "g.bin"
    pairs.tofile(path)
    V = int(pairs.max()) + 1  # the drivers' |V| = max id + 1
    root = gen.max_out_degree_vertex(pairs, V)
    rate = 0.9
    args = [path] + ([] if algo == "wcc" else [root])
    if mode:
        args.append(rate)
    if mode == "_inc_batch":
        args.append(100)
    if mode == "_inc_rt":
        args += [10, 0.99, 16]
    out = tmp_path / "vals.bin"
    r = run(algo + mode, args, env={"RG_WEIGHTS": "splitmix", "RG_DUMP_VALUES": str(out)})
    assert "read: " in r.stderr and "|E|=" in r.stderr and "exec: " in r.stderr
    if mode == "_inc_rt":
        assert "Throughput: " in r.stderr and "P99:" in r.stderr
    vals = np.fromfile(out, dtype=np.uint64)
    if mode:
        imported = int(len(pairs) * rate)
        final = pairs[len(pairs) - imported:]
    else:
        final = pairs
    og = oracle_graph(algo, V, final)
    og.build_tree(root)
    np.testing.assert_array_equal(vals, og.labels()[0])


@pytest.mark.gpu
def test_reference_weights_sssp_inc(tmp_path):
    """Default weights are the reference drivers' (src + dst) % 128."""
    pairs = gen.rmat(9, seed=4)
    path = tmp_path / "g.bin"
    pairs.tofile(path)
    V = int(pairs.max()) + 1
    root = gen.max_out_degree_vertex(pairs, V)
    out = tmp_path / "vals.bin"
    run("sssp_inc", [path, root, 0.9], env={"RG_DUMP_VALUES": str(out)})
    imported = int(len(pairs) * 0.9)
    final = pairs[len(pairs) - imported:]
    og = O.OracleGraph("sssp", V, len(final))
    for s, d in final.tolist():
        og.add_edge(s, d, (s + d) % 128)
    og.build_tree(root)
    np.testing.assert_array_equal(np.fromfile(out, dtype=np.uint64), og.labels()[0])


def test_converters(tmp_path):
    """convert_to_binary[_random|_timestamp]: text edge lists to the binary
    format (utils/convert_to_binary*.cpp)."""
    rng = np.random.default_rng(3)
    edges = rng.integers(0, 1 << 40, size=(500, 2), dtype=np.uint64)
    ts = rng.integers(0, 50, size=500, dtype=np.uint64)
    txt = "\n".join(f"{s} {d}" for s, d in edges.tolist()) + "\n"
    txt_t = "\n".join(f"{s}\t{d}\t{t}" for (s, d), t in zip(edges.tolist(), ts.tolist()))

    def conv(name, text, env=None):
        e = dict(os.environ)
        e.update(env or {})
        r = subprocess.run([os.path.join(BIN, name)], input=text.encode(), capture_output=True, env=e, timeout=60)
        assert r.returncode == 0, r.stderr
        return np.frombuffer(r.stdout, dtype=np.uint64).reshape(-1, 2)

    np.testing.assert_array_equal(conv("convert_to_binary", txt), edges)
    u = conv("convert_to_binary_random", txt)
    np.testing.assert_array_equal(u, conv("convert_to_binary_random", txt))  # rand()'s default state
    np.testing.assert_array_equal(np.sort(u.view("u8,u8"), axis=0), np.sort(edges.view("u8,u8"), axis=0))
    a = conv("convert_to_binary_random", txt, {"RG_SHUFFLE_SEED": "7"})
    b = conv("convert_to_binary_random", txt, {"RG_SHUFFLE_SEED": "7"})
    np.testing.assert_array_equal(a, b)  # seeded: reproducible
    assert not np.array_equal(a, edges)
    np.testing.assert_array_equal(np.sort(a.view("u8,u8"), axis=0), np.sort(edges.view("u8,u8"), axis=0))
    order = sorted(range(500), key=lambda i: (int(ts[i]), int(edges[i, 0]), int(edges[i, 1])))
    np.testing.assert_array_equal(conv("convert_to_binary_timestamp", txt_t), edges[order])


REF_BIN = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref")


@pytest.mark.skipif(not os.path.exists(os.path.join(REF_BIN, "convert_to_binary_random")),
                    reason="reference converters not built (oracle/ref/build_ref.sh)")
def test_converters_byte_identical_to_reference(tmp_path):
    """The three converters against the reference's own (utils/convert_to_binary*.cpp,
    compiled unmodified into oracle/_ref): byte-identical output on the same
    input, the unseeded shuffle included (std::random_shuffle, rand()'s default
    state), with duplicates and a timestamp order with ties."""
    rng = np.random.default_rng(11)
    edges = rng.integers(0, 1 << 36, size=(3000, 2), dtype=np.uint64)
    edges[100:200] = edges[0:100]                      # duplicate edges
    ts = rng.integers(0, 40, size=3000, dtype=np.uint64)
    texts = {"convert_to_binary": "\n".join(f"{s} {d}" for s, d in edges.tolist()) + "\n",
             "convert_to_binary_timestamp": "\n".join(f"{s} {d} {t}" for (s, d), t in
                                                      zip(edges.tolist(), ts.tolist())) + "\n"}
    texts["convert_to_binary_random"] = texts["convert_to_binary"]
    for name, text in texts.items():
        ours = subprocess.run([os.path.join(BIN, name)], input=text.encode(), capture_output=True, timeout=60)
        ref = subprocess.run([os.path.join(REF_BIN, name)], input=text.encode(), capture_output=True, timeout=60)
        assert ours.returncode == 0 and ref.returncode == 0
        assert len(ref.stdout) == 16 * len(edges)
        assert ours.stdout == ref.stdout, name
