"""The CPU oracle port reproduces the reference's own outputs (golden fixtures
made by tests/golden/make_golden.py from the reference-built oracle)."""
import json
import os

import numpy as np
import pytest

from oracle import oracle as O
from risgraph_b200 import gen

from helpers import oracle_graph

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
NAMES = json.load(open(os.path.join(GOLDEN, "index.json")))


def load(name):
    z = np.load(os.path.join(GOLDEN, name + ".npz"))
    return z["val"], z["sums"], json.loads(str(z["meta"]))


@pytest.mark.parametrize("name", NAMES)
def test_port_matches_reference(name):
    val_ref, sums_ref, m = load(name)
    pairs = gen.rmat(m["scale"], seed=m["seed"])
    assert gen.checksum(pairs.reshape(-1)) == m["pairs_checksum"], "generator drifted"
    V, algo = m["V"], m["algo"]
    if m["mode"] == "build":
        og = oracle_graph(algo, V, pairs)
        og.build_tree(m["root"])
    else:
        imported = int(len(pairs) * m["rate"])
        og = oracle_graph(algo, V, pairs[:imported], inc_mode=True)
        og.build_tree(m["root"])
        if m["mode"] == "inc":
            sums = og.run_inc(pairs, imported, m["steps"], m["root"])
        else:
            sums = og.run_batch(pairs, imported, m["batch"], m["nbatches"], m["root"])
        np.testing.assert_array_equal(sums, sums_ref)
    val, par, pw = og.labels()
    np.testing.assert_array_equal(val, val_ref)
    assert og.validate(val, par, pw, m["root"]) == 0


@pytest.mark.parametrize("algo", ["bfs", "sssp", "sswp", "wcc"])
def test_validator_catches_planted_mistakes(algo):
    """The structural tree check rejects a wrong value, a broken parent edge
    and a parent cycle (mistakes planted in the oracle's own output)."""
    pairs = gen.rmat(10, seed=3)
    og = oracle_graph(algo, 1024, pairs)
    og.build_tree(0)
    val, par, pw = og.labels()
    assert og.validate(val, par, pw) == 0
    kids = np.nonzero(par < 1024)[0]
    v = int(kids[len(kids) // 2])
    bad = val.copy(); bad[v] += 1
    assert og.validate(bad, par, pw) != 0
    badp = par.copy(); badp[v] = (int(par[v]) + 1) % 1024
    assert og.validate(val, badp, pw) != 0
    # two vertices pointing at each other
    a, b = int(kids[0]), int(kids[1])
    cyc = par.copy(); cyc[a] = b; cyc[b] = a
    assert og.validate(val, cyc, pw) != 0


def test_reference_oracle_runs_if_built():
    if not O.ref_available():
        pytest.skip("reference oracle binary not built here")
    pairs = gen.rmat(10, seed=3)
    info, arr = O.ref_run("build", "sssp", pairs, 1024, 0)
    og = oracle_graph("sssp", 1024, pairs)
    og.build_tree(0)
    np.testing.assert_array_equal(og.labels()[0], arr["val"])
