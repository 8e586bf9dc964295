"""Regenerate the golden fixtures in tests/golden/ from the reference itself.

The reference's hot path (core/graph.hpp, compiled unmodified by
oracle/ref/Makefile into oracle/_ref/ref_driver) runs on small seeded RMAT
graphs from risgraph_b200.gen; its per-vertex values and per-step value
checksums are stored here.  The reference ships no golden vectors of its own,
so these fixtures are what pins the CPU oracle port and the CUDA path.

    make -C oracle/ref REF=<reference checkout> && python tests/golden/make_golden.py
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402
from risgraph_b200 import gen  # noqa: E402

CASES = []
for scale, seed in ((10, 3), (12, 1)):
    for algo in ("bfs", "sssp", "sswp", "wcc"):
        CASES.append(dict(scale=scale, seed=seed, algo=algo, mode="build"))
        CASES.append(dict(scale=scale, seed=seed, algo=algo, mode="inc", rate=0.9, steps=1000))
        for b in (10, 100):
            CASES.append(dict(scale=scale, seed=seed, algo=algo, mode="batch", rate=0.9, batch=b, nbatches=20))


def case_name(c):
    n = f"rmat{c['scale']}_s{c['seed']}_{c['algo']}_{c['mode']}"
    if c["mode"] == "batch":
        n += f"_b{c['batch']}"
    return n


def main():
    if not O.ref_available():
        sys.exit("oracle/_ref/ref_driver missing: make -C oracle/ref REF=<reference checkout>")
    index = []
    for c in CASES:
        pairs = gen.rmat(c["scale"], seed=c["seed"])
        V = 1 << c["scale"]
        root = 0
        if c["mode"] == "build":
            info, arr = O.ref_run("build", c["algo"], pairs, V, root)
        elif c["mode"] == "inc":
            info, arr = O.ref_run("inc", c["algo"], pairs, V, root, c["rate"], c["steps"])
        else:
            info, arr = O.ref_run("batch", c["algo"], pairs, V, root, c["rate"], c["batch"], c["nbatches"])
        name = case_name(c)
        meta = dict(c, V=V, root=root, E=len(pairs), pairs_checksum=gen.checksum(pairs.reshape(-1)),
                    ref=info)
        np.savez_compressed(os.path.join(HERE, name + ".npz"), val=arr["val"],
                            sums=arr.get("sums", np.zeros(0, np.uint64)), meta=json.dumps(meta))
        index.append(name)
        print(name, info["checksum"])
    with open(os.path.join(HERE, "index.json"), "w") as f:
        json.dump(index, f, indent=0)


if __name__ == "__main__":
    main()
