#!/usr/bin/env python
"""Full-graph dependency-tree build on RMAT-22: GTEPS through the C ABI.

Workload (one step): build_tree from scratch (core/graph.hpp:873-985) of
SSSP (default; --algo bfs|sssp|sswp|wcc) over a directed RMAT graph of scale 22
(4,194,304 vertices, 67,108,864 edges, a/b/c = .57/.19/.19, duplicates and
self-loops kept, seeded order), weights splitmix64(src<<32|dst) % 255 + 1,
rooted at the highest out-degree vertex.  The graph is resident in HBM; the
edge pool (>0.5 GB) is larger than L2, so no flush is needed between steps.

value  = reached edges / device time per build (GTEPS), CUDA events on the
         stream the library launches on, max over ranks.
e2e    = the same through the public API with the result read back: every
         step calls rg_build_tree and copies the value array into pinned host
         memory; wall clock.
served = (N=1) the served incremental path: closed-loop clients stream sliding-
         window inserts and deletes of an RMAT-24 SSSP instance through the
         rg_server API (host buffers in, completions out); best updates/s at
         p99 <= 1 ms for the batched server and for the plain one-update-per-
         launch path, and their ratio.
--impl reference runs the reference's own CPU build_tree (oracle/_ref, the
reference's core/graph.hpp compiled with an OpenMP stand-in for TBB) on the
host cores.  Multi-GPU: independent replicas, one per rank (the path does not
shard); no collective on the data path.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "updates/s at p99≤1ms (served vs per-update GPU); full-graph GTEPS vs HBM"
WEIGHTED = {"bfs": False, "sssp": True, "sswp": True, "wcc": False}
THROTTLE_BITS = {
    0x1: "gpu_idle", 0x2: "applications_clocks_setting", 0x4: "sw_power_cap", 0x8: "hw_slowdown",
    0x10: "sync_boost", 0x20: "sw_thermal_slowdown", 0x40: "hw_thermal_slowdown",
    0x80: "hw_power_brake_slowdown", 0x100: "display_clock_setting",
}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--scale", type=int, default=22)
    ap.add_argument("--algo", default="sssp", choices=list(WEIGHTED))
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-timeout", type=float, default=240.0)
    ap.add_argument("--served-scale", type=int, default=24, help="RMAT scale of the served instance (0 = skip)")
    ap.add_argument("--served-seconds", type=float, default=1.0, help="load duration per client count")
    ap.add_argument("--think-us", type=float, default=50.0, help="mean exponential think time per client")
    ap.add_argument("--batch-sweep", action="store_true",
                    help="only the batched incremental sweep (SSSP and SSWP, batches 1..100k) on RMAT-<served-scale>")
    ap.add_argument("--served-mix", action="store_true",
                    help="only the six-instance served mix (RMAT 24 SSSP, 23 BFS, 22 WCC, 20 SSSP, 18 BFS, 16 WCC)")
    ap.add_argument("--no-autotune", action="store_true", help="keep the default level-mode options")
    ap.add_argument("--wcc-deletions", action="store_true",
                    help="only incremental WCC with heavy deletion on an ER+RMAT mix of 2^wcc-scale vertices")
    ap.add_argument("--wcc-scale", type=int, default=26)
    ap.add_argument("--wcc-updates", type=int, default=1000000)
    return ap.parse_args()


def workload(args):
    return {"workload": f"full-graph {args.algo.upper()} build_tree, RMAT-{args.scale} "
                        f"(V=2^{args.scale}, E=16*V, a/b/c=.57/.19/.19, seed {args.seed}), "
                        f"weights splitmix64(src<<32|dst)%255+1, root = max out-degree vertex",
            "scale": args.scale, "algo": args.algo, "seed": args.seed,
            "l2": "inputs larger than L2 (edge pool > 126 MB); no flush"}


def make_graph_input(args):
    from risgraph_b200 import gen
    pairs = gen.rmat(args.scale, seed=args.seed)
    V = 1 << args.scale
    root = gen.max_out_degree_vertex(pairs, V)
    return pairs, V, root


def reached_edges(pairs, V, values, algo):
    """Distinct stored edges out of reached vertices (both directions for WCC)."""
    src = pairs[:, 0].astype(np.int64)
    dst = pairs[:, 1].astype(np.int64)
    if algo == "wcc":
        key = np.unique(np.concatenate([src * V + dst, dst * V + src]))
        return int(len(key)), V
    init = {"bfs": 65536, "sssp": 134217728, "sswp": 0}[algo]
    reached = values != init
    key = np.unique(src * V + dst)
    ks = key // V
    return int(reached[ks].sum()), int(reached.sum())


def algorithmic_bytes(V, V_r, E_r, algo):
    s_e = 16 if WEIGHTED[algo] else 8
    return 16 * V + 16 * V_r + E_r * (s_e + 8)


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    def __init__(self, index):
        self.index = index
        self.samples = []
        self.proc = None

    def __enter__(self):
        q = ("clocks.sm,clocks.max.sm,clocks_event_reasons.active")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
            t0 = time.time()
            while not self.samples and time.time() - t0 < 5.0:  # nvidia-smi start-up
                time.sleep(0.02)
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 3:
                try:
                    self.samples.append((float(parts[0]), float(parts[1]), int(parts[2], 16)))
                except ValueError:
                    pass

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = sorted(s[0] for s in self.samples)
        mask = 0
        for s in self.samples:
            mask |= s[2]
        reasons = [n for b, n in THROTTLE_BITS.items() if mask & b and n != "gpu_idle"]
        return {"sm_mhz": sm[len(sm) // 2], "sm_max_mhz": max(s[1] for s in self.samples), "reasons": reasons,
                "samples": len(self.samples)}


def cpu_reference(pairs, V, root, algo, repeats, warmup, timeout):
    """The reference's own build_tree (oracle/_ref) on all host cores."""
    from oracle import oracle as O
    if not O.ref_available():
        return None, "oracle/_ref/ref_driver not built"
    threads = os.cpu_count() or 1
    with tempfile.TemporaryDirectory(prefix="rg_bench_") as tmp:
        path = os.path.join(tmp, "g.bin")
        pairs.tofile(path)
        env = dict(os.environ, OMP_NUM_THREADS=str(threads), OMP_PROC_BIND="true")
        cmd = [O.REF_DRIVER, "build", algo, path, str(V), str(root), os.path.join(tmp, "out"), str(repeats),
               str(warmup)]
        try:
            r = subprocess.run(cmd, capture_output=True, text=True, env=env, timeout=timeout)
        except subprocess.TimeoutExpired:
            return None, f"reference build timed out after {timeout}s"
        if r.returncode != 0:
            return None, f"reference driver failed: {r.stderr[-200:]}"
        info = json.loads(r.stdout.strip().splitlines()[-1])
        vals = np.fromfile(os.path.join(tmp, "out.val"), dtype=np.uint64)
    info["threads"] = threads
    return (info, vals), None


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    pairs, V, root = make_graph_input(args)
    res, err = cpu_reference(pairs, V, root, args.algo, args.steps, args.warmup, 1800)
    if res is None:
        print(json.dumps({"impl": "reference", "unavailable": err}))
        return
    info, vals = res
    E_r, V_r = reached_edges(pairs, V, vals, args.algo)
    t = float(np.mean(info["build_times"]))
    value = E_r / t / 1e9
    line = {"metric": METRIC, "value": value, "unit": "GTEPS", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "u64", "data": "synthetic", "config": workload(args),
            "impl": "reference",
            "cpu_baseline": {"value": value, "unit": "GTEPS", "cores": info["threads"], "kind": "reference",
                             "sample": f"RMAT-{args.scale} {args.algo} build_tree x{args.steps} after "
                                       f"{args.warmup} warm-up (load {info['load_s']:.1f}s untimed)"},
            "e2e": {"value": value, "unit": "GTEPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


def served_leg(args):
    """Served incremental SSSP: closed-loop clients with Poisson think times
    send sliding-window inserts and deletes to a resident RMAT instance; the
    client count doubles until p99 passes 1 ms.  Both the batched server and
    the plain one-update-per-launch path run the same sweep; each reports its
    best updates/s with p99 <= 1 ms.  After the sweeps, the incrementally
    maintained distances must equal a from-scratch build of the final graph."""
    import risgraph_b200 as rg
    from risgraph_b200 import gen
    scale = args.served_scale
    pairs = gen.rmat(scale, seed=args.seed)
    V = 1 << scale
    imported = int(len(pairs) * 0.9)
    root = gen.max_out_degree_vertex(pairs, V)
    g = rg.Graph(V, len(pairs), weighted=True)
    g.add_pairs(pairs[:imported], True, want_old=False)
    g.build_tree("sssp", root)
    offset = 0
    out = {"workload": f"served incremental SSSP, RMAT-{scale} (V=2^{scale}, E=16*V), first 90% loaded, "
                       f"sliding-window insert+delete updates, closed-loop clients with exponential think time "
                       f"{args.think_us:g} us, {args.served_seconds:g} s per client count, clients doubled until "
                       f"p99 > 1 ms", "device_bytes": g.device_bytes()}
    for mode, per_update in (("per_update", True), ("served", False)):
        sweep, best = [], None
        with rg.Server(per_update=per_update, max_epoch=1 << 16, target_epoch_ms=0.4) as srv:
            k = srv.attach(g)
            c = 1
            while c <= 8192:
                r, = srv.run_load([dict(instance=k, clients=c, pairs=pairs, imported=imported,
                                        duration_s=args.served_seconds, think_us=args.think_us, weighted=True,
                                        offset=offset, seed=c)])
                offset += r["adds"] + r["dels"]
                pt = {"clients": c, "updates_per_s": r["updates_per_s"], "p50_us": r["p50_us"],
                      "p99_us": r["p99_us"], "p999_us": r["p999_us"], "mean_epoch": r["mean_epoch"],
                      "failed": r["failed"]}
                sweep.append(pt)
                if r["failed"]:
                    break
                if r["p99_us"] <= 1000.0 and (best is None or r["updates_per_s"] > best["updates_per_s"]):
                    best = pt
                if r["p99_us"] > 1000.0 and c >= 4:
                    break
                c *= 2
            srv.detach(k)
        out[mode] = {"best_at_p99_le_1ms": best, "sweep": sweep}
    inc = g.values()
    g.build_tree("sssp", root)
    out["incremental_equals_rebuild"] = bool(np.array_equal(inc, g.values()))
    out["updates_applied"] = offset
    b0, b1 = out["per_update"]["best_at_p99_le_1ms"], out["served"]["best_at_p99_le_1ms"]
    out["served_over_per_update"] = (b1["updates_per_s"] / b0["updates_per_s"]) if b0 and b1 else None
    g.close()
    return out


def max_over_ranks(x, dist):
    """The slowest rank's time (every rank takes part; NCCL ranks reduce on
    their GPU, gloo ranks on the CPU)."""
    if not dist:
        return float(x)
    import torch
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(x)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_throughput(units_per_rank, world, seconds):
    """Whole-job GTEPS of `world` independent replicas, each processing
    units_per_rank edges, timed by the slowest rank."""
    return units_per_rank * world / seconds / 1e9


def batch_sweep(args):
    """Batched incremental SSSP / SSWP: the first 90% of an RMAT graph loaded,
    then sliding-window batches of 1 .. 100,000 insert+delete pairs through
    rg_apply_add_pairs / rg_apply_del_pairs (host buffers in); pairs/s and the
    per-batch latency, then incremental == rebuild."""
    import risgraph_b200 as rg
    from risgraph_b200 import gen
    scale = args.served_scale
    pairs = gen.rmat(scale, seed=args.seed)
    V = 1 << scale
    E = len(pairs)
    imported = int(E * 0.9)
    root = gen.max_out_degree_vertex(pairs, V)
    out = {"workload": f"batched incremental sliding window, RMAT-{scale}, first 90% loaded", "runs": []}
    for algo in ("sssp", "sswp"):
        g = rg.Graph(V, E, weighted=True)
        g.add_pairs(pairs[:imported], True, want_old=False)
        g.build_tree(algo, root)
        lo = imported
        for b in (1, 10, 100, 1000, 10000, 100000):
            nb = int(min(4000, max(20, 3e6 // b)))
            ts = []
            for _ in range(nb):
                if lo + b > E:
                    break
                t0 = time.perf_counter()
                g.apply_add_pairs(algo, pairs[lo:lo + b])
                g.apply_del_pairs(algo, pairs[lo - imported:lo - imported + b])
                ts.append(time.perf_counter() - t0)
                lo += b
            ts = np.array(ts)
            out["runs"].append({"algo": algo, "batch": b, "batches": len(ts),
                                "pairs_per_s": 2 * b * len(ts) / float(ts.sum()),
                                "p50_ms": float(np.percentile(ts, 50)) * 1e3,
                                "p99_ms": float(np.percentile(ts, 99)) * 1e3})
        inc = g.values()
        g.build_tree(algo, root)
        out[f"{algo}_incremental_equals_rebuild"] = bool(np.array_equal(inc, g.values()))
        g.close()
    return out


def served_mix(args):
    """Six resident instances of uneven size (RMAT 24 SSSP, 23 BFS, 22 WCC,
    20 SSSP, 18 BFS, 16 WCC), admitted against an HBM budget, served together;
    closed-loop clients (exponential think time) split evenly, doubled until
    p99 passes 1 ms; the batched server against the per-update path."""
    import risgraph_b200 as rg
    from risgraph_b200 import gen
    spec = [(24, "sssp"), (23, "bfs"), (22, "wcc"), (20, "sssp"), (18, "bfs"), (16, "wcc")]
    insts = []
    for scale, algo in spec:
        pairs = gen.rmat(scale, seed=scale)
        V = 1 << scale
        imported = int(len(pairs) * 0.9)
        root = gen.max_out_degree_vertex(pairs, V)
        g = rg.Graph(V, len(pairs), symmetric=algo == "wcc", dual=algo != "wcc", weighted=algo == "sssp")
        g.add_pairs(pairs[:imported], algo != "wcc", want_old=False)
        g.build_tree(algo, root)
        insts.append(dict(scale=scale, algo=algo, pairs=pairs, imported=imported, g=g, root=root, offset=0))
    dev = sum(i["g"].device_bytes() for i in insts)
    out = {"workload": "six instances RMAT 24 SSSP, 23 BFS, 22 WCC, 20 SSSP, 18 BFS, 16 WCC, sliding windows, "
                       f"closed-loop clients, think {args.think_us:g} us", "device_bytes": dev}
    for mode, per_update in (("per_update", True), ("served", False)):
        sweep, best = [], None
        with rg.Server(hbm_budget_bytes=int(dev * 1.05), per_update=per_update, max_epoch=1 << 16,
                       target_epoch_ms=0.4) as srv:
            ids = [srv.attach(i["g"], directed=i["algo"] != "wcc") for i in insts]
            per = 1
            while per <= 1024:
                loads = [dict(instance=k, clients=per, pairs=i["pairs"], imported=i["imported"],
                              duration_s=args.served_seconds, think_us=args.think_us, weighted=i["algo"] == "sssp",
                              offset=i["offset"], seed=per) for k, i in zip(ids, insts)]
                res = srv.run_load(loads)
                st = srv.stats(reset=True)
                for i, r in zip(insts, res):
                    i["offset"] += r["adds"] + r["dels"]
                pt = {"clients": 6 * per, "updates_per_s": sum(r["updates_per_s"] for r in res),
                      "p50_us": st["p50_us"], "p99_us": st["p99_us"], "p999_us": st["p999_us"],
                      "per_instance_updates_per_s": [r["updates_per_s"] for r in res]}
                sweep.append(pt)
                if st["p99_us"] <= 1000.0 and (best is None or pt["updates_per_s"] > best["updates_per_s"]):
                    best = pt
                if st["p99_us"] > 1000.0 and per >= 4:
                    break
                per *= 2
            for k in ids:
                srv.detach(k)
        out[mode] = {"best_at_p99_le_1ms": best, "sweep": sweep}
    ok = True
    for i in insts:
        inc = i["g"].values()
        i["g"].build_tree(i["algo"], i["root"])
        ok &= bool(np.array_equal(inc, i["g"].values()))
        i["g"].close()
    out["incremental_equals_rebuild"] = ok
    b0, b1 = out["per_update"]["best_at_p99_le_1ms"], out["served"]["best_at_p99_le_1ms"]
    out["served_over_per_update"] = (b1["updates_per_s"] / b0["updates_per_s"]) if b0 and b1 else None
    return out


def wcc_deletions(args):
    """Incremental WCC with heavy deletion: an undirected graph of 2^s vertices
    and 16 * 2^s edges (half uniform endpoints, half RMAT-s), both directions
    stored; the first 80% loaded; then batches of 1,000 updates (500 inserts of
    the next edges, 500 deletes of which half remove the oldest loaded edges and
    half remove current tree edges (a vertex's parent edge), forcing subtree
    repair), each batch one rg_apply_add_del; min-vertex-id labels checked
    against a rebuild at the end."""
    import ctypes
    import risgraph_b200 as rg
    from risgraph_b200 import gen
    scale = args.wcc_scale
    V = 1 << scale
    E = 16 * V
    t0 = time.time()
    pairs = gen.er_rmat_mix(scale, E, seed=args.seed)
    imported = int(E * 0.8)
    g = rg.Graph(V, E, symmetric=True, dual=False, weighted=False)
    g.add_pairs(pairs[:imported], directed=False, want_old=False)
    load_s = time.time() - t0
    t1 = time.time()
    g.build_tree("wcc", 0)
    build_ms = (time.time() - t1) * 1e3
    rng = np.random.default_rng(args.seed)
    par = np.empty(V, np.uint64)
    L = rg.lib()

    def refresh():
        assert L.rg_get_labels(g._h, None, ctypes.c_void_p(par.ctypes.data), None) == 0
        return np.nonzero(par != V)[0]

    batch, half = 1000, 500
    nb = min(args.wcc_updates // batch, (E - imported) // half)
    ts, recomputes, invalidated = [], 0, 0
    have = refresh()
    for k in range(nb):
        if k % 50 == 0 and k:
            have = refresh()
        lo = imported + k * half
        adds = pairs[lo:lo + half]
        old = pairs[k * (half // 2):(k + 1) * (half // 2)]
        vs = rng.choice(have, half // 2, replace=False) if len(have) >= half // 2 else have
        tree = np.stack([par[vs], vs.astype(np.uint64)], axis=1)
        dels = np.concatenate([old, tree]).astype(np.uint64)
        t = time.perf_counter()
        g.apply_add_del("wcc", adds, dels, directed=False)
        ts.append(time.perf_counter() - t)
        st = g.last_stats()
        recomputes += st["recomputes"]
        invalidated += st["invalidated"]
    ts = np.array(ts)
    inc = g.values()
    g.build_tree("wcc", 0)
    ok = bool(np.array_equal(inc, g.values()))
    out = {"workload": f"incremental WCC, ER+RMAT mix: 2^{scale} vertices, {E} undirected edges (half uniform, "
                       f"half RMAT-{scale}) stored both ways, first 80% loaded, {nb} batches of {batch} updates "
                       f"(500 inserts, 250 oldest-edge deletes, 250 tree-edge deletes)",
           "device_bytes": g.device_bytes(), "load_s": load_s, "build_ms": build_ms, "batches": int(nb),
           "updates_per_s": batch * nb / float(ts.sum()) if nb else None,
           "batch_p50_ms": float(np.percentile(ts, 50)) * 1e3 if nb else None,
           "batch_p99_ms": float(np.percentile(ts, 99)) * 1e3 if nb else None,
           "invalidated_per_batch": invalidated / max(nb, 1), "full_recomputes": recomputes,
           "incremental_equals_rebuild": ok}
    g.close()
    return out


def main():
    args = parse()
    if args.wcc_deletions:
        import torch
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        if int(os.environ.get("RANK", "0")) == 0:
            print(json.dumps({"metric": METRIC, "mode": "wcc_deletions", "data": "synthetic", **wcc_deletions(args)}))
        return
    if args.batch_sweep or args.served_mix:
        import torch
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        if int(os.environ.get("RANK", "0")) == 0:
            res = batch_sweep(args) if args.batch_sweep else served_mix(args)
            print(json.dumps({"metric": METRIC, "mode": "batch_sweep" if args.batch_sweep else "served_mix",
                              "data": "synthetic", **res}))
        return
    if args.impl == "reference":
        return run_reference(args)
    import torch
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    import risgraph_b200 as rg

    pairs, V, root = make_graph_input(args)
    algo = args.algo
    directed = algo != "wcc"
    g = rg.Graph(V, len(pairs), symmetric=not directed, weighted=WEIGHTED[algo])
    g.add_pairs(pairs, directed, want_old=False)
    stream = torch.cuda.Stream()
    g.set_stream(stream.cuda_stream)
    # the level-mode knobs for this graph, picked by the library's autotuner
    tune = g.autotune(algo, root, reps=3) if not args.no_autotune else None

    for _ in range(max(args.warmup, 1)):
        g.build_tree(algo, root)
    values = g.values()
    E_r, V_r = reached_edges(pairs, V, values, algo)

    # timed region: device time with CUDA events on the launching stream
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    l0 = g.launch_count()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        for a, b in ev:
            a.record(stream)
            g.build_tree(algo, root)
            b.record(stream)
        torch.cuda.synchronize()
    if dist:
        dist.barrier()
    launches = g.launch_count() - l0
    times = [a.elapsed_time(b) for a, b in ev]
    total_ms = float(sum(times))
    total_ms = max_over_ranks(total_ms, dist)
    value = replica_throughput(E_r * args.steps, world, total_ms / 1e3)

    # end to end through the API: build + value readback into pinned memory
    host_vals = torch.empty(V, dtype=torch.int64, pin_memory=True).numpy().view(np.uint64)
    import ctypes
    L = rg.lib()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        g.build_tree(algo, root)
        rc = L.rg_get_labels(g._h, ctypes.c_void_p(host_vals.ctypes.data), None, None)
        assert rc == 0
    e2e_s = time.perf_counter() - t0
    e2e_s = max_over_ranks(e2e_s, dist)
    assert np.array_equal(host_vals, values)
    e2e = replica_throughput(E_r * args.steps, world, e2e_s)

    # roofline of the level kernels of one build (every level's mode kernels, timed per level)
    g.profile(True)
    g.profile_read()
    nb = 3
    for i in range(nb):
        if i == 0:
            torch.cuda.nvtx.range_push("rg_build")  # the build an ncu traffic capture selects
        g.build_tree(algo, root)
        if i == 0:
            torch.cuda.nvtx.range_pop()
    plaunch, pms = g.profile_read()
    g.profile(False)
    push_ms_per_build = pms / nb
    alg = algorithmic_bytes(V, V_r, E_r, algo)
    peak, peak_kind = load_peaks()
    achieved = alg / (push_ms_per_build / 1e3) / 1e9
    traffic, traffic_src = None, None
    if algo == "sssp":
        # DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) of every level kernel of one
        # SSSP build, from an ncu capture of the RMAT-21 build (32,130,409 reached edges); the
        # pull levels stream the in-edge copy, so the bytes grow with the reached edges
        traffic = 1_497_410_816 * E_r / 32_130_409
        traffic_src = "ncu capture of one RMAT-21 SSSP build, scaled by reached edges"
    roof = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
            "peak_source": peak_kind, "traffic": traffic, "traffic_unit": "bytes per build",
            "traffic_source": traffic_src,
            "kernel": "level kernels of one build (k_level_begin + the level mode's push/pull kernels, all levels)",
            "algorithmic_bytes": alg, "launches_per_build": plaunch / nb, "kernel_ms_per_build": push_ms_per_build}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        res, err = cpu_reference(pairs, V, root, algo, 2, 1, args.cpu_timeout)
        if res is None:
            cpu = {"value": None, "unit": "GTEPS", "cores": os.cpu_count(), "kind": "reference", "sample": err}
        else:
            info, vals = res
            ok = bool(np.array_equal(vals, values))
            t = float(np.mean(info["build_times"]))
            cpu = {"value": E_r / t / 1e9, "unit": "GTEPS", "cores": info["threads"], "kind": "reference",
                   "sample": f"RMAT-{args.scale} {algo} build_tree x2 after 1 warm-up "
                             f"(load {info['load_s']:.1f}s untimed)", "values_match_gpu": ok}

    g.close()
    served = served_leg(args) if (rank == 0 and world == 1 and args.served_scale) else None

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": "GTEPS", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "u64", "data": "synthetic",
                "config": workload(args), "clocks": clk.summary(),
                "e2e": {"value": e2e, "unit": "GTEPS", "h2d_bytes_per_step": 8, "d2h_bytes_per_step": V * 8},
                "gpu_launches": launches, "roofline": roof, "cpu_baseline": cpu,
                "reached": {"V_r": V_r, "E_r": E_r}, "autotune": tune, "served": served}
        print(json.dumps(line))
    if dist:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
