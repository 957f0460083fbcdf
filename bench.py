#!/usr/bin/env python
"""Benchmark of the B200 BFS path (one JSON line on stdout, rank 0).

Workload (default): plain single-source BFS on an R-MAT graph, scale 22
(4,194,304 vertices), edge factor 16 (67,108,864 undirected edges stored as
134,217,728 directed CSR edges), a/b/c/d = .57/.19/.19/.05, self-loops and
duplicates kept, vertex ids permuted by a seeded permutation; 64 sources
drawn with seed 0 among vertices of nonzero degree, each searched
separately.  One step = the 64 searches.  Inputs (the CSR, 554 MB) are
resident in HBM and larger than L2.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Metric: GTEPS = sum over searches of E_c / device time, E_c = sum of the CSR
degrees of the reached vertices (test/bfs/test_bfs.cu:359-367).  Under
torchrun each rank runs the same workload on its own GPU (replicas: the
search does not shard), value = all ranks' edges / max-over-ranks time.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from concurrent.futures import ThreadPoolExecutor

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "BFS GTEPS on 1 B200 (plain vs 64-source batched); served p50/p99 latency"
STRATEGY_NAMES = ["expand-contract", "contract-expand", "two-phase", "hybrid", "direction-optimizing"]

CONFIGS = {
    "rmat22": dict(kind="rmat", scale=22, ef=16,
                   workload="plain single-source BFS, R-MAT scale 22 edge factor 16 (a=.57 b=.19 c=.19 d=.05), "
                            "ids permuted, 64 seeded sources searched separately"),
    "grid2d1000": dict(kind="grid2d", width=1000,
                       workload="plain single-source BFS, 2D 5-point lattice 1000x1000, source 0"),
    "grid3d256": dict(kind="grid3d", width=256,
                      workload="high-diameter BFS, 3D 7-point lattice 256^3, source = centre"),
    "rmat20": dict(kind="rmat", scale=20, ef=16,
                   workload="plain single-source BFS, R-MAT scale 20 edge factor 16 (small case for profiling)"),
    "random21": dict(kind="rr", scale=21, degree=16,
                     workload="batched BFS, 2^21 vertices x 16 uniform out-neighbours symmetrised, 64 sources"),
}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--config", choices=sorted(CONFIGS), default="rmat22")
    ap.add_argument("--strategy", type=int, default=4,
                    help="0 expand-contract, 1 contract-expand, 2 two-phase, 3 hybrid, 4 direction-optimizing")
    ap.add_argument("--mode", type=int, default=0, help="0 fused (persistent), 1 per-level launches, 2 CUDA graph")
    ap.add_argument("--sources", type=int, default=64)
    ap.add_argument("--levels", type=int, default=0,
                    help="print the per-level records of this many instrumented searches (one JSON line) and exit")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=15.0, help="bound on the CPU-baseline sample")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the batched (random 2^21), lattice (grid2d-1000, grid3d-256) and served measurements")
    ap.add_argument("--extras", default="batched,lattices,served",
                    help="which of the extra measurements to run (comma list of batched, lattices, served)")
    ap.add_argument("--only-extras", action="store_true",
                    help="run just the extra measurements (no single-source line); prints them as one JSON line")
    ap.add_argument("--ablate", action="store_true",
                    help="policy ablations (the reference's gather / cull microbenchmarks, test/bfs/microbench/): "
                         "each knob's variants interleaved on the same searches; prints one JSON line and exits")
    ap.add_argument("--policy", action="append", default=[], metavar="KNOB=VALUE",
                    help="override one field of the single-source search's policy (b40c_bfs_policy), e.g. "
                         "warp_contract=-1; repeatable; recorded in the line's config")
    return ap.parse_args()


def policy_overrides(base, items):
    """The policy `base` (or the library defaults, None) with KNOB=VALUE overrides;
    None when there are none and no base."""
    from back40computing_b200 import _native as N
    if not items:
        return base
    pol = N.Policy()
    if base is not None:
        for f, _ in N.Policy._fields_:
            setattr(pol, f, getattr(base, f))
    names = {f for f, _ in N.Policy._fields_}
    for item in items:
        knob, _, value = item.partition("=")
        if knob not in names or not value.lstrip("-").isdigit():
            raise SystemExit(f"--policy {item!r}: expected KNOB=INT with KNOB one of {sorted(names)}")
        setattr(pol, knob, int(value))
    return pol


def build_graph(cfg_name):
    from back40computing_b200 import CsrGraph, BuildRmatGraph, BuildGrid2dGraph, BuildGrid3dGraph, sample_sources
    cfg = CONFIGS[cfg_name]
    g = CsrGraph()
    if cfg["kind"] == "rmat":
        n = 1 << cfg["scale"]
        BuildRmatGraph(n, cfg["ef"] * n, g, True, 0.57, 0.19, 0.19, seed=0, permute=True)
        return g, None
    if cfg["kind"] == "rr":
        from back40computing_b200 import BuildRandomRegularishGraph
        BuildRandomRegularishGraph(1 << cfg["scale"], cfg["degree"], g, seed=0, symmetrize=True)
        return g, None
    if cfg["kind"] == "grid2d":
        BuildGrid2dGraph(cfg["width"], g)
        return g, np.array([0], np.int32)
    w = cfg["width"]
    BuildGrid3dGraph(w, g)
    c = w // 2
    return g, np.array([c * w * w + c * w + c], np.int32)


def sources_for(g, fixed, count):
    from back40computing_b200 import sample_sources
    if fixed is not None:
        return fixed
    return sample_sources(g, count, seed=0)


def visited(deg, labels):
    reached = labels >= 0 if labels is not None else None
    return int(reached.sum()), int(deg[reached].sum())


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region.

    The sampler starts before the warm-up (nvidia-smi needs a moment before its
    first line) and samples every 20 ms; begin() and stop() bracket the timed
    region on the host clock and only the samples whose own nvidia-smi
    timestamp falls inside it count (its piped output arrives in bursts, so
    arrival times say little).  A region too short for any sample (a few steps
    of a small case) falls back to the samples of the 0.3 s after it, and the
    record says which window it describes."""

    Q = ("timestamp,index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []  # (host monotonic time, csv line)
        self._t = None
        self.t0 = self.t1 = None

    def start(self, ready_s=5.0):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "20"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self._t = threading.Thread(target=self._read, daemon=True)
            self._t.start()
        except OSError:
            self.proc = None
            return
        deadline = time.monotonic() + ready_s
        while not self.lines and time.monotonic() < deadline and self.proc.poll() is None:
            time.sleep(0.01)

    @staticmethod
    def _stamp(line):
        """The sample's own time (nvidia-smi's local timestamp) in seconds since the epoch, or None."""
        import datetime
        try:
            return datetime.datetime.strptime(line.split(",")[0].strip(), "%Y/%m/%d %H:%M:%S.%f").timestamp()
        except ValueError:
            return None

    def _read(self):
        for line in self.proc.stdout:
            line = line.strip()
            t = self._stamp(line)
            self.lines.append((t if t is not None else time.time(), line))

    def begin(self):
        self.t0 = time.time()

    def stop(self):
        if self.proc is None:
            return None
        self.t1 = time.time()
        time.sleep(0.3)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        if self._t:
            self._t.join(timeout=2)
        t0 = self.t0 if self.t0 is not None else self.t1
        inside = [ln for t, ln in self.lines if t0 <= t <= self.t1]
        window = "timed region"
        if not inside:
            inside = [ln for t, ln in self.lines if self.t1 < t <= self.t1 + 0.3]
            window = "0.3 s after the timed region (too short for a sample)"
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in inside:
            f = [x.strip() for x in ln.split(",")][1:]  # past the timestamp
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for k, nm in enumerate(names):
                if f[5 + k].lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm), "window": window}


def measured_peak():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def profiled_traffic(cfg_name, strategy):
    """DRAM bytes per search of the dominant kernel from the committed ncu summary, if any."""
    path = os.path.join(ROOT, "profiles", "ec_kernel_traffic.json")
    try:
        with open(path) as f:
            return json.load(f).get(f"{cfg_name}/{strategy}")
    except (OSError, ValueError):
        return None


def cpu_search_fn():
    """The CPU BFS to time: the reference's SimpleReferenceBfs when its harness
    was built (kind "reference"), else the C restatement (kind "port")."""
    import oracle
    if oracle.have_ref():
        def run(ro, ci, s):
            return oracle.ref_bfs(ro, ci, int(s))[0]
        return run, "reference"

    def run(ro, ci, s):
        return oracle.bfs(ro, ci, int(s))[0]
    return run, "port"


def cpu_baseline(g, srcs, deg, budget_s):
    """Serial CPU BFS on a bounded sample of the sources (one core)."""
    import resource
    run, kind = cpu_search_fn()
    edges, t, used, user = 0, 0.0, 0, 0.0
    for s in srcs:
        u0 = resource.getrusage(resource.RUSAGE_THREAD).ru_utime
        t0 = time.perf_counter()
        labels = run(g.row_offsets, g.column_indices, s)
        t += time.perf_counter() - t0
        user += resource.getrusage(resource.RUSAGE_THREAD).ru_utime - u0
        edges += visited(deg, labels)[1]
        used += 1
        if t >= budget_s:
            break
    return {"value": edges / t / 1e9, "unit": "GTEPS", "cores": 1, "kind": kind,
            "host_cores": os.cpu_count(), "wall_s": t, "user_cpu_s": user,
            "sample": f"{used} of {len(srcs)} sources, serial SimpleReferenceBfs, wall clock ({t:.1f} s)"}


def level_report(problem, enact, srcs):
    """Per-level records of instrumented searches: frontier vertices and edges,
    direction, the level's duration (block 0's start of the level to its start
    of the next) and the CTAs' barrier arrival times within it."""
    problem.set_instrument(True)
    out = []
    for s in srcs:
        enact(s)  # warm
        problem.labels()
        enact(s)
        problem.labels()
        recs = problem.level_records()
        search_us = float(problem.recent_search_ms(1)[0]) * 1e3
        arr = problem.cta_arrivals(64)
        levels = []
        for r in recs:
            k, t0 = r["pass_"], int(r["t_ns"])
            row = arr[k].astype(np.int64) if k < arr.shape[0] else np.zeros(0, np.int64)
            got = row[row > 0] - t0
            lv = {"pass": k, "vertices": int(r["vertices"]), "edges": int(r["edges"]),
                  "bottom_up": bool(r["bottom_up"]), "us": round(r.get("ns", 0) / 1e3, 2)}
            if got.size > 1:
                lv["arrive_us"] = {"median": round(float(np.median(got)) / 1e3, 2),
                                   "max": round(float(got.max()) / 1e3, 2), "ctas": int(got.size)}
            levels.append(lv)
        out.append({"source": int(s), "search_us": round(search_us, 2), "levels": levels})
    problem.set_instrument(False)
    return out


# Policy ablations: (strategy, knob, values).  Each variant changes one knob of
# the tuned policy; the first value of every row is the reference point.
ABLATIONS = [
    (4, "warp_bottom_up", [1, -1]),
    (4, "bottom_up_hub_probes", [1, -1]),
    (4, "bottom_up_defer_frontier", [1, -1]),
    (4, "bottom_up_long_list", [256, 64]),
    (4, "bitmask_precheck", [-1, 1]),
    (4, "history_cull", [-1, 1]),
    (4, "ctas_per_sm", [4, 3, 2]),
    (4, "small_frontier_edges", [1024, 256, 4096]),
    (0, "warp_contract", [1, -1]),
    (0, "queue_allocation", [2, 1]),
    (0, "chunk_edges", [2048, 1024, 512]),
    (0, "warp_gather_threshold", [32, 128]),
    (0, "cta_gather_threshold", [512, 256, 2048]),
    (0, "bitmask_precheck", [1, -1]),
    (0, "warp_cull", [-1, 1]),
    (0, "history_cull", [-1, 1]),
    (0, "ctas_per_sm", [4, 3, 2]),
    (1, "warp_contract", [1, -1]),
    (3, "warp_contract", [1, -1]),
]


def ablate(cfg_name, sources=16, rounds=3):
    """Device time per search of one-knob variants of the tuned policy, the
    variants of a row interleaved round by round on the same sources."""
    from back40computing_b200 import CsrProblem, autotune
    from back40computing_b200 import _native as N
    from back40computing_b200.bfs import ENACTORS
    g, fixed = build_graph(cfg_name)
    srcs = sources_for(g, fixed, sources)
    p = CsrProblem.from_graph(g)
    rows = []
    for strategy, knob, values in ABLATIONS:
        kind = "direction-optimizing" if strategy == 4 else "expand-contract"
        tuned = autotune.policy_for(g, kind)
        enactors = []
        for v in values:
            pol = N.Policy()
            if tuned is not None:
                for f, _ in N.Policy._fields_:
                    setattr(pol, f, getattr(tuned, f))
            setattr(pol, knob, v)
            enactors.append(ENACTORS[strategy](policy=pol))
        N.check(p.Reset(enactors[0].GetFrontierType(), 1.3), "Reset")
        times = [[] for _ in values]
        for e in enactors:  # warm-up
            N.check(e._enact(p, int(srcs[0]), 0, 0))
        for _ in range(rounds):
            for i, e in enumerate(enactors):
                for s in srcs:
                    N.check(e._enact(p, int(s), 0, 0))
                times[i].extend(p.recent_search_ms(len(srcs)).tolist())
        rows.append({"strategy": STRATEGY_NAMES[strategy], "knob": knob,
                     "us_per_search": {str(v): round(float(np.mean(t)) * 1e3, 1) for v, t in zip(values, times)},
                     "median_us": {str(v): round(float(np.median(t)) * 1e3, 1) for v, t in zip(values, times)}})
        print(json.dumps(rows[-1]), file=sys.stderr, flush=True)
    p.Destroy()
    return {"workload": CONFIGS[cfg_name]["workload"], "sources": len(srcs), "rounds": rounds, "ablations": rows}


def max_over_ranks(x, dist=None, device="cuda"):
    """The largest of every rank's x (the job's time is its slowest replica's);
    x itself with one rank."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(x)
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_gteps(edges_per_replica, world, seconds):
    """Whole-job throughput of `world` replicas that each traversed
    edges_per_replica edges, timed as the slowest replica's seconds."""
    return float(edges_per_replica) * world / seconds / 1e9


def workload_config(args, g, sources):
    """The line's `config`: the workload alone, the same for both arms (how a
    search runs goes under the line's `search` key)."""
    return {"workload": CONFIGS[args.config]["workload"], "graph": args.config, "vertices": int(g.nodes),
            "edges": int(g.edges), "sources": int(sources),
            "l2": "inputs larger than L2 (CSR %.0f MB)" % ((g.edges + g.nodes) * 4 / 1e6)}


def run_reference(args, rank):
    """--impl reference: the reference's CPU BFS on the host cores (independent
    searches in parallel threads; ctypes releases the GIL during each call)."""
    if rank != 0:
        return
    g, fixed = build_graph(args.config)
    srcs = sources_for(g, fixed, args.sources)
    deg = np.diff(g.row_offsets).astype(np.int64)
    run, kind = cpu_search_fn()
    threads = max(1, min(os.cpu_count() or 1, 64))
    per_step = list(srcs[:max(1, min(len(srcs), threads))])
    if len(per_step) < threads:
        per_step = (per_step * threads)[:threads]
    ec_cache = {}

    def one(s):
        labels = run(g.row_offsets, g.column_indices, s)
        if s not in ec_cache:
            ec_cache[int(s)] = visited(deg, labels)[1]
        return int(s)

    with ThreadPoolExecutor(max_workers=threads) as ex:
        for _ in range(args.warmup):
            list(ex.map(one, per_step))
        t0 = time.perf_counter()
        for _ in range(args.steps):
            list(ex.map(one, per_step))
        dt = time.perf_counter() - t0
    edges = sum(ec_cache[int(s)] for s in per_step) * args.steps
    value = edges / dt / 1e9
    line = {
        "metric": METRIC, "value": value, "unit": "GTEPS", "impl": "reference", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt / args.steps * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int32",
        "data": "synthetic (seeded generator, no dataset)",
        "config": workload_config(args, g, len(srcs)),
        "search": {"sample_per_step": f"{len(per_step)} searches in parallel threads"},
        "cpu_baseline": {"value": value, "unit": "GTEPS", "cores": threads, "kind": kind,
                         "sample": f"{len(per_step)} independent searches per step on {threads} threads"},
        "e2e": {"value": value, "unit": "GTEPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def batched_extra(steps, warmup):
    """64-source batched search on the random 2^21 x 16 symmetrised graph against 64
    one-at-a-time plain searches (direction-optimizing and expand-contract) on the
    same GPU; every slot's labels and search depth are checked against the oracle.
    Algorithmic bytes of a batch: 4 * sum_v deg(v) * L_v + 4 * sum_s V_c(s), L_v =
    the number of distinct levels at which v is in some source's frontier."""
    import oracle
    from back40computing_b200 import CsrProblem, sample_sources
    from back40computing_b200 import _native as N
    from back40computing_b200.bfs import ENACTORS
    g, _ = build_graph("random21")
    deg = np.diff(g.row_offsets).astype(np.int64)
    srcs = sample_sources(g, 64, seed=0)
    from back40computing_b200 import autotune
    pol = autotune.policy_for(g, "batched")
    p = CsrProblem.from_graph(g)
    p.msbfs(srcs, policy=pol)
    depths = p.msbfs_depths()
    ec, vc = [], []
    levels = np.zeros(g.nodes, np.uint64)
    for slot, (s, want, depth) in enumerate(oracle.bfs_many(g.row_offsets, g.column_indices, srcs)):
        lab = p.labels_of(slot)
        v, e = visited(deg, lab)
        ec.append(e)
        vc.append(v)
        m = lab >= 0
        levels[m] |= np.left_shift(np.uint64(1), lab[m].astype(np.uint64))
        if oracle.compare_labels(lab, want) != -1 or depths[slot] != depth:
            raise SystemExit(f"batched parity failure against the oracle (slot {slot}, source {s})")
    lv = np.bitwise_count(levels).astype(np.int64)
    balg = 4.0 * float((deg * lv).sum()) + 4.0 * float(sum(vc))
    for _ in range(warmup):
        p.msbfs(srcs, policy=pol)
    for _ in range(steps):
        p.msbfs(srcs, policy=pol)
    batch_ms = float(p.recent_search_ms(steps).mean())
    seq = {}
    for st in (4, 0):
        e = ENACTORS[st](policy=autotune.policy_for(g, STRATEGY_NAMES[st]))
        N.check(p.Reset(e.GetFrontierType(), 1.3))
        for s in srcs:
            N.check(e._enact(p, int(s), 0, 0))
        seq[STRATEGY_NAMES[st]] = float(p.recent_search_ms(64).sum())
    total = float(sum(ec))
    best_seq = min(seq.values())
    peak, _ = measured_peak()
    achieved = balg / (batch_ms * 1e-3) / 1e9
    out = {"workload": CONFIGS["random21"]["workload"], "batch_ms": batch_ms,
           "gteps": total / (batch_ms * 1e-3) / 1e9, "queries_per_s": 64 / (batch_ms * 1e-3),
           "sequential_ms": seq, "speedup_vs_best_sequential": best_seq / batch_ms,
           "roofline": {"bytes_per_batch_alg": balg, "achieved": achieved, "peak": peak, "unit": "GB/s",
                        "frac": achieved / peak}}
    p.Destroy()
    return out


SERVED_SET = [("rmat16", dict(kind="rmat", scale=16, ef=16)), ("rmat18", dict(kind="rmat", scale=18, ef=16)),
              ("rmat20", dict(kind="rmat", scale=20, ef=16)), ("rmat22", dict(kind="rmat", scale=22, ef=16)),
              ("grid2d2048", dict(kind="grid2d", width=2048)), ("grid3d128", dict(kind="grid3d", width=128))]
SERVED_BUDGET = 6 << 30  # device bytes the server may hold for the six graphs


def served_extra(resident=None, n_requests=20000, baseline_requests=None, rates=(0.5, 0.75, 0.9),
                 slots=(2, 4)):
    """The query server on the six resident graphs: a seeded request stream
    (graph uniform over the six, source uniform over the vertices of nonzero
    degree of it, depth limit unlimited w.p. 0.8 else uniform in 2..8).
      * capacity: all requests queued at t = 0, queries/s to the last answer,
        for each number of in-flight slots in `slots` (each slot a stream of
        its own with its share of every SM) and, for the first, with every
        batch on the whole device;
      * one at a time: one slot, batch width 1 (a plain direction-optimizing
        search per query, whole device), on the whole stream (or its first
        baseline_requests);
      * latency: Poisson arrivals at fractions of the best capacity, p50/p99 of
        finish - arrival on the server clock."""
    from back40computing_b200 import CsrGraph, BuildRmatGraph, BuildGrid2dGraph, BuildGrid3dGraph, sample_sources
    from back40computing_b200.server import BfsServer, latency_summary
    graphs = []
    for name, cfg in SERVED_SET:
        if resident is not None and name == resident[0]:
            graphs.append(resident[1])
            continue
        g = CsrGraph()
        if cfg["kind"] == "rmat":
            n = 1 << cfg["scale"]
            BuildRmatGraph(n, cfg["ef"] * n, g, True, 0.57, 0.19, 0.19, seed=0, permute=True)
        elif cfg["kind"] == "grid2d":
            BuildGrid2dGraph(cfg["width"], g)
        else:
            BuildGrid3dGraph(cfg["width"], g)
        graphs.append(g)
    rng = np.random.default_rng(0)
    gid = rng.integers(0, len(graphs), n_requests).astype(np.int32)
    src = np.empty(n_requests, np.int32)
    for i, g in enumerate(graphs):
        pool = np.flatnonzero(np.diff(g.row_offsets) > 0).astype(np.int32)  # every vertex with an edge
        sel = gid == i
        src[sel] = pool[rng.integers(0, pool.size, int(sel.sum()))]
    lim = np.where(rng.random(n_requests) < 0.8, -1, rng.integers(2, 9, n_requests)).astype(np.int32)
    baseline_requests = baseline_requests or n_requests

    def run(server, count, arrivals):
        t0 = server.now_ns() + 20_000_000
        tk = server.submit_many(gid[:count], src[:count], lim[:count], t0 + arrivals)
        server.drain()
        return server.results(int(tk[0]), count)

    out = {"graphs": [n for n, _ in SERVED_SET], "budget_bytes": SERVED_BUDGET, "requests": n_requests,
           "sources": "uniform over the vertices of nonzero degree"}
    caps = {}
    for k in slots:
        for share in ((0, -1) if k == slots[0] else (0,)):
            name = f"{k} slots" + (", whole device per batch" if share < 0 else "")
            with BfsServer(memory_budget_bytes=SERVED_BUDGET, max_in_flight=k, ctas_per_sm=share) as srv:
                for g in graphs:
                    srv.add_tuned_graph(g)
                out["widths"] = [srv.graph_info(i)[1] for i in range(len(graphs))]
                out["memory_used_bytes"] = srv.counters()["memory_used_bytes"]
                run(srv, 500, np.zeros(500, np.int64))  # warm-up
                caps[name] = latency_summary(run(srv, n_requests, np.zeros(n_requests, np.int64)))
                caps[name].update(max_in_flight=k, ctas_per_sm=share)
    best = max(caps, key=lambda c: caps[c]["queries_per_s"])
    out["capacity_by_config"] = caps
    out["capacity"] = dict(caps[best], config=best)
    k, share = caps[best]["max_in_flight"], caps[best]["ctas_per_sm"]
    with BfsServer(memory_budget_bytes=SERVED_BUDGET, max_in_flight=k, ctas_per_sm=share) as srv:
        for g in graphs:
            srv.add_tuned_graph(g)
        run(srv, 500, np.zeros(500, np.int64))
        sweep = []
        for f in rates:
            rate = f * out["capacity"]["queries_per_s"]
            gaps = rng.exponential(1e9 / rate, n_requests)
            rec = run(srv, n_requests, np.cumsum(gaps).astype(np.int64))
            sm = latency_summary(rec)
            sm["offered_qps"] = rate
            sm["load"] = f
            sweep.append(sm)
        out["latency_sweep"] = sweep
    with BfsServer(memory_budget_bytes=SERVED_BUDGET, max_batch=1, max_in_flight=1, ctas_per_sm=-1) as one:
        for g in graphs:
            one.add_tuned_graph(g)
        run(one, 50, np.zeros(50, np.int64))
        base = latency_summary(run(one, baseline_requests, np.zeros(baseline_requests, np.int64)))
        base["sample"] = (f"all {n_requests} requests" if baseline_requests == n_requests
                          else f"first {baseline_requests} requests of the stream")
        out["one_at_a_time"] = base
    out["speedup_queries_per_s"] = out["capacity"]["queries_per_s"] / base["queries_per_s"]
    return out


def lattice_extra():
    """grid2d-1000 from the corner and grid3d-256 from the centre: the persistent grid,
    the whole-search CUDA graph and per-level launches (expand-contract, tuned policy)."""
    from back40computing_b200 import CsrProblem, autotune
    from back40computing_b200 import _native as N
    from back40computing_b200.bfs import ENACTORS
    out = {}
    for name in ("grid2d1000", "grid3d256"):
        g, srcs = build_graph(name)
        ec = int(g.edges)  # lattices are connected: every edge is reached
        p = CsrProblem.from_graph(g)
        e = ENACTORS[0](policy=autotune.policy_for(g, "expand-contract"))
        N.check(p.Reset(e.GetFrontierType(), 1.3))
        # lattice BFS distance = L1 distance from the source (no wraparound)
        w, dims = CONFIGS[name]["width"], (2 if name.startswith("grid2d") else 3)
        idx = np.arange(g.nodes, dtype=np.int64)
        want = np.zeros(g.nodes, np.int64)
        for k in range(dims):
            want += np.abs(idx // w ** k % w - int(srcs[0]) // w ** k % w)
        want = want.astype(np.int32)
        res = {}
        for mode, mname in ((0, "fused persistent"), (2, "cuda graph"), (1, "per-level launches")):
            for _ in range(2):
                N.check(e._enact(p, int(srcs[0]), mode, 0))
            ms = float(p.recent_search_ms(1)[0])
            if not np.array_equal(p.labels(), want):
                raise SystemExit(f"{name}: {mname} distances differ from the lattice distances")
            res[mname] = {"ms": ms, "gteps": ec / (ms * 1e-3) / 1e9}
        out[name] = res
        p.Destroy()
    return out


def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank)
        return
    import torch
    import torch.distributed as dist
    from datetime import timedelta
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=timedelta(seconds=300), device_id=torch.device("cuda", local))
    from back40computing_b200 import CsrProblem
    from back40computing_b200 import _native as N
    from back40computing_b200.bfs import ENACTORS

    if args.ablate:
        if rank == 0:
            print(json.dumps(ablate(args.config, min(args.sources, 16), max(args.steps, 2))), flush=True)
        if world > 1:
            dist.destroy_process_group()
        return

    if args.only_extras:
        if rank == 0:
            wanted = set(args.extras.split(","))
            extras = {}
            if "batched" in wanted:
                extras["batched"] = batched_extra(max(args.steps, 3), args.warmup)
            if "lattices" in wanted:
                extras["lattices"] = lattice_extra()
            if "served" in wanted:
                extras["served"] = served_extra()
            print(json.dumps(extras), flush=True)
        if world > 1:
            dist.destroy_process_group()
        return

    g, fixed = build_graph(args.config)
    srcs = sources_for(g, fixed, args.sources)
    deg = np.diff(g.row_offsets).astype(np.int64)
    problem = CsrProblem.from_graph(g, device=local)
    # a dedicated (non-default) stream shared by the library and the timing events
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    problem.set_stream(stream.cuda_stream)
    from back40computing_b200 import autotune
    graph_class = autotune.classify(g)
    kind = {0: "expand-contract", 4: "direction-optimizing"}.get(args.strategy)
    policy = policy_overrides(autotune.policy_for(graph_class, kind) if kind else None, args.policy)
    enactor = ENACTORS[args.strategy](policy=policy)
    N.check(problem.Reset(enactor.GetFrontierType(), 1.3), "Reset")

    def enact(s):
        N.check(enactor._enact(problem, int(s), args.mode, 0), "enact")

    if args.levels:
        if rank == 0:
            print(json.dumps({"workload": CONFIGS[args.config]["workload"], "strategy": kind,
                              "searches": level_report(problem, enact, srcs[:args.levels])}), flush=True)
        problem.Destroy()
        if world > 1:
            dist.destroy_process_group()
        return

    # untimed pass: per-source reached vertices/edges; on rank 0 every source's
    # labels are checked against the oracle (the reference's SimpleReferenceBfs
    # in parallel host threads) before anything is timed
    ec, vc = [], []
    checks = None
    if rank == 0:
        import oracle
        checks = oracle.bfs_many(g.row_offsets, g.column_indices, srcs)
    for s in srcs:
        enact(s)
        labels = problem.labels()
        v, e = visited(deg, labels)
        vc.append(v)
        ec.append(e)
        if checks is not None:
            ref_src, want, _ = next(checks)
            assert ref_src == int(s)
            if oracle.compare_labels(labels, want) != -1:
                raise SystemExit(f"parity failure against the oracle (source {s})")
    ec, vc = np.array(ec, np.int64), np.array(vc, np.int64)

    def step():
        for s in srcs:
            enact(s)

    clocks = ClockSampler(local)
    clocks.start()  # before the warm-up: nvidia-smi takes a moment to print its first sample
    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    clocks.begin()
    ev0.record(stream)
    for _ in range(args.steps):
        step()
    ev1.record(stream)
    torch.cuda.synchronize()
    clk = clocks.stop()
    ms = ev0.elapsed_time(ev1)
    if world > 1:
        ms = max_over_ranks(ms, dist)
        dist.barrier()
    n_timed = min(len(srcs) * args.steps, 256)
    kernel_ms = problem.recent_search_ms(n_timed)
    order = [srcs[(len(srcs) * args.steps - n_timed + i) % len(srcs)] for i in range(n_timed)]
    idx = {int(s): i for i, s in enumerate(srcs)}
    balg = np.array([4 * ec[idx[int(s)]] + 8 * vc[idx[int(s)]] for s in order], np.float64)
    peak, peak_kind = measured_peak()
    achieved = balg.sum() / (kernel_ms.sum() * 1e-3) / 1e9
    value = replica_gteps(float(ec.sum()) * args.steps, world, ms * 1e-3)

    # end to end through the public API: every search's source goes up from pinned
    # host memory and its labels come back into pinned host memory; the read-back
    # of search i (two staging slots) overlaps search i + 1 on the device
    hosts = [torch.empty(g.nodes, dtype=torch.int32, pin_memory=True) for _ in range(2)]
    hviews = [h.numpy() for h in hosts]

    def e2e_pass(steps):
        for _ in range(steps):
            for i, s in enumerate(srcs):
                enact(s)
                N.check(problem.ExtractResultsAsync(hviews[i & 1], i & 1), "ExtractResultsAsync")
        for slot in (0, 1):
            N.check(problem.ExtractWait(slot), "ExtractWait")

    e2e_pass(1)  # untimed: staging buffers, copy stream and host pages warmed
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    e2e_pass(args.steps)
    e2e_s = time.perf_counter() - t0
    if world > 1:
        e2e_s = max_over_ranks(e2e_s, dist)
    e2e = {"value": replica_gteps(float(ec.sum()) * args.steps, world, e2e_s), "unit": "GTEPS",
           "h2d_bytes_per_step": 8 * len(srcs), "d2h_bytes_per_step": 4 * g.nodes * len(srcs)}

    # the same searches through the reference's top-down strategies (what its
    # drop-in callers reach), for comparison: device time per search
    topdown = None
    if args.strategy == 4 and rank == 0:
        topdown = {}
        for st in (0, 1, 3):
            td = ENACTORS[st]()
            N.check(problem.Reset(td.GetFrontierType(), 1.3), "Reset")
            for s in srcs:
                N.check(td._enact(problem, int(s), args.mode, 0))
            tk = problem.recent_search_ms(len(srcs))
            topdown[STRATEGY_NAMES[st]] = {"gteps": float(ec.sum() / (tk.sum() * 1e-3) / 1e9),
                                           "kernel_ms_per_search": float(tk.mean()),
                                           "roofline_frac": float(balg.mean() / (tk.mean() * 1e-3) / 1e9 / peak)}

    extras = {}
    if rank == 0 and world == 1 and not args.no_extras:
        wanted = set(args.extras.split(","))
        if "batched" in wanted:
            extras["batched"] = batched_extra(max(args.steps, 3), args.warmup)
        if "lattices" in wanted:
            extras["lattices"] = lattice_extra()
        if "served" in wanted:
            extras["served"] = served_extra((args.config, g) if args.config in dict(SERVED_SET) else None)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(g, srcs, deg, args.cpu_seconds)
    traffic = profiled_traffic(args.config, STRATEGY_NAMES[args.strategy])
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "GTEPS", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "int32", "data": "synthetic (seeded generator, no dataset)",
            "config": workload_config(args, g, len(srcs)),
            "search": {"searches_per_step": len(srcs), "strategy": STRATEGY_NAMES[args.strategy],
                       "policy": (f"autotuned for class {graph_class}" if policy is not None else "library defaults")
                       + ("".join(f", {x}" for x in args.policy)),
                       "mode": ["fused persistent", "per-level launches", "cuda graph"][args.mode],
                       "parallelism": f"replicas x{world}"},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "peak_kind": peak_kind,
                         "traffic": (traffic or {}).get("dram_bytes_per_search"),
                         "bytes_per_search_alg": float(balg.mean()),
                         "kernel_ms_per_search": float(kernel_ms.mean())},
            "cpu_baseline": cpu, "e2e": e2e, "topdown": topdown,
            "gpu_launches": 2 * len(srcs) * args.steps,
            "clocks": clk,
            **extras,
            "edges_per_search": float(ec.mean()), "search_gteps_mean": float((ec / 1e9).mean()
                                                                              / (kernel_ms.mean() * 1e-3)),
        }
        print(json.dumps(line), flush=True)
    problem.Destroy()
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
