"""Policy autotuner: the best kernel policy per graph class, measured on the GPU.

The reference tunes its kernels at compile time per architecture and problem
size (the KernelPolicy template lists of enactor_contract_expand.cuh:273-376
and peers: CTA size, occupancy, grain, gather thresholds, queue sizing).  Here
the policy is a runtime struct (b40c_bfs_policy), so tuning is a measured
search on the target GPU, cached per graph class in ``tuned_policies.json``
next to this file and looked up at run time by :func:`policy_for`.

Graph classes (from the degree distribution, :func:`classify`):
  * ``lattice-narrow`` -- bounded degree, high diameter, levels of at most a few
    thousand vertices (grid2d, small grid3d): most levels fit one CTA;
  * ``lattice-wide``   -- bounded degree, levels of tens of thousands of vertices
    and more (large grid3d): every level wants the whole grid;
  * ``power-law``  -- heavy-tailed degrees (R-MAT);
  * ``uniform``    -- concentrated degrees, low diameter (random / regular-ish).

Usage on a GPU box:  ``python -m back40computing_b200.autotune``
(rewrites the cache; ``--quick`` tunes on smaller representatives).
"""
from __future__ import annotations

import argparse
import json
import os
import time

import numpy as np

from . import _native as N

CACHE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "tuned_policies.json")
CLASSES = ("lattice-narrow", "lattice-wide", "power-law", "uniform")
# a lattice whose estimated level width (vertices^((d-1)/d), d from the mean
# degree) is at most this is narrow
NARROW_WIDTH = 4096
KINDS = ("direction-optimizing", "expand-contract", "batched")

# knob -> values tried (0 = the library default)
SEARCH_SPACE = {
    "threads": [256, 512, 128],
    "ctas_per_sm": [1, 2, 3, 4],
    "chunk_edges": [512, 1024, 2048],
    "warp_gather_threshold": [32, 64, 128],
    "cta_gather_threshold": [256, 512, 1024],
    "small_frontier_edges": [256, 1024, 2048, 4096, 16384],
    "bottom_up_alpha": [6, 14, 24, 48],
    "bottom_up_beta": [12, 24, 48],
    "bitmask_precheck": [1, -1, 2],
    "warp_cull": [1, -1],
    "subgrid_frontier_edges": [-1, 4096, 16384, 65536],
    "history_cull": [-1, 1],
    "bottom_up_prefetch": [1, -1],
    "warp_contract": [1, -1],
    "warp_bottom_up": [1, -1],
}
# knobs that matter to each kind of search
KNOBS = {
    "direction-optimizing": ["threads", "ctas_per_sm", "chunk_edges", "small_frontier_edges", "subgrid_frontier_edges",
                             "bottom_up_alpha", "bottom_up_beta", "warp_gather_threshold", "bitmask_precheck",
                             "history_cull", "bottom_up_prefetch", "warp_bottom_up"],
    "expand-contract": ["threads", "ctas_per_sm", "chunk_edges", "small_frontier_edges", "subgrid_frontier_edges",
                        "warp_gather_threshold", "cta_gather_threshold", "bitmask_precheck", "warp_cull",
                        "history_cull", "warp_contract"],
    "batched": ["threads", "ctas_per_sm", "bottom_up_alpha"],
}


def classify(graph) -> str:
    """Graph class from the degree distribution of the vertices with edges."""
    deg = np.diff(np.asarray(graph.row_offsets, dtype=np.int64))
    nz = deg[deg > 0]
    if nz.size == 0:
        return "uniform"
    mean = float(nz.mean())
    cv = float(nz.std() / mean)
    mx = int(nz.max())
    if mx <= 8 and cv < 0.35:
        # a d-dimensional mesh has about 2d edges per vertex (plus a self-loop
        # in the reference builders) and levels of about n^((d-1)/d) vertices
        dim = max(1, int(mean / 2 + 0.25))
        width = float(nz.size) ** ((dim - 1) / dim)
        return "lattice-narrow" if width <= NARROW_WIDTH else "lattice-wide"
    if cv > 1.0 or mx > 32 * mean:
        return "power-law"
    return "uniform"


def _policy(d: dict | None) -> N.Policy:
    pol = N.Policy()
    for k, v in (d or {}).items():
        setattr(pol, k, int(v))
    return pol


def load_cache(path: str = CACHE) -> dict:
    try:
        with open(path) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def policy_for(graph_or_class, kind: str = "direction-optimizing", path: str = CACHE) -> N.Policy | None:
    """The tuned policy for a graph (or a class name) and a kind of search, or
    None when the cache has no entry (the library defaults then apply)."""
    cls = graph_or_class if isinstance(graph_or_class, str) else classify(graph_or_class)
    entry = load_cache(path).get("classes", {}).get(cls, {}).get(kind)
    return None if entry is None else _policy(entry["policy"])


# ---- tuning (needs a GPU) -----------------------------------------------------------

def _representatives(quick: bool):
    from .graph import CsrGraph, BuildGrid2dGraph, BuildGrid3dGraph, BuildRmatGraph, BuildRandomRegularishGraph
    reps = {}
    g = CsrGraph()
    BuildGrid2dGraph(256 if quick else 1000, g)
    g2 = CsrGraph()
    BuildGrid3dGraph(32 if quick else 64, g2)
    reps["lattice-narrow"] = [("grid2d", g), ("grid3d-narrow", g2)]
    g = CsrGraph()
    BuildGrid3dGraph(100 if quick else 200, g)
    reps["lattice-wide"] = [("grid3d", g)]
    # power-law and uniform: the sizes searched in practice (the grid size that
    # pays off grows with the graph: a 2^20-vertex graph alone tunes to fewer CTAs
    # than a 2^22 one wants)
    reps["power-law"] = []
    for s in ((14, 16) if quick else (20, 22)):
        g = CsrGraph()
        BuildRmatGraph(1 << s, 16 << s, g, True, 0.57, 0.19, 0.19, seed=1, permute=True)
        reps["power-law"].append((f"rmat{s}", g))
    g = CsrGraph()
    s = 16 if quick else 21
    BuildRandomRegularishGraph(1 << s, 16, g, seed=1, symmetrize=True)
    reps["uniform"] = [(f"rr{s}", g)]
    return reps


def _measure(problem, kind, sources, pol, reps=2) -> float:
    """Mean device ms per search (batched: per batch) over `reps` rounds."""
    from .bfs import ENACTORS
    if kind == "batched":
        problem.msbfs(sources, policy=pol)
        ts = []
        for _ in range(reps):
            problem.msbfs(sources, policy=pol)
            ts.append(problem.recent_search_ms(1)[0])
        return float(np.mean(ts))
    strategy = N.DIRECTION_OPTIMIZING if kind == "direction-optimizing" else N.EXPAND_CONTRACT
    e = ENACTORS[strategy](policy=pol)
    for s in sources[:1]:
        N.check(e._enact(problem, int(s), N.ENACT_FUSED, 0), "enact")
    for _ in range(reps):
        for s in sources:
            N.check(e._enact(problem, int(s), N.ENACT_FUSED, 0), "enact")
    return float(problem.recent_search_ms(reps * len(sources)).mean())


def tune_class(graphs, kind, sources_per_graph=4, passes=2, log=print, start=None,
               knobs=None) -> tuple[dict, float, float]:
    """Coordinate search from the defaults (or from `start`, e.g. the cached
    policy): each knob in turn (of `knobs`, default all the kind's) takes the
    value that minimises the summed time over the class's representatives."""
    from .bfs import CsrProblem
    from .graph import sample_sources
    probs = []
    for name, g in graphs:
        p = CsrProblem.from_graph(g)
        k = 64 if kind == "batched" else sources_per_graph
        probs.append((p, sample_sources(g, k, seed=5)))
        N.check(p.Reset(N.VERTEX_FRONTIERS, 1.3), "Reset")

    def cost(d):
        pol = _policy(d)
        try:
            return sum(_measure(p, kind, s, pol) for p, s in probs)
        except N.B40cError as e:  # an infeasible combination (e.g. occupancy) is skipped
            log(f"    {d}: {e}")
            return float("inf")

    best = dict(start or {})
    base = best_t = cost(best)
    for _ in range(passes):
        changed = False
        for knob in (knobs or KNOBS[kind]):
            if knob not in KNOBS[kind]:
                continue
            for v in SEARCH_SPACE[knob]:
                if best.get(knob) == v:
                    continue
                trial = dict(best, **{knob: v})
                t = cost(trial)
                if t < best_t * 0.985:  # keep a change only when it is clearly faster
                    best, best_t, changed = trial, t, True
                    log(f"    {knob}={v}: {t:.3f} ms")
        if not changed:
            break
    for p, _ in probs:
        p.Destroy()
    return best, base, best_t


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--quick", action="store_true", help="smaller representatives (a fast check)")
    ap.add_argument("--out", default=CACHE)
    ap.add_argument("--classes", default=",".join(CLASSES))
    ap.add_argument("--kinds", default=",".join(KINDS))
    ap.add_argument("--knobs", default="", help="tune only these knobs (comma list), from the cached policy")
    args = ap.parse_args(argv)
    import torch
    torch.cuda.init()
    reps = _representatives(args.quick)
    out = load_cache(args.out) if os.path.exists(args.out) else {}
    out.setdefault("classes", {})
    out["device"] = torch.cuda.get_device_name(0)
    out["generated"] = time.strftime("%Y-%m-%dT%H:%M:%SZ", time.gmtime())
    out["how"] = ("coordinate search over SEARCH_SPACE "
                  + (f"of the knobs {args.knobs} from the cached policy" if args.knobs else "from the library defaults")
                  + "; cost = mean device time per search (per batch for 'batched') summed over the class's "
                  f"representatives; quick={args.quick}")
    for cls in args.classes.split(","):
        for kind in args.kinds.split(","):
            print(f"[{cls} / {kind}]", flush=True)
            knobs = [k for k in args.knobs.split(",") if k] or None
            start = out["classes"].get(cls, {}).get(kind, {}).get("policy") if knobs else None
            best, base, t = tune_class(reps[cls], kind, start=start, knobs=knobs)
            out["classes"].setdefault(cls, {})[kind] = {
                "policy": best, "default_ms": base, "tuned_ms": t,
                "graphs": [name for name, _ in reps[cls]]}
            print(f"  default {base:.3f} ms -> tuned {t:.3f} ms  {best}", flush=True)
            with open(args.out, "w") as f:
                json.dump(out, f, indent=1, sort_keys=True)
    return out


if __name__ == "__main__":
    main()
