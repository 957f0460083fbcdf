"""Graph classification and the tuned-policy cache (CPU only)."""
import json

import numpy as np

from back40computing_b200 import CsrGraph, BuildGrid2dGraph, BuildGrid3dGraph, BuildRmatGraph
from back40computing_b200 import BuildRandomRegularishGraph
from back40computing_b200 import autotune


def _g(kind):
    g = CsrGraph()
    if kind == "grid2d":
        BuildGrid2dGraph(60, g)
    elif kind == "grid3d":
        BuildGrid3dGraph(20, g)
    elif kind == "rmat":
        BuildRmatGraph(1 << 12, 1 << 16, g, True, 0.57, 0.19, 0.19, seed=0, permute=True)
    else:
        BuildRandomRegularishGraph(1 << 12, 16, g, seed=0, symmetrize=True)
    return g


def test_classify_builders():
    assert autotune.classify(_g("grid2d")) == "lattice-narrow"
    assert autotune.classify(_g("grid3d")) == "lattice-narrow"
    wide = CsrGraph()
    BuildGrid3dGraph(128, wide)  # levels of ~16k vertices
    assert autotune.classify(wide) == "lattice-wide"
    long2d = CsrGraph()
    BuildGrid2dGraph(1000, long2d)  # levels of at most 1000 vertices
    assert autotune.classify(long2d) == "lattice-narrow"
    assert autotune.classify(_g("rmat")) == "power-law"
    assert autotune.classify(_g("rr")) == "uniform"


def test_policy_lookup(tmp_path):
    path = tmp_path / "cache.json"
    path.write_text(json.dumps({"classes": {"lattice-narrow": {"direction-optimizing": {
        "policy": {"small_frontier_edges": 4096, "ctas_per_sm": 2}}}}}))
    pol = autotune.policy_for(_g("grid2d"), path=str(path))
    assert pol.small_frontier_edges == 4096 and pol.ctas_per_sm == 2 and pol.chunk_edges == 0
    assert autotune.policy_for("power-law", path=str(path)) is None
    assert autotune.policy_for("lattice-narrow", kind="batched", path=str(path)) is None


def test_committed_cache_is_well_formed():
    cache = autotune.load_cache()
    for cls, kinds in cache.get("classes", {}).items():
        assert cls in autotune.CLASSES
        for kind, entry in kinds.items():
            assert kind in autotune.KINDS
            for knob, v in entry["policy"].items():
                assert knob in autotune.SEARCH_SPACE and v in autotune.SEARCH_SPACE[knob]
            assert entry["tuned_ms"] <= entry["default_ms"]
