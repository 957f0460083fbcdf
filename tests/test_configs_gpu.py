"""Parity at the benchmark configurations' full sizes.

Each configuration the benchmark times is checked here against the oracle
(the reference's own SimpleReferenceBfs, run in parallel host threads) or
against the analytic answer of a lattice:
  * R-MAT scale 22 (4,194,304 vertices, 134,217,728 directed edges, ids
    permuted), all 64 benchmark sources, for the direction-optimizing and the
    expand-contract strategies; predecessors on 8 of them;
  * the 3D lattice 256^3 from its centre and the 2D lattice 1000x1000 from
    its corner, in every launch mode;
  * the 64-source batch on the uniform random graph of 2^21 vertices, every
    slot and its search depth.
"""
import numpy as np
import pytest

import oracle
from back40computing_b200 import (CsrGraph, CsrProblem, BuildGrid2dGraph, BuildGrid3dGraph, BuildRmatGraph,
                                  BuildRandomRegularishGraph, sample_sources, autotune, search)
from back40computing_b200 import _native as N
from back40computing_b200.bfs import EXPAND_CONTRACT, DIRECTION_OPTIMIZING, ENACTORS

pytestmark = pytest.mark.gpu

MODES = [N.ENACT_FUSED, N.ENACT_ITERATIVE, N.ENACT_GRAPH]
STRATEGY_NAMES = {EXPAND_CONTRACT: "expand-contract", DIRECTION_OPTIMIZING: "direction-optimizing"}


@pytest.fixture(scope="module")
def rmat22():
    g = CsrGraph()
    BuildRmatGraph(1 << 22, 16 << 22, g, True, 0.57, 0.19, 0.19, seed=0, permute=True)
    return g, sample_sources(g, 64, seed=0)


def _mismatch(got, want):
    bad = oracle.compare_labels(got, want)
    return None if bad == -1 else f"first mismatch at vertex {bad}: got {got[bad]}, want {want[bad]}"


@pytest.mark.parametrize("strategy", [DIRECTION_OPTIMIZING, EXPAND_CONTRACT])
def test_rmat22_all_64_sources(rmat22, strategy):
    g, srcs = rmat22
    pol = autotune.policy_for(g, STRATEGY_NAMES[strategy])
    p = CsrProblem.from_graph(g)
    e = ENACTORS[strategy](policy=pol)
    N.check(p.Reset(e.GetFrontierType(), 1.3))
    for s, want, depth in oracle.bfs_many(g.row_offsets, g.column_indices, srcs):
        N.check(e._enact(p, s, N.ENACT_FUSED, 0))
        got = p.labels()
        err = _mismatch(got, want)
        assert err is None, f"source {s}: {err}"
        assert e.GetStatistics()[1] == depth, f"source {s}: search depth"
    p.Destroy()


@pytest.mark.parametrize("strategy", [DIRECTION_OPTIMIZING, EXPAND_CONTRACT])
def test_rmat22_predecessors(rmat22, strategy):
    """Predecessor mode at full size: every label is a parent exactly one level
    up joined by a real edge (the reference's rule, test_bfs.cu:387-439)."""
    g, srcs = rmat22
    p = CsrProblem.from_graph(g, mark_predecessors=True)
    e = ENACTORS[strategy](policy=autotune.policy_for(g, STRATEGY_NAMES[strategy]))
    N.check(p.Reset(e.GetFrontierType(), 1.3))
    for s, dist, _ in oracle.bfs_many(g.row_offsets, g.column_indices, srcs[::8]):
        N.check(e._enact(p, s, N.ENACT_FUSED, 0))
        preds = p.labels()
        assert preds[s] == -2
        assert oracle.check_predecessors(g.row_offsets, g.column_indices, dist, preds) == (-1, 0), f"source {s}"
        assert np.array_equal(preds >= 0, dist > 0)
    p.Destroy()


def _lattice_distance(width, dims, src_coord):
    idx = np.arange(width ** dims, dtype=np.int64)
    d = np.zeros(idx.size, np.int64)
    for k in range(dims):
        c = (idx // width ** k) % width
        d += np.abs(c - src_coord[k])
    return d.astype(np.int32)


@pytest.mark.parametrize("mode", MODES)
def test_grid3d_256_centre_every_mode(mode):
    w = 256
    g = CsrGraph()
    BuildGrid3dGraph(w, g)
    c = w // 2
    src = c * w * w + c * w + c
    want = _lattice_distance(w, 3, (c, c, c))
    p = CsrProblem.from_graph(g)
    for strategy in (EXPAND_CONTRACT, DIRECTION_OPTIMIZING):
        got = search(p, src, strategy=strategy, mode=mode, policy=autotune.policy_for(g, STRATEGY_NAMES[strategy]))
        assert np.array_equal(got, want), f"{STRATEGY_NAMES[strategy]}: {_mismatch(got, want)}"
        e = ENACTORS[strategy]()
        e._problem = p
        assert e.GetStatistics()[1] == 3 * c + 1  # depths 0..384
    p.Destroy()


@pytest.mark.parametrize("mode", MODES)
def test_grid2d_1000_corner_every_mode(mode):
    g = CsrGraph()
    BuildGrid2dGraph(1000, g)
    want = _lattice_distance(1000, 2, (0, 0))
    p = CsrProblem.from_graph(g)
    got = search(p, 0, strategy=EXPAND_CONTRACT, mode=mode, policy=autotune.policy_for(g, "expand-contract"))
    assert np.array_equal(got, want), _mismatch(got, want)
    p.Destroy()


def test_random21_batched_all_64_slots():
    g = CsrGraph()
    BuildRandomRegularishGraph(1 << 21, 16, g, seed=0, symmetrize=True)
    srcs = sample_sources(g, 64, seed=0)
    p = CsrProblem.from_graph(g)
    p.msbfs(srcs, policy=autotune.policy_for(g, "batched"))
    depths = p.msbfs_depths()
    for slot, (s, want, depth) in enumerate(oracle.bfs_many(g.row_offsets, g.column_indices, srcs)):
        err = _mismatch(p.labels_of(slot), want)
        assert err is None, f"slot {slot} (source {s}): {err}"
        assert depths[slot] == depth, f"slot {slot}: search depth"
    p.Destroy()
