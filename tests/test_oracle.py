"""The CPU oracle (oracle/bfs_oracle.c) pinned against the reference's own
SimpleReferenceBfs: the committed golden fixtures (tests/golden, generated
from the reference by make_golden.py), the compiled reference when present,
and the analytic lattice distances."""
import numpy as np
import pytest

import oracle


def test_oracle_matches_golden(golden):
    n_checked = 0
    for name, c in golden.items():
        ro, ci = c["row_offsets"], c["column_indices"]
        for k, s in enumerate(c["sources"]):
            labels, depth = oracle.bfs(ro, ci, int(s))
            assert oracle.compare_labels(labels, c[f"labels{k}"]) == -1, name
            assert depth == int(c[f"depth{k}"]), name
            n_checked += 1
    assert n_checked >= 15


def _manhattan2d(w, src):
    sy, sx = divmod(src, w)
    y, x = np.divmod(np.arange(w * w), w)
    return (np.abs(y - sy) + np.abs(x - sx)).astype(np.int32)


def test_grid2d_1000_analytic():
    from back40computing_b200 import CsrGraph, BuildGrid2dGraph
    g = CsrGraph()
    BuildGrid2dGraph(1000, g)
    assert g.nodes == 1_000_000 and g.edges == 4_996_000
    labels, depth = oracle.bfs(g.row_offsets, g.column_indices, 0)
    assert np.array_equal(labels, _manhattan2d(1000, 0))
    assert depth == 1999  # max distance 1998, search depth = max label + 1
    nv, ev = oracle.visited_stats(g.row_offsets, labels)
    assert nv == 1_000_000 and ev == 4_996_000


def test_grid3d_analytic_center():
    from back40computing_b200 import CsrGraph, BuildGrid3dGraph
    w = 32
    g = CsrGraph()
    BuildGrid3dGraph(w, g)
    c = w // 2
    src = c * w * w + c * w + c
    labels, depth = oracle.bfs(g.row_offsets, g.column_indices, src)
    z, rem = np.divmod(np.arange(w ** 3), w * w)
    y, x = np.divmod(rem, w)
    expect = (np.abs(z - c) + np.abs(y - c) + np.abs(x - c)).astype(np.int32)
    assert np.array_equal(labels, expect)
    assert depth == int(expect.max()) + 1


def test_depth_limited_oracle(golden):
    c = golden["grid2d_16"]
    full, _ = oracle.bfs(c["row_offsets"], c["column_indices"], 0)
    lim, _ = oracle.bfs(c["row_offsets"], c["column_indices"], 0, depth_limit=5)
    assert np.array_equal(lim, np.where(full <= 5, full, -1))


def test_predecessor_validator_catches_planted_errors(golden):
    c = golden["rmat_s10_ef8_u"]
    ro, ci = c["row_offsets"], c["column_indices"]
    s = int(c["sources"][0])
    dist, _ = oracle.bfs(ro, ci, s)
    # a valid tree: for every reached v != s pick a neighbour one level up
    preds = np.full(dist.size, -1, np.int32)
    preds[s] = -2
    for v in np.flatnonzero(dist > 0):
        for u in ci[ro[v]:ro[v + 1]]:  # undirected graph: neighbours of v include its parents
            if dist[u] == dist[v] - 1:
                preds[v] = u
                break
    assert oracle.check_predecessors(ro, ci, dist, preds) == (-1, 0)
    v = int(np.flatnonzero(dist == 2)[0])
    bad = preds.copy()
    bad[v] = s  # two levels up
    assert oracle.check_predecessors(ro, ci, dist, bad)[0] == v
    bad = preds.copy()
    bad[v] = -1  # parentless but reached
    assert oracle.check_predecessors(ro, ci, dist, bad) == (v, 1)


@pytest.mark.skipif(not oracle.have_ref(), reason="reference harness not built")
@pytest.mark.parametrize("kind,args", [
    ("grid2d", (33,)), ("grid3d", (9,)), ("rmat", (2048, 16384, 1, 0.57, 0.19, 0.19, 5)),
    ("random", (3000, 9000, 0, 7)), ("rr", (2000, 3, 11)),
])
def test_oracle_matches_compiled_reference(kind, args):
    ro, ci = oracle.ref_build(kind, *args)
    rng = np.random.default_rng(1)
    for s in rng.integers(0, ro.size - 1, size=4):
        rl, rd, _ = oracle.ref_bfs(ro, ci, int(s))
        ol, od = oracle.bfs(ro, ci, int(s))
        assert oracle.compare_labels(ol, rl) == -1
        assert od == rd
